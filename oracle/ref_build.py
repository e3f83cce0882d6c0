"""Build recipe for the reference's own kernel sources as host code (the ``oracle/_ref`` checker).

TEST INFRASTRUCTURE ONLY.  SDPviBe ships its elementwise MPF kernels and its Cholesky base case as
CUDA C strings compiled at run time through CuPy/NVRTC (``sdpvibe/mpf.py:23-141``,
``sdpvibe/basecase.py:13-246``).  This recipe reads those strings where they lie in the reference
tree (without importing the reference), applies the same placeholder substitutions the reference
applies (``mpf.py:149``, ``basecase.py:254``), compiles them with g++ against
``ref_host_shim.h`` and writes the shared objects to ``oracle/_ref/`` (git-ignored).  It also
provides a minimal ``cupy`` stand-in so the reference's own Python (run on CPU torch) can launch
those kernels while generating golden vectors.

Nothing here is part of the product; only tests, ``smoke()`` and the CPU-baseline leg of
``bench.py`` may use it.
"""
import ast
import ctypes
import hashlib
import os
import re
import subprocess
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
# The reference tree is named by SDPV_REFERENCE_ROOT (no default): without it the checkers that need the
# reference's sources are not built, and extract_src refuses with a message.
REFERENCE_ROOT = os.environ.get("SDPV_REFERENCE_ROOT")

_KERNEL_RE = re.compile(r'extern\s+"C"\s+__global__\s+void\s+(\w+)\s*\(([^)]*)\)', re.S)


def extract_src(relpath, name="_SRC"):
    """Return the string literal assigned to `name` in a reference module (parsed, not imported)."""
    if not REFERENCE_ROOT:
        raise RuntimeError("set SDPV_REFERENCE_ROOT to the reference (SDPviBe) source tree")
    path = os.path.join(REFERENCE_ROOT, relpath)
    tree = ast.parse(open(path).read(), path)
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == name for t in node.targets):
            return node.value.value
    raise KeyError(f"{name} not found in {path}")


def _params(text):
    out = []
    for p in text.split(","):
        p = " ".join(p.split())
        if not p:
            continue
        m = re.match(r"(.*?)(\w+)$", p)
        ctype, ident = m.group(1).strip(), m.group(2)
        out.append((ctype, ident))
    return out


def _ctypes_of(ctype):
    if "*" in ctype:
        return ctypes.c_void_p
    base = ctype.replace("const", "").strip()
    return {"int": ctypes.c_int32, "i64": ctypes.c_int64, "long long": ctypes.c_int64,
            "u32": ctypes.c_uint32, "unsigned": ctypes.c_uint32, "unsigned int": ctypes.c_uint32}[base]


def _launchers(code):
    coop = ("__syncthreads" in code) or ("__syncwarp" in code)
    lines, sigs = [], {}
    for name, ptext in _KERNEL_RE.findall(code):
        ps = _params(ptext)
        decl = ", ".join(f"{t} {i}" for t, i in ps)
        args = ", ".join(i for _, i in ps)
        lines.append(f'extern "C" void sdpvref_launch_{name}(unsigned grid, unsigned block'
                     f'{", " + decl if decl else ""}) {{\n'
                     f'  sdpvref_run(grid, block, {"true" if coop else "false"}, [&] {{ {name}({args}); }});\n}}')
        sigs[name] = [_ctypes_of(t) for t, _ in ps]
    return "\n".join(lines), sigs


def compile_code(code, tag="mod"):
    """Compile one reference kernel-source string (placeholders already substituted) -> (CDLL, signatures)."""
    os.makedirs(REF_OUT, exist_ok=True)
    launch, sigs = _launchers(code)
    full = f'#include "{os.path.join(HERE, "ref_host_shim.h")}"\n{code}\n{launch}\n'
    h = hashlib.sha1(full.encode()).hexdigest()[:16]
    so = os.path.join(REF_OUT, f"{tag}_{h}.so")
    if not os.path.exists(so):
        src = os.path.join(REF_OUT, f"{tag}_{h}.cpp")
        with open(src, "w") as f:
            f.write(full)
        tmp = so + f".tmp{os.getpid()}"
        subprocess.check_call(["g++", "-O2", "-std=c++20", "-shared", "-fPIC", "-pthread", "-w",
                               "-o", tmp, src])
        os.replace(tmp, so)
    lib = ctypes.CDLL(so)
    for name, argt in sigs.items():
        fn = getattr(lib, f"sdpvref_launch_{name}")
        fn.argtypes = [ctypes.c_uint32, ctypes.c_uint32] + argt
        fn.restype = None
    return lib, sigs


# ------------------------------------------------------------------ cupy stand-in (golden generation)
def _arg(a):
    import numpy as np
    import torch
    if torch.is_tensor(a):
        assert a.device.type == "cpu" and a.is_contiguous()
        return a.data_ptr()
    if isinstance(a, (np.integer,)):
        return int(a)
    return a


class _Kernel:
    def __init__(self, lib, name):
        self.fn = getattr(lib, f"sdpvref_launch_{name}")

    def __call__(self, grid, block, args):
        self.fn(int(grid[0]), int(block[0]), *[_arg(a) for a in args])


class RawModule:
    """Stand-in for cupy.RawModule: compiles the kernel string for the host."""

    def __init__(self, code, options=()):
        self.lib, _ = compile_code(code, "rt")

    def get_function(self, name):
        return _Kernel(self.lib, name)


def install_cupy_shim():
    """Register a fake `cupy` exposing what the reference uses (RawModule, from_dlpack, int32/int64)."""
    import numpy as np
    m = types.ModuleType("cupy")
    m.RawModule = RawModule
    m.from_dlpack = lambda t: t
    m.int32 = np.int32
    m.int64 = np.int64
    sys.modules["cupy"] = m
    return m


# ------------------------------------------------------------------ prebuilt checkers for the tests
def mpf_code(L):
    """sdpvibe/mpf.py:146-151 substitutions for limb count L."""
    return extract_src("sdpvibe/mpf.py").replace("__L__", str(L)).replace("__LMAX__", "160")


def basecase_code(WL, LF, BT):
    """sdpvibe/basecase.py:251-256 substitutions."""
    return (extract_src("sdpvibe/basecase.py").replace("__WL__", str(WL)).replace("__LF__", str(LF))
            .replace("__BT__", str(BT)))


PREBUILT_MPF_L = (1, 2, 4, 10, 24, 26, 27, 28, 34, 64)
PREBUILT_BASECASE = ((24 + 24, 24, 32), (26 + 24, 26, 32), (4 + 24, 4, 32), (34 + 24, 34, 32))


def prebuilt_path(kind, *key):
    return os.path.join(REF_OUT, f"{kind}_" + "_".join(map(str, key)) + ".so")


def build_prebuilt():
    """Compile the reference kernels for the limb counts the tests use (needs the reference tree)."""
    if not REFERENCE_ROOT or not os.path.isdir(REFERENCE_ROOT):
        return False
    os.makedirs(REF_OUT, exist_ok=True)
    for L in PREBUILT_MPF_L:
        _link(compile_code(mpf_code(L), f"mpfsrc_L{L}"), prebuilt_path("mpf", L))
    for key in PREBUILT_BASECASE:
        _link(compile_code(basecase_code(*key), "basesrc_" + "_".join(map(str, key))),
              prebuilt_path("basecase", *key))
    return True


def _link(res, dst):
    lib, _ = res
    src = lib._name
    if os.path.abspath(src) != os.path.abspath(dst):
        import shutil
        shutil.copyfile(src, dst + ".tmp")
        os.replace(dst + ".tmp", dst)




# ------------------------------------------------------------------ the reference's CPU timing baseline
MPF_BASELINE = os.path.join(REF_OUT, "mpf_baseline")


def build_cpu_baseline():
    """cpu_baseline/mpf_baseline.c (GMP mpf + OpenMP, the reference's CPU comparison) compiled where it
    lies, as the reference documents: gcc -O2 -fopenmp mpf_baseline.c -l:libgmp.so.10 -lm."""
    src = os.path.join(REFERENCE_ROOT, "cpu_baseline", "mpf_baseline.c") if REFERENCE_ROOT else ""
    if not src or not os.path.exists(src):
        return os.path.exists(MPF_BASELINE)
    os.makedirs(REF_OUT, exist_ok=True)
    if os.path.exists(MPF_BASELINE) and os.path.getmtime(MPF_BASELINE) >= os.path.getmtime(src):
        return True
    tmp = MPF_BASELINE + ".tmp"
    subprocess.check_call(["gcc", "-O2", "-fopenmp", src, "-o", tmp, "-l:libgmp.so.10", "-lm"])
    os.replace(tmp, MPF_BASELINE)
    return True


if __name__ == "__main__":
    print("kernel checkers:", "built" if build_prebuilt() else "reference tree absent")
    print("cpu baseline:", "built" if build_cpu_baseline() else "reference tree absent")
