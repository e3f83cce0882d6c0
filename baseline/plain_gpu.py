"""The "plain per-bucket GPU path": the reference SDPviBe's own solver and kernels on this GPU.

The reference (installed from its source tree into baseline/_ref, which is not part of this repository)
runs unmodified through its own Python API -- its Triton kernels JIT-compiled for this GPU, its CUDA C
kernel strings, its per-bucket Cholesky recursion, its chunk streams -- with two stand-ins around it,
neither of which touches its arithmetic:

* ``cupy``: the reference compiles its CUDA C strings with CuPy/NVRTC (sdpvibe/mpf.py:146-151,
  sdpvibe/basecase.py:251-256).  CuPy is not installed here; the stand-in compiles the same strings with
  nvcc for this GPU (cubin, loaded and launched through the CUDA driver API on torch's current stream), and
  ``from_dlpack`` passes the torch tensor through.
* the CRT digit-sum kernel (sdpvibe/rns.py:138-159) calls ``tl.dot(int8, int8, int32 accumulator)``
  without ``out_dtype``, which Triton 3.6 rejects; its source is taken from the installed module, the two
  ``tl.dot`` calls get ``out_dtype=tl.int32`` (the type the accumulator already has), and the compiled
  kernel replaces the module attribute.  The installed files are not edited.

``run_plain_solver`` builds the reference's SDP object from the same block data as this repository's
Ising-structured benchmark SDP and times the reference's own ``Solver.run``.
"""
import ctypes
import hashlib
import inspect
import os
import subprocess
import sys
import tempfile
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SITE = os.path.join(HERE, "_ref")
CACHE = os.path.join(tempfile.gettempdir(), "sdpv_plain_cubins")


# ------------------------------------------------------------------ cupy stand-in (nvcc + driver API)
class _Driver:
    def __init__(self):
        self.lib = ctypes.CDLL("libcuda.so.1")
        v = ctypes.c_void_p
        self.lib.cuModuleLoadData.argtypes = [ctypes.POINTER(v), ctypes.c_char_p]
        self.lib.cuModuleGetFunction.argtypes = [ctypes.POINTER(v), v, ctypes.c_char_p]
        self.lib.cuLaunchKernel.argtypes = [v, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                                            ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, v, ctypes.POINTER(v), v]

    def check(self, r, what):
        if r != 0:
            raise RuntimeError(f"{what}: CUDA driver error {r}")


_DRV = None


def _arch():
    import torch
    major, minor = torch.cuda.get_device_capability()
    return f"sm_{major}{minor}" + ("a" if major >= 9 else "")


class _Kernel:
    def __init__(self, fn):
        self.fn = fn

    def __call__(self, grid, block, args, shared_mem=0, stream=None):
        import torch
        vals = []
        for a in args:
            if torch.is_tensor(a):
                assert a.is_cuda and a.is_contiguous()
                vals.append(ctypes.c_void_p(a.data_ptr()))
            elif isinstance(a, np.int32):
                vals.append(ctypes.c_int32(int(a)))
            elif isinstance(a, (np.int64, int)):
                vals.append(ctypes.c_int64(int(a)))
            else:
                raise TypeError(f"kernel argument of type {type(a)}")
        params = (ctypes.c_void_p * len(vals))(*[ctypes.cast(ctypes.pointer(v), ctypes.c_void_p) for v in vals])
        g = tuple(grid) + (1,) * (3 - len(grid))
        b = tuple(block) + (1,) * (3 - len(block))
        s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _DRV.check(_DRV.lib.cuLaunchKernel(self.fn, g[0], g[1], g[2], b[0], b[1], b[2], shared_mem, s, params, None),
                   "cuLaunchKernel")


class RawModule:
    """compiles a CUDA C string with nvcc for the current GPU and loads it (cupy.RawModule's role)"""

    def __init__(self, code, options=()):
        global _DRV
        import torch
        torch.cuda.init()
        if _DRV is None:
            _DRV = _Driver()
        arch = _arch()
        opts = [o for o in options if o.startswith("-std")]
        key = hashlib.sha256((code + arch + " ".join(opts)).encode()).hexdigest()[:20]
        os.makedirs(CACHE, exist_ok=True)
        cubin = os.path.join(CACHE, f"{key}.cubin")
        if not os.path.exists(cubin):
            src = os.path.join(CACHE, f"{key}.cu")
            with open(src, "w") as f:
                f.write(code)
            subprocess.check_call([os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc"), "-cubin", f"-arch={arch}", "-O3"]
                                  + opts + ["-o", cubin + ".tmp", src])
            os.replace(cubin + ".tmp", cubin)
        with open(cubin, "rb") as f:
            self.image = f.read()
        self.mod = ctypes.c_void_p()
        _DRV.check(_DRV.lib.cuModuleLoadData(ctypes.byref(self.mod), self.image), "cuModuleLoadData")

    def get_function(self, name):
        fn = ctypes.c_void_p()
        _DRV.check(_DRV.lib.cuModuleGetFunction(ctypes.byref(fn), self.mod, name.encode()), "cuModuleGetFunction")
        return _Kernel(fn)


def install():
    """Put the stand-in cupy and the installed reference on the path; patch the CRT digit-sum kernel's
    Triton source.  Returns the reference's modules (rns, mpf, solver)."""
    if not os.path.isdir(os.path.join(REF_SITE, "sdpvibe")):
        raise RuntimeError("the reference is not installed in baseline/_ref (python -m pip install --no-index "
                           "--no-build-isolation --find-links /opt/wheelhouse --target baseline/_ref <reference>)")
    cp = types.ModuleType("cupy")
    cp.RawModule = RawModule
    cp.from_dlpack = lambda t: t
    cp.int32, cp.int64 = np.int32, np.int64
    sys.modules["cupy"] = cp
    if REF_SITE not in sys.path:
        sys.path.insert(0, REF_SITE)
    import triton
    import triton.language as tl
    import sdpvibe.rns as rns
    src = inspect.getsource(rns._crt_dot_kernel.fn)
    fixed = src.replace("tl.dot(c, h, hi)", "tl.dot(c, h, hi, out_dtype=tl.int32)") \
               .replace("tl.dot(c, l, lo)", "tl.dot(c, l, lo, out_dtype=tl.int32)")
    assert fixed != src, "the CRT digit-sum kernel's tl.dot calls were not found"
    ns = dict(rns.__dict__)
    fname = os.path.join(CACHE, "crt_dot_fixed.py")
    os.makedirs(CACHE, exist_ok=True)
    with open(fname, "w") as f:
        f.write(fixed.replace("@triton.jit\n", "", 1))
    code = compile(fixed.replace("@triton.jit\n", "", 1), fname, "exec")
    exec(code, ns)
    rns._crt_dot_kernel = triton.jit(ns["_crt_dot_kernel"])
    import sdpvibe.mpf as mpf
    import sdpvibe.solver as solver
    return rns, mpf, solver


# ------------------------------------------------------------------ the c3 solver on the reference
def reference_sdp(L, nblocks=300, N=1000, seed=0):
    """The reference's SDP object built from the same block data as sdpvibe_b200.synthetic.ising_like_sdp:
    every array converted once by this repository's exact host-to-MPF conversion and handed to the
    reference's own SDP._build (its chunking by dimension and layout)."""
    import mpmath as mp
    _, mpf_ref, solver_ref = install()
    from sdpvibe_b200 import solver as S
    from sdpvibe_b200.synthetic import ising_like_shapes, damped_bases
    blocks, N = ising_like_shapes(nblocks, N, seed=seed)
    rng = np.random.default_rng(seed + 1)
    data = []
    for bl in blocks:                                     # the draw order of ising_like_sdp
        Ve, Vo = damped_bases(bl["d"], bl["he"], bl["ho"])
        npair = bl["dim"] * (bl["dim"] + 1) // 2
        data.append((Ve, Vo, S._rand_host_mpf(rng, (bl["K"] * npair, 1), L),
                     S._rand_host_mpf(rng, (bl["K"] * npair, N), L)))
    b = S._rand_host_mpf(rng, (N, 1), L)

    def conv(x):
        if x is None:
            return None
        v = S._host_mpf(x, L)
        return mpf_ref.MPF(v.m, v.e)

    shapes = [dict(dim=bl["dim"], K=bl["K"], he=bl["he"], ho=bl["ho"]) for bl in blocks]
    sdp = solver_ref.SDP.__new__(solver_ref.SDP)
    mp.mp.prec = mpf_ref.NBITS(L) + 64
    sdp._build(shapes, lambda j: tuple(conv(x) for x in data[j]), conv(b), mp.mpf(0), L,
               solver_ref.Layout(shapes, N, L))
    return sdp, solver_ref


def run_plain_solver(iters=20, L=26):
    """Per-iteration device times (s) of the reference's Solver.run on the c3 SDP, first `iters` iterations."""
    import torch
    sdp, solver_ref = reference_sdp(L)
    sol = solver_ref.Solver(sdp, L)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    marks, walls = [], []
    start.record()
    t0 = time.perf_counter()

    def on_it(row):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        marks.append(ev)
        walls.append(time.perf_counter() - t0)
    sol.run(max_iter=iters, verbose=False, on_iteration=on_it)
    torch.cuda.synchronize()
    evs = [start] + marks
    return [evs[i].elapsed_time(evs[i + 1]) * 1e-3 for i in range(len(evs) - 1)], walls
