"""The C-ABI library builds for sm_100a, loads without a GPU and exports every entry point that
include/*.h declares (no compute calls here)."""
import ctypes
import glob
import os
import re

from conftest import ROOT


def declared():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names += re.findall(r"^\s*(?:int|const char\*)\s+(sdpv_\w+)\s*\(", txt, re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared()
    assert "sdpv_rns_gemm" in names and "sdpv_residues" in names and "sdpv_crt_norm" in names
    assert len(names) >= 18


def test_library_exports_every_declared_symbol():
    from sdpvibe_b200 import _lib
    h = _lib.lib()                          # builds in-tree if missing, loads with no GPU present
    missing = [n for n in declared() if not hasattr(h, n)]
    assert not missing, missing
    assert h.sdpv_version() >= 1


def test_python_binding_covers_header():
    from sdpvibe_b200 import _lib
    assert set(declared()) <= set(_lib._SIGS)


def test_tuning_knobs_validated():
    """the launch-shape knobs accept their documented ranges only (host-side, no GPU)"""
    import ctypes
    from sdpvibe_b200 import _lib
    h = _lib.lib()
    v = ctypes.c_int(0)
    for knob, good, bad in ((0, (1, 4), (0, 5)), (1, (0, 32, 64), (8, 80)), (2, (0, 64), (-16, 128)),
                            (3, (8, 16), (0, 12, 24)), (4, (1, 2, 4, 8, 16), (0, 3, 12, 32))):
        assert h.sdpv_tune_get(knob, ctypes.byref(v)) == 0
        old = v.value
        for g in good:
            assert h.sdpv_tune_set(knob, g) == 0
        for b in bad:
            assert h.sdpv_tune_set(knob, b) == _lib.EINVAL
        assert h.sdpv_tune_set(knob, old) == 0
    assert h.sdpv_tune_set(3, 1) == _lib.EINVAL


def test_context_moduli_group_validated():
    """sdpv_ctx_create_g refuses moduli groups other than 1, 2, 4, 8, 16 before touching the device"""
    import ctypes
    from sdpvibe_b200 import _lib
    h = _lib.lib()
    out = ctypes.c_void_p()
    for G in (0, 3, 6, 32, -1):
        assert h.sdpv_ctx_create_g(26, G, ctypes.byref(out)) == _lib.EINVAL
    assert h.sdpv_ctx_create_g(0, 16, ctypes.byref(out)) == _lib.EINVAL
