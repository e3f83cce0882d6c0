"""ctypes binding of libsdpv_b200.so (the C ABI declared in include/sdpv_b200.h).

Torch tensors are passed as raw device pointers; every call runs on torch's current stream of the
current device, like the reference's kernels.  A status other than SDPV_OK raises the exception the
reference raises in the same situation.  There is no CPU fallback: without the library or a GPU,
the first call fails loudly.
"""
import ctypes
import os
import threading

import torch

from . import _trace

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsdpv_b200.so")

OK, EOVERFLOW, ENOTSPD, ETIMEOUT, EINVAL, ECUDA, ENOMEM = range(7)
ERR_OVERFLOW, ERR_TIMEOUT, ERR_NOTSPD = 1, 2, 4

_P, _I, _L = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
_SIGS = {
    "sdpv_version": [],
    "sdpv_last_error": [],
    "sdpv_ctx_create": [_I, ctypes.POINTER(_P)],
    "sdpv_ctx_create_g": [_I, _I, ctypes.POINTER(_P)],
    "sdpv_ctx_destroy": [_P],
    "sdpv_ctx_query": [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "sdpv_ctx_moduli": [_P, _P],
    "sdpv_shift_round": [_P, _I, _L, _P, _I, _P, _P, _P],
    "sdpv_add_same": [_P, _P, _I, _L, _I, _P, _P],
    "sdpv_bitlen": [_P, _I, _L, _P, _P],
    "sdpv_badd_align": [_P, _P, _P, _P, _I, _L, _L, _L, _I, _P, _P, _P],
    "sdpv_mpf_mul": [_I, _L, _P, _P, _P, _P, _I, _P, _P, _P],
    "sdpv_mpf_add": [_I, _L, _P, _P, _P, _P, _I, _P, _P, _P],
    "sdpv_mpf_add_if": [_I, _L, _P, _P, _P, _P, _I, _P, _P, _P, _P],
    "sdpv_gram_columns": [_L, _P, _P, _P, _L, _L, _I, _P, _P, _P, _P, _P],
    "sdpv_zero_if": [_P, _L, _P, _P],
    "sdpv_mpf_norm": [_I, _I, _L, _P, _P, _P, _P, _P],
    "sdpv_mpf_from_f64": [_I, _L, _P, _P, _P, _P],
    "sdpv_schur_assemble": [_I, _L, _I, _I, _I, _P, _P, _P, _P, _P, _P, _L, _P, _P, _P],
    "sdpv_bigfloat_index": [_P, _L, _L, _L, _I, _P, _P],
    "sdpv_tune_set": [_I, _I],
    "sdpv_tune_get": [_I, _P],
    "sdpv_bigfloat_unpack": [_P, _P, _L, _I, _I, _P, _P, _P],
    "sdpv_bigfloat_pack": [_P, _P, _L, _I, _I, _P, _P, _P],
    "sdpv_top_max": [_P, _P, _I, _L, _L, _L, _I, _P, _P],
    "sdpv_align": [_P, _P, _I, _L, _L, _L, _P, _I, _I, _I, _P, _P],
    "sdpv_residues": [_P, _P, _L, _L, _L, _L, _I, _I, _P, _P, _L, _P],
    "sdpv_residues_u8": [_P, _P, _L, _L, _L, _L, _I, _I, _P, _P, _L, _P],
    "sdpv_residues_rows": [_P, _P, _L, _L, _L, _L, _I, _I, _P, _P, _L, _P],
    "sdpv_align_rows": [_P, _P, _I, _L, _L, _L, _P, _I, _I, _L, _P, _P],
    "sdpv_align_t": [_P, _P, _I, _L, _L, _L, _P, _I, _I, _L, _P, _P],
    "sdpv_rns_gemm": [_P, _P, _P, _P, _P, _L, _L, _P, _L, _I, _I, _L, _L, _L, _L, _I, _P],
    "sdpv_crt_block": [_P, _P, _L, _L, _L, _L, _L, _P, _P, _P],
    "sdpv_crt_norm": [_P, _P, _L, _L, _L, _L, _L, _L, _P, _P, _I, _P, _P, _P],
    "sdpv_crt_norm_if": [_P, _P, _L, _L, _L, _L, _L, _L, _P, _P, _I, _P, _P, _P, _P],
    "sdpv_chol_tiles": [_P, _P, _L, _I, _I, _I, _P],
    "sdpv_trinv_tiles": [_P, _P, _P, _P, _L, _I, _I, _I, _P],
    "sdpv_trinv_tiles_noalloc": [_P, _P, _P, _L, _I, _I, _I, _P],
    "sdpv_trsv_tiles": [_P, _P, _P, _L, _I, _I, _I, _P],
    "sdpv_eig_sym_f64": [_P, _L, _I, _P, _P, _P, _P],
    "sdpv_get_error": [ctypes.POINTER(ctypes.c_uint), _P],
    "sdpv_rns_gemm_grouped": [_P, _P, _P, _L, _L, _P, _P, _L, _L, _L, _I, _I, _P, _L, _P, _L, _L, _I, _I, _P],
    "sdpv_grp_copy": [_P, _P, _I, _P, _L, _I, _P, _L, _P],
    "sdpv_grp_finish_fixed": [_P, _I, _L, _L, _P, _P, _I, _I, _P, _P, _L, _P],
    "sdpv_grp_merge": [_P, _L, _P, _L, _I, _P, _L, _P],
    "sdpv_grp_solve_round": [_P, _P, _I, _L, _L, _P, _L, _P, _L, _I, _P, _P, _L, _P],
    "sdpv_grp_tile_widen": [_P, _L, _I, _L, _I, _I, _P, _L, _P, _P],
    "sdpv_grp_tile_narrow": [_P, _P, _I, _I, _P, _L, _I, _L, _P, _P, _L, _P, _P, _L, _P],
    "sdpv_device_status": [_P],
    "sdpv_wait_probe": [ctypes.c_uint, _I, _P],
}

_lib = None
_lock = threading.Lock()


def lib():
    """Load the library (building it in-tree first if it is missing)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    from .build import build
                    build()
                h = ctypes.CDLL(LIB_PATH)
                for name, argt in _SIGS.items():
                    f = getattr(h, name)
                    f.argtypes = argt
                    f.restype = ctypes.c_char_p if name == "sdpv_last_error" else ctypes.c_int
                _apply_tuning(h)
                _lib = h
    return _lib


TUNING_TABLE = os.path.join(HERE, "tuning_b200.json")


def _apply_tuning(h):
    """the autotuner's launch-shape knobs (sdpvibe_b200/autotune.py), when its table was made on this GPU
    model; SDPV_TUNING=0 keeps the defaults"""
    if os.environ.get("SDPV_TUNING", "1") == "0" or not os.path.exists(TUNING_TABLE):
        return
    try:
        import json
        with open(TUNING_TABLE) as f:
            table = json.load(f)
        if not torch.cuda.is_available() or table.get("device") != torch.cuda.get_device_name():
            return
    except (OSError, ValueError, RuntimeError):
        return
    ids = {"crt_ctas": 0, "narrow_max": 1, "pack_max": 2, "res_warps": 3, "moduli_group": 4}
    for name, value in table.get("knobs", {}).items():
        if name in ids:
            h.sdpv_tune_set(ids[name], int(value))


def stream():
    """torch's current stream on the current device, as a cudaStream_t (the direct C lookups: the
    torch.cuda.current_stream() wrapper costs more than a small kernel launch)."""
    return ctypes.c_void_p(torch._C._cuda_getCurrentRawStream(torch._C._cuda_getDevice()))


def ptr(t):
    """Device pointer of a tensor (None -> NULL).  Tensors must be CUDA and contiguous."""
    if t is None:
        return None
    if not t.is_cuda:
        raise RuntimeError("sdpvibe_b200 kernels need CUDA tensors (no CPU fallback)")
    assert t.is_contiguous(), "kernel operands must be contiguous"
    return ctypes.c_void_p(t.data_ptr())


def ptr_strided(t):
    """Device pointer of a tensor view whose strides the caller passes explicitly."""
    if not t.is_cuda:
        raise RuntimeError("sdpvibe_b200 kernels need CUDA tensors (no CPU fallback)")
    return ctypes.c_void_p(t.data_ptr())


def check(status, what=""):
    if status == OK:
        return
    if status == EOVERFLOW:
        raise OverflowError("result does not fit in the requested number of limbs")
    if status == ENOTSPD:
        raise ValueError("matrix is not positive definite (diagonal)")
    if status == EINVAL:
        raise ValueError(f"{what}: invalid argument")
    if status == ETIMEOUT:
        raise RuntimeError(f"{what}: a device pipeline wait timed out")
    msg = lib().sdpv_last_error()
    raise RuntimeError(f"{what}: CUDA error {msg.decode() if msg else ''} (status {status})")


def call(name, *args):
    end = _trace.before(name) if _trace._active is not None else None
    check(getattr(lib(), name)(*args), name)
    if end is not None:
        end.record()


def device_status():
    """Synchronise the current stream and raise what the device error word holds (and clear it):
    RuntimeError for a bounded wait that timed out, ValueError for a non-positive pivot, OverflowError
    for a rounding overflow."""
    check(lib().sdpv_device_status(stream()), "device status")


def device_error_flags():
    """Read and clear the device error word of the current device (synchronises the stream)."""
    v = ctypes.c_uint(0)
    check(lib().sdpv_get_error(ctypes.byref(v), stream()), "sdpv_get_error")
    return v.value
