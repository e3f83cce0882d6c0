"""Limb-level bookkeeping in limb-plane layout: drop-in for ``sdpvibe.limbops``.

A batch of B multiword integers is an int32 tensor X of shape (L, B); X[k, e] is the k-th 32-bit limb
(little endian, two's complement) of entry e (sdpvibe/limbops.py:1-10).  Every function here is one
CUDA kernel of libsdpv_b200 on torch's current stream.
"""
import torch

from . import _lib

dev = "cuda"
BB = 256
ERR = {}          # kept for API compatibility; the overflow flag lives in the library's device error word


def check_errors():
    """Raise OverflowError if a rounding step flagged an overflow since the last check
    (sdpvibe/limbops.py:165-169).  Synchronises the current stream."""
    if _lib.device_error_flags() & _lib.ERR_OVERFLOW:
        raise OverflowError("a rounding step overflowed its limb budget")


def shift_round(X, s, Lout, check=False):
    """X: (Lin, B) int32 limbs; s: (B,) int64 -> round_half_up(X / 2^s) as (Lout, B)
    (sdpvibe/limbops.py:173-185)."""
    Lin, B = X.shape
    X = X.contiguous()
    s = s.to(torch.int64).contiguous()
    out = torch.empty((Lout, B), dtype=torch.int32, device=X.device)
    flag = torch.empty((B,), dtype=torch.int32, device=X.device) if check else None
    _lib.call("sdpv_shift_round", _lib.ptr(X), Lin, B, _lib.ptr(s), Lout, _lib.ptr(out), _lib.ptr(flag), _lib.stream())
    if check and bool(flag.any()):
        raise OverflowError("result does not fit in the requested number of limbs")
    return out


def add_same(A, Bm, sgn=1):
    """A + sgn*B for (L, B) int32 limbs with identical exponents (exact, wraps mod 2^(32L))."""
    L, Bn = A.shape
    A = A.contiguous()
    Bm = Bm.contiguous()
    out = torch.empty_like(A)
    _lib.call("sdpv_add_same", _lib.ptr(A), _lib.ptr(Bm), L, Bn, int(sgn), _lib.ptr(out), _lib.stream())
    return out


def bitlen_words(X):
    """(L, B) int32 limbs -> (B,) int64 bit length of v (v >= 0) or of ~v (v < 0)."""
    L, B = X.shape
    X = X.contiguous()
    out = torch.empty((B,), dtype=torch.int64, device=X.device)
    _lib.call("sdpv_bitlen", _lib.ptr(X), L, B, _lib.ptr(out), _lib.stream())
    return out
