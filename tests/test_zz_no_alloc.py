"""The allocation-free triangular inverse (sdpv_trinv_tiles_noalloc).

It exists for callers that cannot allocate device memory when they need the inverse -- for example a
process whose device memory is already handed to another allocator.  It must give exactly what
sdpv_trinv_tiles gives with a caller-allocated scratch, call after call (its scratch is a fixed array
that keeps the previous call's contents), and refuse sizes beyond its fixed scratch.  This file is
collected last so that a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

BT = 32


def _factored_tiles(ntiles, L, seed):
    """Lower Cholesky factors (upper part zero) and pivot reciprocals of SPD tiles, via the C ABI."""
    from sdpvibe_b200 import _lib
    rng = np.random.default_rng(seed)
    WL, LF = L + 24, L
    F = 32 * LF
    tiles = []
    for _ in range(ntiles):
        G = rng.integers(-60, 61, size=(BT, BT)).astype(object)
        A = G.dot(G.T) + np.eye(BT, dtype=object) * (40 * BT)
        sh = [int(A[i, i]).bit_length() // 2 + 1 for i in range(BT)]
        for i in range(BT):
            for j in range(BT):
                v = (int(A[i, j]) << F) >> (sh[i] + sh[j])
                u = v % (1 << (32 * WL))
                tiles.append([((u >> (32 * k)) + (1 << 31)) % (1 << 32) - (1 << 31) for k in range(WL)])
    W = torch.tensor(tiles, dtype=torch.int32).view(ntiles, BT, BT, WL).cuda()
    RINV = torch.zeros((ntiles, BT, WL), dtype=torch.int32, device="cuda")
    _lib.call("sdpv_chol_tiles", _lib.ptr(W), _lib.ptr(RINV), ntiles, BT, WL, LF, _lib.stream())
    tri = torch.tril(torch.ones(BT, BT, dtype=torch.bool, device="cuda"))
    W[:, ~tri] = 0
    return W, RINV, WL, LF


@pytest.mark.parametrize("ntiles,L", [(5, 24), (3, 26)])
def test_noalloc_inverse_matches_allocating_entry_point(ntiles, L):
    from sdpvibe_b200 import _lib
    Lw, RINV, WL, LF = _factored_tiles(ntiles, L, seed=ntiles * 100 + L)
    X_ref = torch.empty_like(Lw)
    scratch = torch.empty_like(Lw)
    _lib.call("sdpv_trinv_tiles", _lib.ptr(Lw), _lib.ptr(RINV), _lib.ptr(X_ref), _lib.ptr(scratch), ntiles, BT, WL,
              LF, _lib.stream())
    for _ in range(2):                              # two calls in a row: the shared scratch is reused
        X = torch.full_like(Lw, -1)
        _lib.call("sdpv_trinv_tiles_noalloc", _lib.ptr(Lw), _lib.ptr(RINV), _lib.ptr(X), ntiles, BT, WL, LF,
                  _lib.stream())
        torch.cuda.synchronize()
        assert torch.equal(X, X_ref)                # integer fixed point: exact agreement


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from sdpvibe_b200 import _lib
    WL, LF = 50, 26
    too_many = (4 << 20) // (BT * BT * WL) + 1
    dummy = torch.zeros(16, dtype=torch.int32, device="cuda")
    st = _lib.lib().sdpv_trinv_tiles_noalloc(_lib.ptr(dummy), _lib.ptr(dummy), _lib.ptr(dummy), too_many, BT, WL, LF,
                                             _lib.stream())
    assert st == _lib.EINVAL
    assert b"exceeds the fixed scratch" in _lib.lib().sdpv_last_error()
