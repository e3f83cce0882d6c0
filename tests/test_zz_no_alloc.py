"""The allocation-free triangular inverse (sdpv_trinv_tiles_noalloc).

It exists for callers that cannot allocate device memory when they need the inverse -- for example a
process whose device memory is already handed to another allocator.  It must give exactly what
sdpv_trinv_tiles gives with a caller-allocated scratch, call after call (for WL > 64 its scratch is a
fixed array that keeps the previous call's contents), accept every size its fixed scratch holds, refuse
larger ones, and take no device memory after its first call.  This file is collected last so that a
failure here comes after every other test has run.
"""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

BT = 32
SCRATCH_WORDS = 4 << 20
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _factored_tiles(ntiles, L, seed, distinct=4):
    """Lower Cholesky factors (upper part zero) and pivot reciprocals of SPD tiles, via the C ABI;
    `distinct` different tiles repeated to ntiles."""
    from sdpvibe_b200 import _lib
    rng = np.random.default_rng(seed)
    WL, LF = L + 24, L
    F = 32 * LF
    tiles = []
    for _ in range(min(distinct, ntiles)):
        G = rng.integers(-60, 61, size=(BT, BT)).astype(object)
        A = G.dot(G.T) + np.eye(BT, dtype=object) * (40 * BT)
        sh = np.array([int(A[i, i]).bit_length() // 2 + 1 for i in range(BT)], dtype=object)
        V = (A * (1 << F)) // (2 ** (sh[:, None] + sh[None, :]))      # exact: floor of a positive shift
        U = V % (1 << (32 * WL))
        words = np.empty((BT, BT, WL), np.int64)
        for k in range(WL):
            words[:, :, k] = ((U >> (32 * k)) % (1 << 32)).astype(np.int64)
        tiles.append(words.astype(np.uint32).view(np.int32))
    W = np.stack([tiles[t % len(tiles)] for t in range(ntiles)])
    Wd = torch.from_numpy(W).cuda()
    RINV = torch.zeros((ntiles, BT, WL), dtype=torch.int32, device="cuda")
    _lib.call("sdpv_chol_tiles", _lib.ptr(Wd), _lib.ptr(RINV), ntiles, BT, WL, LF, _lib.stream())
    tri = torch.tril(torch.ones(BT, BT, dtype=torch.bool, device="cuda"))
    Wd[:, ~tri] = 0
    return Wd, RINV, WL, LF


def _inverse(Lw, RINV, WL, LF):
    from sdpvibe_b200 import _lib
    X = torch.empty_like(Lw)
    scratch = torch.empty_like(Lw)
    _lib.call("sdpv_trinv_tiles", _lib.ptr(Lw), _lib.ptr(RINV), _lib.ptr(X), _lib.ptr(scratch), Lw.shape[0], BT, WL,
              LF, _lib.stream())
    return X


def _inverse_noalloc(Lw, RINV, WL, LF):
    from sdpvibe_b200 import _lib
    X = torch.full_like(Lw, -1)
    _lib.call("sdpv_trinv_tiles_noalloc", _lib.ptr(Lw), _lib.ptr(RINV), _lib.ptr(X), Lw.shape[0], BT, WL, LF,
              _lib.stream())
    torch.cuda.synchronize()
    return X


@pytest.mark.parametrize("L,sizes", [(24, (5, 2, 150)), (26, (3, 7, 1)), (48, (6, 2, 9))])
def test_noalloc_inverse_matches_allocating_entry_point(L, sizes):
    """Calls in a row with different tiles and sizes (larger, then smaller, ...): every call equals the
    allocating entry point.  L = 48 (WL = 72 > 64) runs on the fixed scratch, so stale contents of a larger
    earlier call must not leak into a smaller later one; L = 24 with 150 tiles is beyond what the fixed
    scratch would hold and runs without it."""
    for i, n in enumerate(sizes):
        Lw, RINV, WL, LF = _factored_tiles(n, L, seed=1000 * L + i)
        X_ref = _inverse(Lw, RINV, WL, LF)
        for _ in range(2):                          # two calls in a row on the same inputs as well
            assert torch.equal(_inverse_noalloc(Lw, RINV, WL, LF), X_ref)   # integer fixed point: exact


def test_noalloc_largest_size_on_the_fixed_scratch():
    """The largest call the fixed scratch holds at WL = 72 runs and matches the allocating entry point."""
    L = 48
    WL = L + 24
    n = SCRATCH_WORDS // (BT * BT * WL)
    Lw, RINV, WL, LF = _factored_tiles(n, L, seed=7, distinct=3)
    assert torch.equal(_inverse_noalloc(Lw, RINV, WL, LF), _inverse(Lw, RINV, WL, LF))


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from sdpvibe_b200 import _lib
    WL, LF = 74, 50
    too_many = SCRATCH_WORDS // (BT * BT * WL) + 1
    dummy = torch.zeros(16, dtype=torch.int32, device="cuda")
    st = _lib.lib().sdpv_trinv_tiles_noalloc(_lib.ptr(dummy), _lib.ptr(dummy), _lib.ptr(dummy), too_many, BT, WL, LF,
                                             _lib.stream())
    assert st == _lib.EINVAL
    assert b"exceeds the fixed scratch" in _lib.lib().sdpv_last_error()


_FRESH = r"""
import sys, torch
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
from test_zz_no_alloc import _factored_tiles, _inverse
from sdpvibe_b200 import _lib
Lw, RINV, WL, LF = _factored_tiles(4, 48, seed=3)       # loads the tile module (the fixed array with it)
X_ref = _inverse(Lw, RINV, WL, LF)
outs = [torch.full_like(Lw, -1) for _ in range(3)]        # every output allocated before the reading


def call(X, n):
    _lib.call("sdpv_trinv_tiles_noalloc", _lib.ptr(Lw), _lib.ptr(RINV), _lib.ptr(X), n, 32, WL, LF, _lib.stream())


call(outs[0], 4)                                          # the first allocation-free call
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
call(outs[1], 4)
call(outs[2], 2)
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
assert torch.equal(outs[0], X_ref) and torch.equal(outs[1], X_ref) and torch.equal(outs[2][:2], X_ref[:2])
assert free1 == free0, (free0, free1)
print("ok")
"""


def test_noalloc_fresh_process_lazy_loading_takes_no_memory_after_first_call():
    """In a fresh process with lazy module loading: after the first tile call the allocation-free inverse
    takes no further device memory (the output tensors of the checks are allocated before the reading)."""
    env = dict(os.environ, CUDA_MODULE_LOADING="LAZY")
    r = subprocess.run([sys.executable, "-c", _FRESH, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
