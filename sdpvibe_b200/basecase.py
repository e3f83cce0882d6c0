"""Cholesky base case on CUDA cores: drop-in for ``sdpvibe.basecase``.

Tiles of 32 x 32 entries in a wide fixed-point format (WL = L + 24 words, F = 32 L fraction bits),
entry-major (..., 32, 32, WL) as in sdpvibe/basecase.py.  The factorisation and the triangular inverse
run in libsdpv_b200 (sdpv_chol_tiles, sdpv_trinv_tiles), one CTA per tile, with the reference's
arithmetic (truncated product-scanning multiply, Newton d^-1/2 from a double seed), so results are
bit-identical.
"""
import torch

from . import _lib
from .rns import dev
from .mpmat import MP, rescale, bitlen_limbs, headroom_bits

BT = 32


def _soa_to_aos(X):
    return X.permute(*range(1, X.dim()), 0).contiguous()


def _aos_to_soa(X):
    return X.permute(X.dim() - 1, *range(0, X.dim() - 1)).contiguous()


def tile_factor(W, WL, LF):
    """W: (nb, 32, 32, WL) int32 wide fixed point (entry-major) -> (L factor with zero upper part,
    X = L^-1), both (nb, 32, 32, WL)."""
    nb = W.shape[0]
    Lw = W.contiguous().clone()
    RINV = torch.zeros((nb, BT, WL), dtype=torch.int32, device=Lw.device)
    _lib.call("sdpv_chol_tiles", _lib.ptr(Lw), _lib.ptr(RINV), nb, BT, WL, LF, _lib.stream())
    tri = torch.tril(torch.ones(BT, BT, dtype=torch.bool, device=Lw.device))
    Lw[:, ~tri] = 0
    X = torch.empty_like(Lw)
    scratch = torch.empty_like(Lw)
    _lib.call("sdpv_trinv_tiles", _lib.ptr(Lw), _lib.ptr(RINV), _lib.ptr(X), _lib.ptr(scratch), nb, BT, WL, LF,
              _lib.stream())
    return Lw, X


class Tile:
    """Cholesky factor of a diagonal tile (wide, entry-major) with its inverse (sdpvibe/basecase.py:259-261)."""
    __slots__ = ("Lw", "RINV", "b", "WL", "LF", "X", "Lmp")


def chol_tile(A, LI=24, threads=256, want_inverse=False):
    """A: MP (32 x 32) fixed point -> (L factor with A's exponent, Tile[, X = L^-1])
    (sdpvibe/basecase.py:268-288)."""
    b = A.shape[0]
    assert b == BT
    L, e = A.L, A.uniform_exp()
    LF, WL = L, L + LI
    F = 32 * LF
    W = _soa_to_aos(rescale(A, -F, WL).limbs)[None]                # (1, b, b, WL)
    Lw, X = tile_factor(W, WL, LF)
    Lout = rescale(MP(_aos_to_soa(Lw[0]), -F), e, L)
    t = Tile()
    t.Lw, t.b, t.WL, t.LF = Lw[0], b, WL, LF
    t.RINV = None
    t.Lmp = Lout
    Xs = _aos_to_soa(X[0])
    top = int(bitlen_limbs(Xs).max()) - F
    t.X = rescale(MP(Xs, -F), top - headroom_bits(L), L)
    if not want_inverse:
        return Lout, t
    return Lout, t, t.X


def chol_inv_tile(A, LI=24, threads=256):
    Lout, _, X = chol_tile(A, LI, threads, want_inverse=True)
    return Lout, X


def apply_tile_inverse(t, B, refine=0):
    """P = L_tile^-1 B with the explicit tile inverse (+ refinement), B: MP (b x m) with per-column
    exponents (sdpvibe/basecase.py:296-307)."""
    from .mpmat import gemm_nt, add
    tr = lambda M: MP(M.limbs.transpose(1, 2).contiguous(), 0)
    P = gemm_nt(t.X, tr(B), out_exp="col", bt_rowexp=B.exp)
    for _ in range(refine):
        LP = gemm_nt(t.Lmp, tr(P), out_exp="col", bt_rowexp=P.exp)
        Rr = add(B, LP, -1, out_exp="col")
        D = gemm_nt(t.X, tr(Rr), out_exp="col", bt_rowexp=Rr.exp)
        P = add(P, D, 1, out_exp="align")
    return P
