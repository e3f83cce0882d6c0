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


def tile_factor(W, WL, LF, want_inverse=True):
    """W: (nb, 32, 32, WL) int32 wide fixed point (entry-major) -> (L factor with zero upper part,
    X = L^-1 (None unless want_inverse), both (nb, 32, 32, WL); pivot reciprocals (nb, 32, WL))."""
    nb = W.shape[0]
    Lw = W.contiguous().clone()
    RINV = torch.zeros((nb, BT, WL), dtype=torch.int32, device=Lw.device)
    _lib.call("sdpv_chol_tiles", _lib.ptr(Lw), _lib.ptr(RINV), nb, BT, WL, LF, _lib.stream())
    tri = torch.tril(torch.ones(BT, BT, dtype=torch.bool, device=Lw.device))
    Lw[:, ~tri] = 0
    if not want_inverse:
        return Lw, None, RINV
    X = torch.empty_like(Lw)
    scratch = torch.empty_like(Lw)
    _lib.call("sdpv_trinv_tiles", _lib.ptr(Lw), _lib.ptr(RINV), _lib.ptr(X), _lib.ptr(scratch), nb, BT, WL, LF,
              _lib.stream())
    return Lw, X, RINV


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
    Lw, X, RINV = tile_factor(W, WL, LF, want_inverse)
    Lout = rescale(MP(_aos_to_soa(Lw[0]), -F), e, L)
    t = Tile()
    t.Lw, t.b, t.WL, t.LF = Lw[0], b, WL, LF
    t.RINV = RINV[0]
    t.Lmp = Lout
    t.X = None
    if not want_inverse:
        return Lout, t
    Xs = _aos_to_soa(X[0])
    top = int(bitlen_limbs(Xs).max()) - F
    t.X = rescale(MP(Xs, -F), top - headroom_bits(L), L)
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


def trsv_tile(t, Vlimbs, vexp, out_exp=None):
    """Solve L y = v for many vectors with a factored tile, by substitution on CUDA cores
    (sdpvibe/basecase.py:310-331).  Vlimbs (L, nvec, b) limb planes, vexp (nvec,) exponents (value =
    mantissa 2^vexp); out_exp None: per-vector exponent from the result's bit length, an int: fixed.
    Returns (limbs (L, nvec, b), exponents (nvec,))."""
    from .limbops import shift_round, bitlen_words
    L, nvec, b = Vlimbs.shape
    F = 32 * t.LF
    FX = 32 * L - 40
    # each vector as fixed point with exponent -FX (its own scale), widened exactly
    Wsoa = rescale(MP(Vlimbs.reshape(L, 1, nvec * b), -FX), -F, t.WL).limbs          # (WL, 1, nvec*b)
    W = _soa_to_aos(Wsoa.reshape(t.WL, nvec, b))                                      # (nvec, b, WL)
    _lib.call("sdpv_trsv_tiles", _lib.ptr(t.Lw), _lib.ptr(t.RINV), _lib.ptr(W), nvec, BT, t.WL, t.LF, _lib.stream())
    Ws = _aos_to_soa(W).view(t.WL, nvec * b)
    base = vexp + FX - F                                                              # exponent of the wide words
    if out_exp is None:
        ne = bitlen_words(Ws).view(nvec, b).amax(1) + base - headroom_bits(L)
    else:
        ne = torch.full((nvec,), int(out_exp), dtype=torch.int64, device=Vlimbs.device)
    s = (ne - base)[:, None].expand(nvec, b).reshape(-1)
    return shift_round(Ws, s, L).view(L, nvec, b), ne
