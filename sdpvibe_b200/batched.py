"""Batched multiprecision linear algebra over many equal-sized blocks: drop-in for ``sdpvibe.batched``.

A BMP holds a stack of nb matrices: limbs int32 (L, nb, R, C) limb planes and exp, a Python int
(uniform) or an (nb, C) int64 tensor (sdpvibe/batched.py:16-42).  The recursive Cholesky and the
triangular solves follow the reference's recursion, split points, refinement counts and rounding points
exactly (batched.py:234-352), so results are bit-identical; every product is the exact residue GEMM of
rns.py over all nb blocks in one launch, and the 32 x 32 diagonal tiles use the CUDA-core base case of
basecase.py.
"""
import torch

from . import _lib
from .rns import dev
from .mpmat import ctx, headroom_bits, residue_product
from .limbops import shift_round, add_same, bitlen_words
from .basecase import _soa_to_aos, _aos_to_soa, tile_factor


class BMP:
    __slots__ = ("limbs", "exp")

    def __init__(self, limbs, exp):
        self.limbs, self.exp = limbs, exp

    @property
    def shape(self):
        return tuple(self.limbs.shape[1:])

    @property
    def L(self):
        return self.limbs.shape[0]

    def expt(self):
        nb, R, C = self.shape
        if isinstance(self.exp, int):
            return torch.full((nb, C), self.exp, dtype=torch.int64, device=dev)
        return self.exp

    def __getitem__(self, idx):
        r, c = idx
        e = self.exp if isinstance(self.exp, int) else self.exp[:, c].contiguous()
        return BMP(self.limbs[:, :, r, c].contiguous(), e)

    def t(self):
        assert isinstance(self.exp, int)
        return BMP(self.limbs.transpose(2, 3).contiguous(), self.exp)

    def flat(self):
        return self.limbs.reshape(self.L, -1)


def brescale(A, new_exp, Lout=None):
    """batched.py:45-52: re-round to exponent(s) new_exp (int or (nb, C) tensor)."""
    nb, R, C = A.shape
    Lo = Lout or A.L
    if isinstance(new_exp, int) and isinstance(A.exp, int):
        s = torch.full((nb * R * C,), new_exp - A.exp, dtype=torch.int64, device=dev)
        return BMP(shift_round(A.flat(), s, Lo).view(Lo, nb, R, C), new_exp)
    ne = new_exp if torch.is_tensor(new_exp) else torch.full((nb, C), int(new_exp), dtype=torch.int64, device=dev)
    s = (ne - A.expt())[:, None, :].expand(nb, R, C).reshape(-1)
    return BMP(shift_round(A.flat(), s, Lo).view(Lo, nb, R, C), ne.clone())


def badd(A, B, alpha=1, out_exp=None):
    """batched.py:82-92: exact same-exponent add, or 'align' (both rounded to max(ea, eb) + 1 per column)."""
    nb, R, C = A.shape
    L = A.L
    if isinstance(out_exp, int) and isinstance(A.exp, int) and isinstance(B.exp, int) and \
            A.exp == out_exp and B.exp == out_exp:
        return BMP(add_same(A.flat(), B.flat(), alpha).view(L, nb, R, C), out_exp)
    assert out_exp == "align"
    out = torch.empty((L, nb, R, C), dtype=torch.int32, device=dev)
    e = torch.empty((nb, C), dtype=torch.int64, device=dev)
    Am, Bm = A.limbs.contiguous(), B.limbs.contiguous()
    EA, EB = A.expt().contiguous(), B.expt().contiguous()
    _lib.call("sdpv_badd_align", _lib.ptr(Am), _lib.ptr(Bm), _lib.ptr(EA), _lib.ptr(EB), L, nb, R, C, int(alpha),
              _lib.ptr(out), _lib.ptr(e), _lib.stream())
    return BMP(out, e)


def bgemm_nt(A, Bt, out_exp="col", kc=4096, bt_rowexp=None):
    """batched.py:165-197: C[b] = A[b] @ Bt[b]^T for all b, exact, then rounded.  A: uniform int exponent
    (or per-block in column 0); Bt: int exponent or per-row exponents bt_rowexp (nb, N); out_exp 'col',
    'mat' or int.  kc is accepted for compatibility."""
    nb, M, K = A.shape
    nb2, N, K2 = Bt.shape
    assert nb == nb2 and K == K2
    L = A.L
    R = ctx(L)
    eA = A.exp if isinstance(A.exp, int) else A.exp[:, 0]
    acc = (torch.empty if K else torch.zeros)((R.n, nb * M, N), dtype=torch.int16, device=dev)
    if K:
        Av = A.limbs.reshape(L, nb * M, K)
        if A.limbs.data_ptr() == Bt.limbs.data_ptr() and M == N:
            residue_product(R, Av, Av, acc, nb=nb, fresh=True)
        else:
            residue_product(R, Av, Bt.limbs.reshape(L, nb * N, K), acc, nb=nb, fresh=True)
    eB = Bt.exp if bt_rowexp is None else bt_rowexp
    if isinstance(eA, int) and isinstance(eB, int):
        e_in = eA + eB
    else:
        eA_t = eA if torch.is_tensor(eA) else torch.full((nb,), eA, dtype=torch.int64, device=dev)
        eB_t = eB if torch.is_tensor(eB) else torch.full((nb, N), eB, dtype=torch.int64, device=dev)
        if eB_t.dim() == 1:
            eB_t = eB_t[:, None].expand(nb, N)
        e_in = eA_t[:, None] + eB_t
    return _bcrt_round(acc, nb, M, N, e_in, out_exp, L)


def _bcrt_round(acc, nb, M, N, e_in, out_exp, L):
    """batched.py:200-231: CRT of all nb*M x N entries, then one rounding to a fixed exponent, per
    (block, column) 'col', or per block 'mat' (one extra rounding)."""
    R = ctx(L)
    rows = nb * M
    Wd, bl, _ = R.crt_block(acc, N, 0, N, rows)                   # entries (b*M + i)*N + j
    fixed = isinstance(e_in, int) and isinstance(out_exp, int)
    if fixed:
        s = torch.full((rows * N,), out_exp - e_in, dtype=torch.int64, device=dev)
        return BMP(shift_round(Wd, s, L).view(L, nb, M, N), out_exp)
    e_in = e_in if torch.is_tensor(e_in) else torch.full((nb, N), e_in, dtype=torch.int64, device=dev)
    if isinstance(out_exp, str):
        sj = bl.view(nb, M, N).amax(1) - headroom_bits(L)
        ej = e_in + sj
    else:
        ej = torch.full((nb, N), int(out_exp), dtype=torch.int64, device=dev)
        sj = ej - e_in
    s = sj[:, None, :].expand(nb, M, N).reshape(-1)
    out = shift_round(Wd, s, L).view(L, nb, M, N)
    if isinstance(out_exp, int):
        return BMP(out, out_exp)
    C = BMP(out, ej.contiguous())
    if out_exp == "mat":
        C = brescale(C, ej.amax(1, keepdim=True).expand(nb, N).contiguous())
    return C


class BTile:
    __slots__ = ("X", "Lmp")


def bchol_tile(A, LI=24, threads=256):
    """batched.py:243-262: A: BMP (nb, b, b) fixed point -> (L BMP, BTile with the inverse X)."""
    nb, b, _ = A.shape
    L, e = A.L, A.exp
    LF, WL = L, L + LI
    F = 32 * LF
    Ws = brescale(A, -F, WL).limbs                                 # (WL, nb, b, b)
    Lw, X, _ = tile_factor(_soa_to_aos(Ws), WL, LF)                # (nb, b, b, WL) each
    Lout = brescale(BMP(_aos_to_soa(Lw), -F), e, L)
    Xs = _aos_to_soa(X)
    top = bitlen_words(Xs.reshape(WL, -1)).view(nb, b * b).amax(1) - F
    ex = (top - headroom_bits(L))[:, None].expand(nb, b).contiguous()
    t = BTile()
    t.Lmp = Lout
    t.X = brescale(BMP(Xs, torch.full((nb, b), -F, dtype=torch.int64, device=dev)), ex, L)
    return Lout, t


def _split(n, bt):
    return (n // 2 + bt - 1) // bt * bt


def _ntiles(n, bt):
    if n <= bt:
        return 1
    n1 = _split(n, bt)
    return _ntiles(n1, bt) + _ntiles(n - n1, bt)


def bchol(A, bt=32, refine=1):
    """batched.py:274-288: batched recursive Cholesky of equilibrated fixed-point blocks -> (L, tiles)."""
    nb, n, _ = A.shape
    L, e = A.L, A.exp
    if n <= bt:
        assert n == bt
        Lt, t = bchol_tile(A)
        return Lt, [t]
    n1 = _split(n, bt)
    L11, t1 = bchol(A[:n1, :n1], bt, refine)
    L21 = btrsm_right(A[n1:, :n1], L11, t1, bt, refine)
    S = badd(A[n1:, n1:], bgemm_nt(L21, L21, out_exp=e), -1, out_exp=e)
    L22, t2 = bchol(S, bt, refine)
    out = torch.zeros((L, nb, n, n), dtype=torch.int32, device=dev)
    out[:, :, :n1, :n1] = L11.limbs
    out[:, :, n1:, :n1] = L21.limbs
    out[:, :, n1:, n1:] = L22.limbs
    return BMP(out, e), t1 + t2


def btrsm_right(B, Lf, tiles, bt=32, refine=1):
    """batched.py:291-305: X with X L^T = B (fixed point)."""
    nb, m, n = B.shape
    e = Lf.exp
    if n <= bt:
        t = tiles[0]
        X = bgemm_nt(B, t.X, out_exp=e, bt_rowexp=t.X.exp)
        for _ in range(refine):
            Rr = badd(B, bgemm_nt(X, t.Lmp, out_exp=e), -1, out_exp=e)
            X = badd(X, bgemm_nt(Rr, t.X, out_exp=e, bt_rowexp=t.X.exp), 1, out_exp=e)
        return X
    n1 = _split(n, bt)
    k1 = _ntiles(n1, bt)
    X1 = btrsm_right(B[:, :n1], Lf[:n1, :n1], tiles[:k1], bt, refine)
    B2 = badd(B[:, n1:], bgemm_nt(X1, Lf[n1:, :n1], out_exp=e), -1, out_exp=e)
    X2 = btrsm_right(B2, Lf[n1:, n1:], tiles[k1:], bt, refine)
    return BMP(torch.cat([X1.limbs, X2.limbs], 3), e)


def _tr(B):
    """limbs of B^T per block, as the 'Bt' operand (row exponents passed separately)"""
    return BMP(B.limbs.transpose(2, 3).contiguous(), 0)


def _bleaf(X, Lm, B, refine):
    """batched.py:313-319: P = Lm^-1 B with the explicit tile inverse (+ refinement steps)."""
    P = bgemm_nt(X, _tr(B), out_exp="col", bt_rowexp=B.expt())
    for _ in range(refine):
        Rr = badd(B, bgemm_nt(Lm, _tr(P), out_exp="col", bt_rowexp=P.expt()), -1, out_exp="align")
        P = badd(P, bgemm_nt(X, _tr(Rr), out_exp="col", bt_rowexp=Rr.expt()), 1, out_exp="align")
    return P


def btrsm_left(Lf, B, tiles, bt=32, refine=0):
    """batched.py:322-335: P = L^-1 B, B (nb, n, m) with per-(block, column) exponents."""
    nb, n, m = B.shape
    if n <= bt:
        t = tiles[0]
        return _bleaf(t.X, t.Lmp, B, refine)
    n1 = _split(n, bt)
    k1 = _ntiles(n1, bt)
    P1 = btrsm_left(Lf[:n1, :n1], B[:n1, :], tiles[:k1], bt, refine)
    U = bgemm_nt(Lf[n1:, :n1], _tr(P1), out_exp="col", bt_rowexp=P1.expt())
    B2 = badd(B[n1:, :], U, -1, out_exp="align")
    P2 = btrsm_left(Lf[n1:, n1:], B2, tiles[k1:], bt, refine)
    ee = torch.maximum(P1.expt(), P2.expt())
    P1, P2 = brescale(P1, ee), brescale(P2, ee)
    return BMP(torch.cat([P1.limbs, P2.limbs], 2), ee)


def btrsm_left_T(Lf, B, tiles, bt=32, refine=1):
    """batched.py:338-352: P = L^-T B."""
    nb, n, m = B.shape
    if n <= bt:
        t = tiles[0]
        XT = BMP(t.X.limbs.transpose(2, 3).contiguous(), t.X.exp)    # per-block uniform exponent
        return _bleaf(XT, t.Lmp.t(), B, refine)
    n1 = _split(n, bt)
    k1 = _ntiles(n1, bt)
    P2 = btrsm_left_T(Lf[n1:, n1:], B[n1:, :], tiles[k1:], bt, refine)
    U = bgemm_nt(Lf[n1:, :n1].t(), _tr(P2), out_exp="col", bt_rowexp=P2.expt())
    B1 = badd(B[:n1, :], U, -1, out_exp="align")
    P1 = btrsm_left_T(Lf[:n1, :n1], B1, tiles[:k1], bt, refine)
    ee = torch.maximum(P1.expt(), P2.expt())
    P1, P2 = brescale(P1, ee), brescale(P2, ee)
    return BMP(torch.cat([P1.limbs, P2.limbs], 2), ee)
