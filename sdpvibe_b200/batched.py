"""Batched multiprecision linear algebra over many equal-sized blocks: drop-in for ``sdpvibe.batched``.

A BMP holds a stack of nb matrices: limbs int32 (L, nb, R, C) limb planes and exp, a Python int
(uniform) or an (nb, C) int64 tensor (sdpvibe/batched.py:16-42).  brescale / badd / bgemm_nt are one
kernel each (bgemm_nt: the exact residue GEMM of rns.py over all nb blocks in one launch, then one CRT and
one rounding).  bchol and the triangular solves keep the reference's signatures and results and run on the
grouped work-list engine (``grouped``).
"""
import torch

from . import _lib
from .rns import dev
from .mpmat import lib_ctx, headroom_bits, residue_product
from .limbops import shift_round, add_same, bitlen_words


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
    R = lib_ctx(L)
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
    R = lib_ctx(L)
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
    """A diagonal tile of a factorisation: X (its inverse, one exponent per block) and Lmp (its factor)."""
    __slots__ = ("X", "Lmp")


# ------------------------------------------------------------------ factorisation and solves (drop-in API)
# The reference's recursive bchol / btrsm_* (sdpvibe/batched.py:274-352).  Here they run on the grouped
# work-list engine (sdpvibe_b200.grouped), which computes the same products and roundings for every block.

def _tiles_of(fac, e):
    out = []
    for j in range(fac.batches[0][1]):
        Xm, xe, Lm = fac.diag_tile(0, j)
        t = BTile()
        t.X = BMP(Xm, xe[:, None].expand(Xm.shape[1], 32).contiguous())
        t.Lmp = BMP(Lm, e)
        out.append(t)
    return out


def bchol(A, bt=32, refine=1):
    """batched.py:274-288: batched Cholesky of equilibrated fixed-point blocks -> (L, tiles)."""
    from . import grouped
    assert bt == 32 and isinstance(A.exp, int)
    fac = grouped.Factorisation([A.limbs], A.exp, refine)
    return BMP(fac.dense(0), A.exp), _tiles_of(fac, A.exp)


def _factor(Lf, tiles):
    from . import grouped
    return grouped.factor_from_tiles(Lf.limbs, Lf.exp, [t.X.limbs for t in tiles], [t.X.exp[:, 0] for t in tiles])


def btrsm_right(B, Lf, tiles, bt=32, refine=1):
    """batched.py:291-305: X with X L^T = B (fixed point, B at L's exponent)."""
    from . import grouped
    assert bt == 32
    return BMP(grouped.right_solve(_factor(Lf, tiles), B.limbs, refine), Lf.exp)


def _left(Lf, B, tiles, refine, lower):
    from . import grouped
    if refine:
        raise NotImplementedError("the grouped triangular solves implement refine = 0 (the solver's setting)")
    nb, n, m = B.shape
    out = grouped.solve(_factor(Lf, tiles), [(B.limbs.contiguous(), B.expt().contiguous())], lower)
    Pm, pe = out[0]
    return BMP(Pm[:, :, :n].contiguous(), pe)


def btrsm_left(Lf, B, tiles, bt=32, refine=0):
    """batched.py:322-335: P = L^-1 B, B (nb, n, m) with per-(block, column) exponents."""
    return _left(Lf, B, tiles, refine, True)


def btrsm_left_T(Lf, B, tiles, bt=32, refine=0):
    """batched.py:338-352: P = L^-T B (the solver calls it with refine = 0)."""
    return _left(Lf, B, tiles, refine, False)
