"""Oracle restatement of the reference's multiprecision orchestration -- TEST INFRASTRUCTURE ONLY.

numpy in, numpy out, built on the C primitives of ``oracle``.  Each function follows the reference
function it names (file:line).  Block-floating matrices ("MP") are (limbs (L, R, C), exp) with exp a
Python int or an int64 array (C,); per-entry floats ("MPF") are (m (L, *shape), e (*shape)).
"""
import numpy as np

from . import (EZ, NBITS, headroom_bits, fx_exp, tables, residues, accumulate, crt_block, shift_round, add_same,
               bitlen, mpf_norm, mpf_add, mpf_mul, badd_align)


def _vec(e, C):
    if isinstance(e, (int, np.integer)):
        return np.full((C,), int(e), np.int64)
    e = np.asarray(e, np.int64)
    return np.broadcast_to(e, (C,)).copy() if e.ndim == 0 else e.copy()


def exact_acc(T, A, Bt, lower=False):
    """Residue accumulator (n, M, N) of the exact product A @ Bt^T (A (L, M, K), Bt (L, N, K))."""
    M, K = A.shape[1:]
    N = Bt.shape[1]
    acc = np.zeros((T.n, M, N), np.int16)
    if K == 0:
        return acc
    ah, al = residues(T, A, 0, K)
    bh, bl = residues(T, Bt, 0, K)
    return accumulate(T, ah, al, bh, bl, acc, 0, lower)


# ------------------------------------------------------------------ mpmat (sdpvibe/mpmat.py)
def rescale(limbs, exp, new_exp, Lout=None):
    """mpmat.py:108-117: re-round to exponent(s) new_exp."""
    L, R, C = limbs.shape
    Lo = Lout or L
    if isinstance(new_exp, (int, np.integer)) and isinstance(exp, (int, np.integer)):
        out, _ = shift_round(limbs.reshape(L, -1), np.full((R * C,), int(new_exp) - int(exp), np.int64), Lo)
        return out.reshape(Lo, R, C), int(new_exp)
    ne = _vec(new_exp, C)
    s = np.broadcast_to((ne - _vec(exp, C))[None, :], (R, C)).reshape(-1)
    out, _ = shift_round(limbs.reshape(L, -1), s, Lo)
    return out.reshape(Lo, R, C), ne


def crt_round(T, acc, e_in, out_exp, L):
    """mpmat.py:205-236: CRT of the residue accumulator, output exponent fixed / 'col' / 'mat'."""
    n, M, N = acc.shape
    Wd, bl = crt_block(T, acc, N, 0, N, M)                     # entries i*N + j
    fixed = isinstance(e_in, (int, np.integer)) and isinstance(out_exp, (int, np.integer))
    if fixed:
        out, _ = shift_round(Wd, np.full((M * N,), int(out_exp) - int(e_in), np.int64), L)
        return out.reshape(L, M, N), int(out_exp)
    e_in = _vec(e_in, N)
    if isinstance(out_exp, str):
        sj = bl.reshape(M, N).max(0) - headroom_bits(L)
        ej = e_in + sj
    else:
        ej = _vec(out_exp, N)
        sj = ej - e_in
    out, _ = shift_round(Wd, np.broadcast_to(sj[None, :], (M, N)).reshape(-1), L)
    out = out.reshape(L, M, N)
    if out_exp == "mat":
        return rescale(out, ej, int(ej.max()))
    return out, ej


def gemm_nt(A, eA, Bt, eB, out_exp="col", bt_rowexp=None):
    """mpmat.py:169-202: C = A @ Bt^T exact, then rounded (panel splitting does not change results)."""
    L = A.shape[0]
    T = tables(L)
    e_in = (int(eA) + np.asarray(bt_rowexp, np.int64)) if bt_rowexp is not None else int(eA) + int(eB)
    acc = exact_acc(T, A, Bt)
    return crt_round(T, acc, e_in, out_exp, L)


def mp_add(A, eA, B, eB, alpha=1, out_exp=None):
    """mpmat.py:135-156."""
    L, R, C = A.shape
    if isinstance(out_exp, (int, np.integer)) and isinstance(eA, (int, np.integer)) and \
            isinstance(eB, (int, np.integer)) and eA == out_exp and eB == out_exp:
        return add_same(A.reshape(L, -1), B.reshape(L, -1), alpha).reshape(L, R, C), int(out_exp)
    ea, eb = _vec(eA, C), _vec(eB, C)
    if out_exp == "align":
        e = np.maximum(ea, eb) + 1
        a, _ = rescale(A, ea, e); b, _ = rescale(B, eb, e)
        return add_same(a.reshape(L, -1), b.reshape(L, -1), alpha).reshape(L, R, C), e
    e = np.minimum(ea, eb)
    d = int(max((ea - e).max(), (eb - e).max()))
    Lw = L + (d + 31) // 32 + 2
    a, _ = rescale(A, ea, e, Lw); b, _ = rescale(B, eb, e, Lw)
    W = add_same(a.reshape(Lw, -1), b.reshape(Lw, -1), alpha).reshape(Lw, R, C)
    if out_exp is None or out_exp in ("mat", "col"):
        top = bitlen(W).reshape(R, C) + e[None, :]
        top = top.max(0) if out_exp == "col" else top.max()
        out_exp = top - headroom_bits(L)
    return rescale(W, e, out_exp, L)


# ------------------------------------------------------------------ mpf (sdpvibe/mpf.py)
def top(m, e):
    """mpf.py:348-351: per-entry e + bitlen, EZ for zeros."""
    bl = bitlen(m)
    return np.where(e == EZ, EZ, e + bl)


def align_rows(m, e):
    """mpf.py:390-398: common exponent per row (last axis) -> (mantissas, row exponents)."""
    L = m.shape[0]
    tp = top(m, e)
    E = tp.max(-1) - NBITS(L)
    E = np.where(E < EZ // 2, 0, E)
    s = E[..., None] - e
    s = np.where(e == EZ, 1 << 30, s)
    out, _ = shift_round(m.reshape(L, -1), s.reshape(-1), L)
    return out.reshape(m.shape), E


def _T(m, e):
    return np.ascontiguousarray(np.swapaxes(m, -1, -2)), np.ascontiguousarray(np.swapaxes(e, -1, -2))


def mpf_gemm(Am, Ae, Bm, Be, transA=False, transB=False):
    """mpf.py:401-452: C = op(A) op(B); rows of op(A) / columns of op(B) aligned, exact product,
    CRT, renormalised per entry."""
    two_d = Ae.ndim == 2
    if two_d:
        Am, Ae, Bm, Be = Am[:, None], Ae[None], Bm[:, None], Be[None]
    if transA:
        Am, Ae = _T(Am, Ae)
    if not transB:
        Bm, Be = _T(Bm, Be)
    L, nb, M, K = Am.shape
    N = Bm.shape[2]
    T = tables(L)
    A_al, rA = align_rows(Am, Ae)
    B_al, cB = align_rows(Bm, Be)
    out_m = np.empty((L, nb, M, N), np.int32)
    out_e = np.empty((nb, M, N), np.int64)
    for b in range(nb):
        acc = exact_acc(T, A_al[:, b], B_al[:, b])
        Wd, _ = crt_block(T, acc, N, 0, N, M)
        ein = (rA[b][:, None] + cB[b][None, :]).reshape(-1)
        m, e = mpf_norm(Wd, ein, L)
        out_m[:, b] = m.reshape(L, M, N)
        out_e[b] = e.reshape(M, N)
    if two_d:
        return out_m[:, 0], out_e[0]
    return out_m, out_e


class GramAcc:
    """mpf.py:536-630: Q = sum_c P_c^T P_c accumulated in residues against running column reference
    exponents, one CRT at the end; a column outgrowing its HEAD bits of headroom forces a flush.
    Only the lower triangle (row >= column) of the result is defined."""
    HEAD = 28

    def __init__(self, N, L, E_ref=None):
        self.N, self.L = N, L
        self.T = tables(L + 1)
        self.E = np.array(E_ref, np.int64, copy=True) if E_ref is not None else np.full((N,), EZ, np.int64)
        self.Tmax = np.full((N,), EZ, np.int64)
        self.acc = None
        self.part = None
        self.flushes = 0

    def add(self, Pm, Pe):
        L, N = self.L, self.N
        tp = top(Pm, Pe).max(0)
        live = tp > EZ // 2
        self.Tmax = np.maximum(self.Tmax, tp)
        known = self.E > EZ // 2
        if bool((live & known & (tp > self.E + self.HEAD)).any()):
            self._flush()
            self.E = np.where(live & (tp > self.E), tp, self.E)
            known = self.E > EZ // 2
        self.E = np.where(live & ~known, tp, self.E)
        PTm, PTe = _T(Pm, Pe)                                   # (L, N, rows), (N, rows)
        rows = PTm.shape[2]
        s = (self.E - NBITS(L))[:, None] - PTe
        s = np.where(PTe == EZ, 1 << 30, s)
        X, _ = shift_round(PTm.reshape(L, -1), s.reshape(-1), L + 1)
        X = X.reshape(L + 1, N, rows)
        if self.acc is None:
            self.acc = np.zeros((self.T.n, N, N), np.int16)
        if rows:
            ah, al = residues(self.T, X, 0, rows)
            self.acc = accumulate(self.T, ah, al, ah, al, self.acc, 0, lower=True)

    def _crt(self):
        L, N = self.L, self.N
        rE = np.where(self.E > EZ // 2, self.E - NBITS(L), 0)
        Wd, _ = crt_block(self.T, self.acc, N, 0, N, N)
        ein = (rE[:, None] + rE[None, :]).reshape(-1)
        m, e = mpf_norm(Wd, ein, L)
        return m.reshape(L, N, N), e.reshape(N, N)

    def _flush(self):
        if self.acc is None:
            return
        q = self._crt()
        self.part = q if self.part is None else mpf_add(*self.part, *q, 1)
        self.acc = None
        self.flushes += 1

    def next_reference(self, margin=4):
        return np.where(self.Tmax > EZ // 2, self.Tmax + margin, self.Tmax)

    def precision_loss(self):
        ok = (self.Tmax > EZ // 2) & (self.E > EZ // 2)
        return int((self.E - self.Tmax)[ok].max()) if bool(ok.any()) else 0

    def result(self):
        if self.acc is None:
            return self.part
        q = self._crt()
        self.acc = None
        return q if self.part is None else mpf_add(*self.part, *q, 1)
