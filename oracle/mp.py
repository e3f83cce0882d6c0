"""Oracle restatement of the reference's multiprecision orchestration -- TEST INFRASTRUCTURE ONLY.

numpy in, numpy out, built on the C primitives of ``oracle``.  Each function follows the reference
function it names (file:line).  Block-floating matrices ("MP") are (limbs (L, R, C), exp) with exp a
Python int or an int64 array (C,); per-entry floats ("MPF") are (m (L, *shape), e (*shape)).
"""
import numpy as np

from . import (EZ, NBITS, headroom_bits, fx_exp, tables, residues, accumulate, crt_block, shift_round, add_same,
               bitlen, mpf_norm, mpf_add, mpf_mul, badd_align, chol_tiles, trinv_tiles)


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


# ------------------------------------------------------------------ batched fixed-point (sdpvibe/batched.py)
# A BMP is (limbs (L, nb, R, C), exp) with exp a Python int or an int64 array (nb, C).
def expt(exp, nb, C):
    if isinstance(exp, (int, np.integer)):
        return np.full((nb, C), int(exp), np.int64)
    return np.asarray(exp, np.int64)


def bslice(limbs, exp, r, c):
    """BMP.__getitem__ (batched.py:33-36)."""
    e = exp if isinstance(exp, (int, np.integer)) else np.ascontiguousarray(np.asarray(exp)[:, c])
    return np.ascontiguousarray(limbs[:, :, r, c]), e


def brescale(limbs, exp, new_exp, Lout=None):
    """batched.py:45-52."""
    L, nb, R, C = limbs.shape
    Lo = Lout or L
    if isinstance(new_exp, (int, np.integer)) and isinstance(exp, (int, np.integer)):
        out, _ = shift_round(limbs.reshape(L, -1), np.full((nb * R * C,), int(new_exp) - int(exp), np.int64), Lo)
        return out.reshape(Lo, nb, R, C), int(new_exp)
    ne = np.asarray(new_exp, np.int64) if not isinstance(new_exp, (int, np.integer)) else np.full((nb, C), int(new_exp), np.int64)
    s = np.broadcast_to((ne - expt(exp, nb, C))[:, None, :], (nb, R, C)).reshape(-1)
    out, _ = shift_round(limbs.reshape(L, -1), s, Lo)
    return out.reshape(Lo, nb, R, C), ne.copy()


def _bcrt_round(T, acc, nb, M, N, e_in, out_exp, L):
    """batched.py:200-231 (column blocks do not change results)."""
    Wd, bl = crt_block(T, acc, N, 0, N, nb * M)
    fixed = isinstance(e_in, (int, np.integer)) and isinstance(out_exp, (int, np.integer))
    if fixed:
        out, _ = shift_round(Wd, np.full((nb * M * N,), int(out_exp) - int(e_in), np.int64), L)
        return out.reshape(L, nb, M, N), int(out_exp)
    e_in = expt(e_in, nb, N)
    if isinstance(out_exp, str):
        sj = bl.reshape(nb, M, N).max(1) - headroom_bits(L)
        ej = e_in + sj
    else:
        ej = np.full((nb, N), int(out_exp), np.int64)
        sj = ej - e_in
    out, _ = shift_round(Wd, np.broadcast_to(sj[:, None, :], (nb, M, N)).reshape(-1), L)
    out = out.reshape(L, nb, M, N)
    if isinstance(out_exp, (int, np.integer)):
        return out, int(out_exp)
    if out_exp == "mat":
        return brescale(out, ej, np.broadcast_to(ej.max(1, keepdims=True), (nb, N)).copy())
    return out, ej


def bgemm_nt(A, eA, Bt, eB, out_exp="col", bt_rowexp=None):
    """batched.py:165-197: C[b] = A[b] Bt[b]^T exact, then rounded."""
    L, nb, M, K = A.shape
    N = Bt.shape[2]
    T = tables(L)
    acc = np.zeros((T.n, nb * M, N), np.int16)
    for b in range(nb):
        acc[:, b * M:(b + 1) * M] = exact_acc(T, np.ascontiguousarray(A[:, b]), np.ascontiguousarray(Bt[:, b]))
    eA_ = eA if isinstance(eA, (int, np.integer)) else np.asarray(eA)[:, 0]
    eBv = eB if bt_rowexp is None else bt_rowexp
    if isinstance(eA_, (int, np.integer)) and isinstance(eBv, (int, np.integer)):
        e_in = int(eA_) + int(eBv)
    else:
        eA_t = np.asarray(eA_, np.int64) if not isinstance(eA_, (int, np.integer)) else np.full((nb,), int(eA_), np.int64)
        eB_t = np.asarray(eBv, np.int64) if not isinstance(eBv, (int, np.integer)) else np.full((nb, N), int(eBv), np.int64)
        if eB_t.ndim == 1:
            eB_t = np.broadcast_to(eB_t[:, None], (nb, N))
        e_in = eA_t[:, None] + eB_t
    return _bcrt_round(T, acc, nb, M, N, e_in, out_exp, L)


def badd(A, eA, B, eB, alpha=1, out_exp=None):
    """batched.py:82-92."""
    L, nb, R, C = A.shape
    if isinstance(out_exp, (int, np.integer)) and isinstance(eA, (int, np.integer)) and \
            isinstance(eB, (int, np.integer)) and eA == out_exp and eB == out_exp:
        return add_same(A.reshape(L, -1), B.reshape(L, -1), alpha).reshape(A.shape), int(out_exp)
    assert out_exp == "align"
    return badd_align(A, B, expt(eA, nb, C), expt(eB, nb, C), alpha)


class BTile:
    __slots__ = ("X", "Xe", "Lmp", "Le")


def _soa_to_aos(X):
    return np.ascontiguousarray(np.moveaxis(X, 0, -1))


def _aos_to_soa(X):
    return np.ascontiguousarray(np.moveaxis(X, -1, 0))


def bchol_tile(A, e, LI=24):
    """batched.py:243-262: 32x32 base case in WL = L+24 limbs, F = 32L fraction bits."""
    L, nb, b, _ = A.shape
    LF, WL = L, L + LI
    F = 32 * LF
    Ws, _ = brescale(A, e, -F, WL)
    W = _soa_to_aos(Ws).view(np.uint32)                       # (nb, b, b, WL)
    Lw, RINV = chol_tiles(W, b, WL, LF)
    tri = np.tril(np.ones((b, b), bool))
    Lw[:, ~tri] = 0
    X = trinv_tiles(Lw, RINV, b, WL, LF)
    Lout, _ = brescale(_aos_to_soa(Lw.view(np.int32)), -F, e, L)
    Xs = _aos_to_soa(X.view(np.int32))                        # (WL, nb, b, b)
    top = bitlen(Xs).reshape(nb, b * b).max(1) - F
    ex = np.broadcast_to((top - headroom_bits(L))[:, None], (nb, b)).copy()
    t = BTile()
    t.Lmp, t.Le = Lout, e
    t.X, t.Xe = brescale(Xs, np.full((nb, b), -F, np.int64), ex, L)
    return Lout, t


def _split(n, bt):
    return (n // 2 + bt - 1) // bt * bt


def _ntiles(n, bt):
    if n <= bt:
        return 1
    n1 = _split(n, bt)
    return _ntiles(n1, bt) + _ntiles(n - n1, bt)


def bchol(A, e, bt=32, refine=1):
    """batched.py:274-288: recursive Cholesky of equilibrated fixed-point blocks (exp e int)."""
    L, nb, n, _ = A.shape
    if n <= bt:
        assert n == bt
        Lt, t = bchol_tile(A, e)
        return Lt, [t]
    n1 = _split(n, bt)
    L11, t1 = bchol(np.ascontiguousarray(A[:, :, :n1, :n1]), e, bt, refine)
    L21 = btrsm_right(np.ascontiguousarray(A[:, :, n1:, :n1]), e, L11, e, t1, bt, refine)
    G, _ = bgemm_nt(L21, e, L21, e, out_exp=e)
    S, _ = badd(np.ascontiguousarray(A[:, :, n1:, n1:]), e, G, e, -1, out_exp=e)
    L22, t2 = bchol(S, e, bt, refine)
    out = np.zeros((L, nb, n, n), np.int32)
    out[:, :, :n1, :n1] = L11
    out[:, :, n1:, :n1] = L21
    out[:, :, n1:, n1:] = L22
    return out, t1 + t2


def btrsm_right(B, eB, Lf, e, tiles, bt=32, refine=1):
    """batched.py:291-305: X with X L^T = B (fixed point, exponent e)."""
    L, nb, m, n = B.shape
    if n <= bt:
        t = tiles[0]
        X, _ = bgemm_nt(B, eB, t.X, t.Xe, out_exp=e, bt_rowexp=t.Xe)
        for _ in range(refine):
            G, _ = bgemm_nt(X, e, t.Lmp, t.Le, out_exp=e)
            Rr, _ = badd(B, eB, G, e, -1, out_exp=e)
            D, _ = bgemm_nt(Rr, e, t.X, t.Xe, out_exp=e, bt_rowexp=t.Xe)
            X, _ = badd(X, e, D, e, 1, out_exp=e)
        return X
    n1 = _split(n, bt)
    k1 = _ntiles(n1, bt)
    X1 = btrsm_right(np.ascontiguousarray(B[:, :, :, :n1]), eB, np.ascontiguousarray(Lf[:, :, :n1, :n1]), e,
                     tiles[:k1], bt, refine)
    G, _ = bgemm_nt(X1, e, np.ascontiguousarray(Lf[:, :, n1:, :n1]), e, out_exp=e)
    B2, _ = badd(np.ascontiguousarray(B[:, :, :, n1:]), eB, G, e, -1, out_exp=e)
    X2 = btrsm_right(B2, e, np.ascontiguousarray(Lf[:, :, n1:, n1:]), e, tiles[k1:], bt, refine)
    return np.concatenate([X1, X2], 3)


def _tr(B):
    return np.ascontiguousarray(np.swapaxes(B, 2, 3))


def _bleaf(X, Xe, Lm, Le, B, eB, refine):
    """batched.py:313-319: P = Lm^-1 B with the explicit tile inverse."""
    nb, m = B.shape[1], B.shape[3]
    P, Pe = bgemm_nt(X, Xe, _tr(B), 0, out_exp="col", bt_rowexp=expt(eB, nb, m))
    for _ in range(refine):
        U, Ue = bgemm_nt(Lm, Le, _tr(P), 0, out_exp="col", bt_rowexp=expt(Pe, nb, m))
        Rr, Re = badd(B, eB, U, Ue, -1, out_exp="align")
        D, De = bgemm_nt(X, Xe, _tr(Rr), 0, out_exp="col", bt_rowexp=expt(Re, nb, m))
        P, Pe = badd(P, Pe, D, De, 1, out_exp="align")
    return P, Pe


def btrsm_left(Lf, e, B, eB, tiles, bt=32, refine=0):
    """batched.py:322-335: P = L^-1 B, per-(block, column) exponents."""
    L, nb, n, m = B.shape
    if n <= bt:
        t = tiles[0]
        return _bleaf(t.X, t.Xe, t.Lmp, t.Le, B, eB, refine)
    n1 = _split(n, bt)
    k1 = _ntiles(n1, bt)
    P1, P1e = btrsm_left(np.ascontiguousarray(Lf[:, :, :n1, :n1]), e, np.ascontiguousarray(B[:, :, :n1, :]), eB,
                         tiles[:k1], bt, refine)
    U, Ue = bgemm_nt(np.ascontiguousarray(Lf[:, :, n1:, :n1]), e, _tr(P1), 0, out_exp="col",
                     bt_rowexp=expt(P1e, nb, m))
    B2, B2e = badd(np.ascontiguousarray(B[:, :, n1:, :]), eB, U, Ue, -1, out_exp="align")
    P2, P2e = btrsm_left(np.ascontiguousarray(Lf[:, :, n1:, n1:]), e, B2, B2e, tiles[k1:], bt, refine)
    ee = np.maximum(expt(P1e, nb, m), expt(P2e, nb, m))
    P1, _ = brescale(P1, P1e, ee)
    P2, _ = brescale(P2, P2e, ee)
    return np.concatenate([P1, P2], 2), ee


def btrsm_left_T(Lf, e, B, eB, tiles, bt=32, refine=1):
    """batched.py:338-352: P = L^-T B."""
    L, nb, n, m = B.shape
    if n <= bt:
        t = tiles[0]
        return _bleaf(_tr(t.X), t.Xe, _tr(t.Lmp), t.Le, B, eB, refine)
    n1 = _split(n, bt)
    k1 = _ntiles(n1, bt)
    P2, P2e = btrsm_left_T(np.ascontiguousarray(Lf[:, :, n1:, n1:]), e, np.ascontiguousarray(B[:, :, n1:, :]), eB,
                           tiles[k1:], bt, refine)
    U, Ue = bgemm_nt(_tr(Lf[:, :, n1:, :n1]), e, _tr(P2), 0, out_exp="col", bt_rowexp=expt(P2e, nb, m))
    B1, B1e = badd(np.ascontiguousarray(B[:, :, :n1, :]), eB, U, Ue, -1, out_exp="align")
    P1, P1e = btrsm_left_T(np.ascontiguousarray(Lf[:, :, :n1, :n1]), e, B1, B1e, tiles[:k1], bt, refine)
    ee = np.maximum(expt(P1e, nb, m), expt(P2e, nb, m))
    P1, _ = brescale(P1, P1e, ee)
    P2, _ = brescale(P2, P2e, ee)
    return np.concatenate([P1, P2], 2), ee


def mpf_from_int_value(v, L):
    """Normalised MPF of a Python integer (from_mp([v], L) of sdpvibe/mpf.py:291-304 for integers)."""
    m, e = mpf_norm(np.array([[v]], np.int32) if L == 1 else _int_limbs(v, L), np.zeros(1, np.int64), L)
    return m, e


def _int_limbs(v, L):
    u = v % (1 << (32 * L))
    return np.array([[((u >> (32 * k)) + (1 << 31)) % (1 << 32) - (1 << 31)] for k in range(L)], np.int32)


class Chol:
    """mpf.py:461-532: A = L L^T per block with L = D^-1 Lt, D = diag(2^-k) (Lt fixed point, k integer);
    blocks padded to a multiple of bt with the fixed-point identity."""
    SOLVE_REFINE = 0

    def __init__(self, Am, Ae, bt=32, refine=1):
        self.two_d = Ae.ndim == 2
        if self.two_d:
            Am, Ae = Am[:, None], Ae[None]
        L, nb, n, _ = Am.shape
        self.nb, self.n, self.L, self.bt, self.refine = nb, n, L, bt, refine
        idx = np.arange(n)
        tpd = top(Am, Ae)[:, idx, idx]
        if bool((Am[-1][:, idx, idx] < 0).any()) or bool((tpd <= EZ // 2).any()):
            raise ValueError("matrix is not positive definite (diagonal)")
        k = (tpd + 1) // 2
        self.k = k
        npad = max(bt, (n + bt - 1) // bt * bt)
        self.npad = npad
        efx = fx_exp(L)
        s = (efx - (Ae - k[:, :, None] - k[:, None, :])).reshape(-1)
        s = np.where(Ae.reshape(-1) == EZ, 1 << 30, s)
        Af, _ = shift_round(Am.reshape(L, -1), s, L)
        P = np.zeros((L, nb, npad, npad), np.int32)
        P[:, :, :n, :n] = Af.reshape(L, nb, n, n)
        if npad > n:
            om, oe = mpf_from_int_value(1, L)
            onefx, _ = shift_round(om, np.array([efx - int(oe[0])], np.int64), L)
            ii = np.arange(n, npad)
            P[:, :, ii, ii] = onefx[:, :1, None]
        self.efx = efx
        self.Lt, self.tiles = bchol(P, efx, bt, refine)

    def _to_bmp(self, Bm, Be):
        L = self.L
        TBm, TBe = _T(Bm, Be)                                   # rows of B^T = columns of B
        al, cE = align_rows(TBm, TBe)                           # (L, nb, m, n), (nb, m)
        P = np.zeros((L, self.nb, self.npad, Bm.shape[-1]), np.int32)
        P[:, :, :self.n] = np.swapaxes(al, 2, 3)
        return P, cE

    def _from_bmp(self, P, Pe):
        L, m = self.L, P.shape[3]
        X = np.ascontiguousarray(P[:, :, :self.n]).reshape(L, -1)
        ein = np.broadcast_to(expt(Pe, self.nb, m)[:, None, :], (self.nb, self.n, m)).reshape(-1)
        om, oe = mpf_norm(X, ein, L)
        return om.reshape(L, self.nb, self.n, m), oe.reshape(self.nb, self.n, m)

    def _io(self, Bm, Be, f):
        if self.two_d:
            m, e = f(Bm[:, None], Be[None])
            return m[:, 0], e[0]
        return f(Bm, Be)

    def solve_lower(self, Bm, Be):
        def f(Bm, Be):
            sh = np.where(Be == EZ, EZ, Be - self.k[:, :, None])
            P, Pe = btrsm_left(self.Lt, self.efx, *self._to_bmp(Bm, sh), self.tiles, self.bt, self.SOLVE_REFINE)
            return self._from_bmp(P, Pe)
        return self._io(Bm, Be, f)

    def solve_upper(self, Bm, Be):
        def f(Bm, Be):
            P, Pe = btrsm_left_T(self.Lt, self.efx, *self._to_bmp(Bm, Be), self.tiles, self.bt, self.SOLVE_REFINE)
            m, e = self._from_bmp(P, Pe)
            return m, np.where(e == EZ, EZ, e - self.k[:, :, None])
        return self._io(Bm, Be, f)

    def solve(self, Bm, Be):
        return self.solve_upper(*self.solve_lower(Bm, Be))


def mpf_from_float(V, L):
    """solver.py:1012-1018: float64 array -> MPF exactly (53-bit mantissa as two 32-bit limbs, then
    mpf_norm).  Returns (m (L, *shape), e (*shape))."""
    V = np.asarray(V, dtype=np.float64)
    m, e = np.frexp(V)
    mi = (m * 2.0 ** 53).astype(np.int64).reshape(-1)
    w = np.stack([(mi & 0xFFFFFFFF).astype(np.uint32).view(np.int32), (mi >> 32).astype(np.int32)])
    ein = np.where(mi != 0, e.reshape(-1).astype(np.int64) - 53, EZ)
    om, oe = mpf_norm(w, ein, L)
    return om.reshape(L, *V.shape), oe.reshape(V.shape)
