"""CPU oracle for the multiprecision hot path -- TEST INFRASTRUCTURE ONLY.

This package is the checker the CUDA path is compared against.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import it; the product
(``sdpvibe_b200``) never does.

* ``liboracle.so`` (``oracle.c``): plain C restatement of the reference's integer kernels.
* this module: numpy bindings plus the RNS tables of ``sdpvibe/rns.py:166-191`` computed with
  Python integers.
* ``oracle.mp``: restatement of the reference's Python orchestration (mpmat / mpf / batched /
  linalg), built on the primitives here.

Parity is pinned: ``tests/test_oracle_golden.py`` checks every primitive against golden vectors
produced by running the reference itself (``tests/golden/make_golden.py``).
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

EZ = -(1 << 40)                                   # sdpvibe/mpf.py:21


def NBITS(L): return 32 * L - 2                   # sdpvibe/mpf.py:223
def headroom_bits(L): return 32 * L - 32          # sdpvibe/mpmat.py:64
def fx_exp(L): return -(32 * L - 40)              # sdpvibe/linalg.py:19


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _LIB
    if _LIB is None:
        so = os.path.join(HERE, "liboracle.so")
        src = os.path.join(HERE, "oracle.c")
        if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
            build()
        _LIB = ctypes.CDLL(so)
    return _LIB


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ------------------------------------------------------------------ limb-plane primitives
def shift_round(X, s, Lout):
    """round_half_up(X / 2^s) to Lout limbs; returns (out (Lout, B) int32, per-entry overflow flags)."""
    X = _c(X, np.int32); s = _c(np.broadcast_to(s, (X.shape[1],)), np.int64)
    Lin, B = X.shape
    out = np.empty((Lout, B), np.int32); flag = np.empty((B,), np.int32)
    lib().or_shift_round(_p(X), ctypes.c_int(Lin), ctypes.c_int64(B), _p(s), ctypes.c_int(Lout), _p(out), _p(flag))
    return out, flag


def add_same(A, B, sgn=1):
    A = _c(A, np.int32); B = _c(B, np.int32)
    out = np.empty_like(A)
    lib().or_add_same(_p(A), _p(B), ctypes.c_int(A.shape[0]), ctypes.c_int64(A.shape[1]), ctypes.c_int(sgn), _p(out))
    return out


def bitlen(X):
    X = _c(X, np.int32)
    L = X.shape[0]; B = int(np.prod(X.shape[1:]))
    out = np.empty((B,), np.int64)
    lib().or_bitlen(_p(X), ctypes.c_int(L), ctypes.c_int64(B), _p(out))
    return out.reshape(X.shape[1:])


def badd_align(A, B, EA, EB, sign):
    """A, B: (L, nb, rows, cols); EA, EB: (nb, cols) -> (out, EO)."""
    A = _c(A, np.int32); B = _c(B, np.int32)
    L, nb, rows, cols = A.shape
    EA = _c(np.broadcast_to(EA, (nb, cols)), np.int64); EB = _c(np.broadcast_to(EB, (nb, cols)), np.int64)
    out = np.empty_like(A); EO = np.empty((nb, cols), np.int64)
    lib().or_badd_align(_p(A), _p(B), _p(EA), _p(EB), ctypes.c_int(L), ctypes.c_int64(nb), ctypes.c_int64(rows),
                        ctypes.c_int64(cols), ctypes.c_int(sign), _p(out), _p(EO))
    return out, EO


def mpf_mul(Am, Ae, Bm, Be):
    Am = _c(Am, np.int32); Bm = _c(Bm, np.int32)
    L = Am.shape[0]; shape = Am.shape[1:]; n = int(np.prod(shape))
    Ae = _c(Ae, np.int64).reshape(-1); Be = _c(Be, np.int64).reshape(-1)
    bs = int(Be.size == 1 and n != 1)
    O = np.empty((L, n), np.int32); eO = np.empty((n,), np.int64)
    lib().or_mpf_mul(ctypes.c_int(L), ctypes.c_int64(n), _p(Am), _p(Ae), _p(Bm), _p(Be), ctypes.c_int(bs), _p(O), _p(eO))
    return O.reshape((L,) + shape), eO.reshape(shape)


def mpf_add(Am, Ae, Bm, Be, sgn=1):
    Am = _c(Am, np.int32); Bm = _c(Bm, np.int32)
    L = Am.shape[0]; shape = Am.shape[1:]; n = int(np.prod(shape))
    Ae = _c(Ae, np.int64).reshape(-1); Be = _c(Be, np.int64).reshape(-1)
    O = np.empty((L, n), np.int32); eO = np.empty((n,), np.int64)
    lib().or_mpf_add(ctypes.c_int(L), ctypes.c_int64(n), _p(Am), _p(Ae), _p(Bm), _p(Be), ctypes.c_int(sgn), _p(O), _p(eO))
    return O.reshape((L,) + shape), eO.reshape(shape)


def mpf_norm(X, eI, L):
    X = _c(X, np.int32); LI, n = X.shape
    eI = _c(np.broadcast_to(eI, (n,)), np.int64)
    O = np.empty((L, n), np.int32); eO = np.empty((n,), np.int64)
    lib().or_mpf_norm(ctypes.c_int(L), ctypes.c_int(LI), ctypes.c_int64(n), _p(X), _p(eI), _p(O), _p(eO))
    return O, eO


# ------------------------------------------------------------------ RNS tables (sdpvibe/rns.py:22-35, 166-191)
def _primes_desc(hi, lo):
    s = np.ones(hi + 1, bool); s[:2] = False
    for p in range(2, int(hi ** 0.5) + 1):
        if s[p]:
            s[p * p::p] = False
    return [int(p) for p in range(hi, lo, -1) if s[p]]


def _sdigits(x, base, n):
    """signed digits in [-base/2, base/2) of a Python int"""
    h = base // 2; out = []
    for _ in range(n):
        r = ((x + h) % base) - h; out.append(r); x = (x - r) // base
    assert x == 0
    return out


def _words(x, W):
    """two's-complement 32-bit words of a Python int"""
    u = x % (1 << (32 * W))
    return [(u >> (32 * k)) & 0xffffffff for k in range(W)]


class RNSTables:
    """Moduli and tables for exact products of L-limb integers with inner dimension <= kmax."""

    def __init__(self, L, kmax=1 << 17, G=16):
        self.L, self.G, self.NB = L, G, 4 * L
        bound = kmax * (1 << (32 * L - 1)) ** 2
        mods, M = [], 1
        for p in _primes_desc(32639, 2 ** 14):
            if M > 4 * bound and len(mods) % G == 0:
                break
            mods.append(p); M *= p
        self.mods, self.M, self.n = mods, M, len(mods)
        self.m32 = np.array(mods, np.int32)
        self.c14 = np.array([pow(2, 14, m) for m in mods], np.int32)
        cen = lambda v, m: v - m if v > m // 2 else v
        T = np.array([[cen(pow(256, j, m), m) for j in range(self.NB)] for m in mods], np.int64)
        self.Tlo = (((T + 64) % 128) - 64).astype(np.int8)
        self.Thi = ((T - self.Tlo) // 128).astype(np.int8)
        self.C1 = np.array([(128 * int(T[i].sum())) % m for i, m in enumerate(mods)], np.int32)
        self.C2 = np.array([pow(2, 32 * L, m) for m in mods], np.int32)
        self.E = (math.ceil(M.bit_length() / 8) + 2 + 7) // 8 * 8
        self.W = self.E // 4
        self.inv = np.array([pow(M // m % m, -1, m) for m in mods], np.int32)
        self.Ct = np.array([_sdigits(M // m, 256, self.E) for m in mods], np.int8).T.copy()   # (E, n)
        self.Md = np.array(_sdigits(M, 256, self.E), np.int32)
        self.Mi_words = np.array([_words(M // m, self.W) for m in mods], np.uint32)          # (n, W)
        self.M_words = np.array(_words(M, self.W), np.uint32)


_TABLES = {}


def tables(L):
    if L not in _TABLES:
        _TABLES[L] = RNSTables(L)
    return _TABLES[L]


def residues(T, X, k0, kc, g0=0, G=None):
    """X (L, rows, ld) int32 -> (hi, lo) (G, rows, kp) int8, kp = kc rounded up to 16."""
    X = _c(X, np.int32)
    L, rows, ld = X.shape
    G = G or T.n
    kp = -(-kc // 16) * 16
    hi = np.empty((G, rows, kp), np.int8); lo = np.empty_like(hi)
    mods = _c(T.m32[g0:g0 + G], np.int32)
    lib().or_residues(_p(X), ctypes.c_int(L), ctypes.c_int64(rows), ctypes.c_int64(ld), ctypes.c_int64(k0),
                      ctypes.c_int64(kc), ctypes.c_int64(kp), _p(mods), ctypes.c_int(G), _p(hi), _p(lo))
    return hi, lo


def accumulate(T, Ahi, Alo, Bhi, Blo, acc, g0=0, lower=False):
    """acc[g0:g0+G] <- (acc + residues of A B^T) mod m, canonical in [0, m) (in place on a copy, returned).
    Exact: per-modulus float64 BLAS products of centred residues (|sum| < 2^53)."""
    G, M, KC = Ahi.shape; N = Bhi.shape[1]
    out = np.array(acc, np.int16, copy=True)
    a = 128 * Ahi.astype(np.float64) + Alo
    b = 128 * Bhi.astype(np.float64) + Blo
    assert KC * (1 << 28) < (1 << 53)
    for g in range(G):
        m = int(T.m32[g0 + g])
        s = np.fmod(a[g] @ b[g].T, m).astype(np.int64)
        v = (s + m + out[g0 + g].astype(np.int64)) % m
        if lower:
            keep = np.tril(np.ones((M, N), bool))
            v = np.where(keep, v, out[g0 + g])
        out[g0 + g] = v.astype(np.int16)
    return out


def crt_block(T, acc, N, j0, w, rows):
    """acc (n, rows_total, N) int16 -> (words (W, rows*w) int32, bit lengths (rows*w,) int64)."""
    acc = _c(acc, np.int16)
    B = rows * w
    out = np.empty((T.W, B), np.int32); bl = np.empty((B,), np.int64)
    mods = _c(T.m32, np.int32); inv = _c(T.inv, np.int32)
    Mi = _c(T.Mi_words, np.uint32); Mw = _c(T.M_words, np.uint32)
    lib().or_crt_block(_p(acc), ctypes.c_int64(acc.shape[1] * acc.shape[2]), ctypes.c_int64(N), ctypes.c_int64(j0),
                       ctypes.c_int64(w), ctypes.c_int64(rows), ctypes.c_int(T.n), _p(mods), _p(inv), _p(Mi),
                       _p(Mw), ctypes.c_int(T.W), _p(out), _p(bl))
    return out, bl


# ------------------------------------------------------------------ Cholesky base case
def chol_tiles(W, BT, WL, LF):
    """W: (nb, BT, BT, WL) uint32 wide fixed point (in place on a copy) -> (L factor, RINV (nb, BT, WL))."""
    A = np.array(W, np.uint32, copy=True)
    nb = A.shape[0]
    RINV = np.zeros((nb, BT, WL), np.uint32)
    lib().or_chol_tiles(_p(A), _p(RINV), ctypes.c_int64(nb), ctypes.c_int(BT), ctypes.c_int(WL), ctypes.c_int(LF))
    return A, RINV


def trinv_tiles(Lw, RINV, BT, WL, LF):
    Lw = _c(Lw, np.uint32); RINV = _c(RINV, np.uint32)
    nb = Lw.shape[0]
    X = np.zeros_like(Lw)
    lib().or_trinv_tiles(_p(Lw), _p(RINV), _p(X), ctypes.c_int64(nb), ctypes.c_int(BT), ctypes.c_int(WL),
                         ctypes.c_int(LF))
    return X


def trsv_tiles(Lt, RINV, V, BT, WL, LF):
    """basecase.py:228-245: y with L y = v for each vector of V (nvec, BT, WL) (one factored tile Lt
    (BT, BT, WL), pivot reciprocals RINV (BT, WL)) -> Y (nvec, BT, WL)."""
    Lt = _c(Lt, np.uint32); RINV = _c(RINV, np.uint32)
    Y = np.array(V, np.uint32, copy=True)
    nvec = Y.shape[0]
    lib().or_trsv_tiles(_p(Lt), _p(RINV), _p(Y), ctypes.c_int64(nvec), ctypes.c_int(BT), ctypes.c_int(WL),
                        ctypes.c_int(LF))
    return Y


def to_limbs(values, L):
    """Python ints -> (L, n) int32 limb planes (two's complement)."""
    return np.array([[((v >> (32 * k)) + (1 << 31)) % (1 << 32) - (1 << 31) for v in values]
                     for k in range(L)], dtype=np.int32).reshape(L, len(values))


def to_ints(X):
    """(L, ...) int32 limb planes -> flat list of Python ints."""
    X = np.asarray(X)
    L = X.shape[0]
    u = (X.reshape(L, -1).astype(np.int64) & 0xffffffff).T
    out = []
    for row in u:
        v = 0
        for k in range(L - 1, -1, -1):
            v = (v << 32) | int(row[k])
        if v >= 1 << (32 * L - 1):
            v -= 1 << (32 * L)
        out.append(v)
    return out
