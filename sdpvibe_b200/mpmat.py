"""Block-floating multiprecision matrices and the exact RNS GEMM: drop-in for ``sdpvibe.mpmat``.

An MP matrix holds limbs (int32 (L, rows, cols) limb planes) and exponents (a Python int e0 when
uniform, else an int64 (cols,) tensor): value[i, j] = int(limbs[:, i, j]) * 2**exp[j]
(sdpvibe/mpmat.py:1-8).  gemm_nt computes the exact product with the residue kernels of rns.py and
rounds every entry once.
"""
import ctypes

import torch

from . import _lib
from .rns import RNS, dev
from .limbops import shift_round, add_same, bitlen_words

KC_MAX = 32768            # inner-dimension chunk of one residue GEMM launch (int32 bound of unsigned digits)
RES_BUDGET = 4 << 30      # residue bytes per launch before the moduli are split into groups


class MP:
    """e0: Python int when the exponent is uniform (avoids device syncs), else None."""
    __slots__ = ("limbs", "_exp", "e0")

    def __init__(self, limbs, exp):
        self.limbs = limbs
        if isinstance(exp, int):
            self.e0, self._exp = exp, None
        elif torch.is_tensor(exp) and exp.dim() == 0:
            self.e0, self._exp = None, exp.expand(limbs.shape[2]).clone()
        else:
            self.e0, self._exp = None, exp

    @property
    def exp(self):
        if self._exp is None:
            self._exp = torch.full((self.limbs.shape[2],), self.e0, dtype=torch.int64, device=self.limbs.device)
        return self._exp

    @property
    def shape(self):
        return tuple(self.limbs.shape[1:])

    @property
    def L(self):
        return self.limbs.shape[0]

    def t(self):
        """transpose; requires a single exponent"""
        return MP(self.limbs.transpose(1, 2).contiguous(), self.uniform_exp())

    def uniform_exp(self):
        if self.e0 is not None:
            return self.e0
        e = int(self._exp[0])
        assert bool((self._exp == e).all()), "matrix has per-column exponents"
        self.e0 = e
        return e

    def __getitem__(self, idx):
        r, c = idx
        if self.e0 is not None:
            return MP(self.limbs[:, r, c].contiguous(), self.e0)
        return MP(self.limbs[:, r, c].contiguous(), self._exp[c].contiguous())

    def flat(self):
        return self.limbs.reshape(self.L, -1)


def transpose_rows(B):
    """B (n x m) with per-column exponents -> limbs of B^T (m x n) and the row exponents (m,)"""
    return MP(B.limbs.transpose(1, 2).contiguous(), 0), B.exp


def headroom_bits(L):
    return 32 * L - 32


# ------------------------------------------------------------------ host conversions (tests)
def from_ints(rows, exp, L):
    """rows: list of lists of Python ints (mantissas) -> MP"""
    R, C = len(rows), len(rows[0])
    mask = (1 << 32) - 1
    flat = []
    for row in rows:
        for v in row:
            assert abs(v) < 1 << (32 * L - 1)
            u = v % (1 << (32 * L))
            flat.append([(u >> (32 * k)) & mask for k in range(L)])
    arr = torch.tensor(flat, dtype=torch.int64).view(R, C, L).permute(2, 0, 1).contiguous()
    arr = torch.where(arr >= 1 << 31, arr - (1 << 32), arr).to(torch.int32)
    return MP(arr.to(dev), exp)


def to_ints(A):
    """MP -> list of lists of Python int mantissas, list of column exponents"""
    L = A.L
    a = (A.limbs.cpu().to(torch.int64) % (1 << 32)).permute(1, 2, 0)
    R, C = A.shape
    out = []
    for i in range(R):
        row = []
        for j in range(C):
            v = 0
            for k in reversed(range(L)):
                v = (v << 32) | int(a[i, j, k])
            if v >= 1 << (32 * L - 1):
                v -= 1 << (32 * L)
            row.append(v)
        out.append(row)
    return out, A.exp.cpu().tolist()


# ------------------------------------------------------------------ re-rounding
def _exp_vec(e, C):
    if torch.is_tensor(e):
        return e if e.dim() == 1 else e.expand(C)
    return torch.full((C,), int(e), dtype=torch.int64, device=dev)


def rescale(A, new_exp, Lout=None):
    """re-round A to exponent(s) new_exp (int, 0-d or (cols,) tensor), optionally to Lout limbs
    (sdpvibe/mpmat.py:108-117)"""
    R, C = A.shape
    Lo = Lout or A.L
    if isinstance(new_exp, int) and A.e0 is not None:
        s = torch.full((R * C,), new_exp - A.e0, dtype=torch.int64, device=dev)
        return MP(shift_round(A.flat(), s, Lo).view(Lo, R, C), new_exp)
    ne = _exp_vec(new_exp, C)
    s = (ne - A.exp)[None, :].expand(R, C).reshape(-1)
    return MP(shift_round(A.flat(), s, Lo).view(Lo, R, C), ne.clone())


def bitlen_limbs(X):
    return bitlen_words(X.reshape(X.shape[0], -1))


def normalize(A, mode="mat"):
    R, C = A.shape
    top = bitlen_limbs(A.limbs).view(R, C) + A.exp[None, :]
    t = top.max() if mode == "mat" else top.amax(0)
    return rescale(A, t - headroom_bits(A.L))


def neg(A):
    R, C = A.shape
    return MP(add_same(torch.zeros_like(A.flat()), A.flat(), -1).view(A.L, R, C),
              A.e0 if A.e0 is not None else A.exp.clone())


def add(A, B, alpha=1, out_exp=None):
    """A + alpha*B (alpha = +-1), sdpvibe/mpmat.py:135-156: exact when exponents agree and out_exp
    equals them; 'align' rounds both to the larger exponent + 1 per column; otherwise exact in a wider
    format, then one rounding to out_exp / 'col' / 'mat' / None (= 'mat')."""
    assert A.shape == B.shape and A.L == B.L
    R, C = A.shape
    L = A.L
    if isinstance(out_exp, int) and A.e0 == out_exp and B.e0 == out_exp:
        return MP(add_same(A.flat(), B.flat(), alpha).view(L, R, C), out_exp)
    if out_exp == "align":
        e = torch.maximum(A.exp, B.exp) + 1
        a = rescale(A, e)
        b = rescale(B, e)
        return MP(add_same(a.flat(), b.flat(), alpha).view(L, R, C), e)
    e = torch.minimum(A.exp, B.exp)
    d = int(max((A.exp - e).max(), (B.exp - e).max()))
    Lw = L + (d + 31) // 32 + 2
    a = rescale(A, e, Lw)
    b = rescale(B, e, Lw)
    W = MP(add_same(a.flat(), b.flat(), alpha).view(Lw, R, C), e.clone())
    if out_exp is None or out_exp in ("mat", "col"):
        top = bitlen_limbs(W.limbs).view(R, C) + W.exp[None, :]
        top = top.amax(0) if out_exp == "col" else top.max()
        out_exp = top - headroom_bits(L)
    return rescale(W, out_exp, L)


# ------------------------------------------------------------------ GEMM
_ctx = {}


def moduli_group():
    """the moduli group G of the library's own contexts (the autotuner's SDPV_TUNE_MOD_GROUP knob; 16, the
    reference's, unless its table chose another)"""
    v = ctypes.c_int(16)
    _lib.check(_lib.lib().sdpv_tune_get(4, ctypes.byref(v)), "sdpv_tune_get")
    return v.value


def _context(L, G):
    key = (L, torch.cuda.current_device(), G)
    if key not in _ctx:
        _ctx[key] = RNS(L, G=G)
    return _ctx[key]


def ctx(L):
    """the RNS context of L-limb products in the reference's format (groups of 16 moduli), one per limb count
    and device (sdpvibe/mpmat.py:163-166)"""
    return _context(L, 16)


def lib_ctx(L):
    """the context this library's own products use: the moduli group of the autotuner's table (the results
    are the same bits for every group; only the residue format, internal to each product, differs)"""
    return _context(L, moduli_group())


def residue_product(R, Av, Bv, acc, nb=1, syrk=False, fresh=False, kvalid=None):
    """acc += residues of the exact products of nb stacked blocks: Av (L, nb*M, K), Bv (L, nb*N, K); with
    kvalid only the first kvalid of the K entries of each row are used.  fresh: acc holds no data yet (the
    first K chunk overwrites instead of adding)."""
    K = Av.shape[2] if kvalid is None else kvalid
    rows = Av.shape[1] + (0 if syrk else Bv.shape[1])
    per_mod = rows * min(K, KC_MAX) * 2
    GR = R.n if R.n * per_mod <= RES_BUDGET else max(16, (RES_BUDGET // per_mod) // 16 * 16)
    for k0 in range(0, K, KC_MAX):
        kk = min(KC_MAX, K - k0)
        for g0 in range(0, R.n, GR):
            G = min(GR, R.n - g0)
            Ah, Al = R.residues(Av, k0, kk, g0, G, spread=True, unsigned=True)
            first = fresh and k0 == 0
            if syrk:
                R.accumulate(Ah, Al, None, None, acc, g0, nb=nb, syrk=True, fresh=first, unsigned=True)
            else:
                Bh, Bl = R.residues(Bv, k0, kk, g0, G, spread=True, unsigned=True)
                R.accumulate(Ah, Al, Bh, Bl, acc, g0, nb=nb, fresh=first, unsigned=True)
            del Ah, Al


def residue_product_rows(R, Xr, nI, Rp, K, acc, fresh=False):
    """residue_product(R, X, None, acc, syrk=True) of operand rows (mpf.aligned_rows: nI columns of Rp rows,
    K of them used): acc += residues of X X^T, lower triangle."""
    per_mod = nI * min(K, KC_MAX) * 2
    GR = R.n if R.n * per_mod <= RES_BUDGET else max(128, (RES_BUDGET // per_mod) // 128 * 128)
    for k0 in range(0, K, KC_MAX):                  # KC_MAX is a multiple of 128
        kk = min(KC_MAX, K - k0)
        for g0 in range(0, R.n, GR):
            G = min(GR, R.n - g0)
            Ah, Al = R.residues_rows(Xr, nI, Rp, k0, kk, g0, G)
            R.accumulate(Ah, Al, None, None, acc, g0, syrk=True, fresh=fresh and k0 == 0, unsigned=True)
            del Ah, Al


def gemm_nt(A, Bt, out_exp="col", kc=4096, colblock=None, bt_rowexp=None):
    """C = A @ Bt^T, exact, then rounded (sdpvibe/mpmat.py:169-202).  A: (M, K) single exponent; Bt:
    (N, K) single exponent, or per-row exponents bt_rowexp (N,).  out_exp: 'col', 'mat', or an int /
    (N,) tensor of target exponents.  kc and colblock are accepted for compatibility."""
    M, K = A.shape
    N, K2 = Bt.shape
    assert K == K2
    L = A.L
    R = lib_ctx(L)
    eA = A.uniform_exp()
    e_in = (eA + bt_rowexp) if bt_rowexp is not None else eA + Bt.uniform_exp()
    acc = (torch.empty if K else torch.zeros)((R.n, M, N), dtype=torch.int16, device=dev)
    same = A.limbs.data_ptr() == Bt.limbs.data_ptr() and M == N
    if K:
        if same:
            _same_product(R, A.limbs, acc)
        else:
            residue_product(R, A.limbs, Bt.limbs, acc, syrk=False, fresh=True)
    return _crt_round(acc, e_in, out_exp, L)


def _same_product(R, X, acc):
    """A @ A^T: full square (both triangles), residues computed once."""
    K = X.shape[2]
    for k0 in range(0, K, KC_MAX):
        kk = min(KC_MAX, K - k0)
        Ah, Al = R.residues(X, k0, kk, spread=True, unsigned=True)
        R.accumulate(Ah, Al, Ah, Al, acc, fresh=(k0 == 0), unsigned=True)


def _crt_round(acc, e_in, out_exp, L, colblock=None):
    """sdpvibe/mpmat.py:205-236: CRT, then one rounding to a fixed / per-column ('col') / common
    ('mat', one extra rounding) exponent."""
    R = lib_ctx(L)
    n, M, N = acc.shape
    if colblock is None:
        colblock = max(1, min(N, (1 << 24) // max(M, 1)))
    out = torch.empty((L, M, N), dtype=torch.int32, device=dev)
    fixed = isinstance(e_in, int) and isinstance(out_exp, int)
    if not fixed:
        e_in = _exp_vec(e_in, N)
        exps = torch.empty((N,), dtype=torch.int64, device=dev)
    for j0 in range(0, N, colblock):
        w = min(colblock, N - j0)
        Wd, bl, Bq = R.crt_block(acc, N, j0, w, M)
        if fixed:
            s = torch.full((Bq,), out_exp - e_in, dtype=torch.int64, device=dev)
        else:
            if isinstance(out_exp, str):
                sj = bl.view(M, w).amax(0) - headroom_bits(L)
                ej = e_in[j0:j0 + w] + sj
            else:
                ej = _exp_vec(out_exp, N)[j0:j0 + w]
                sj = ej - e_in[j0:j0 + w]
            s = sj[None, :].expand(M, w).reshape(-1)
            exps[j0:j0 + w] = ej
        out[:, :, j0:j0 + w] = shift_round(Wd, s, L).view(L, M, w)
    if fixed:
        return MP(out, out_exp)
    C = MP(out, exps)
    if out_exp == "mat":
        C = rescale(C, exps.max())
    return C
