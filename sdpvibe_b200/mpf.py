"""Per-entry multiprecision floating point arrays on B200: drop-in for ``sdpvibe.mpf``.

MPF: m int32 (L, *shape) limb planes (little endian, two's complement), e int64 (*shape);
value = m * 2^e; normalised: |m| has NB = 32L-2 bits (zero: m = 0, e = EZ) (sdpvibe/mpf.py:1-10).

Elementwise operations are libsdpv_b200 kernels with the reference's rounding (magnitude half up).
``gemm`` aligns rows of op(A) / columns of op(B), forms the exact product with the residue kernels and
renormalises each entry inside the CRT kernel (one launch for CRT + rounding).  ``GramAcc`` keeps
Q = sum_c P_c^T P_c in residue form across chunks (lower-triangle tiles only) with one CRT at the end.
"""
import os

import mpmath as mp
import numpy as np
import torch

from . import _lib, graphs
from .limbops import shift_round, bitlen_words
from .mpmat import lib_ctx, KC_MAX, RES_BUDGET
from .rns import dev

EZ = -(1 << 40)                                      # exponent of zero (sdpvibe/mpf.py:21)
LMAX_WIDE = 160


class MPF:
    __slots__ = ("m", "e")

    def __init__(self, m, e):
        self.m, self.e = m, e

    @property
    def L(self):
        return self.m.shape[0]

    @property
    def shape(self):
        return tuple(self.e.shape)

    def __getitem__(self, idx):
        if not isinstance(idx, tuple):
            idx = (idx,)
        return MPF(self.m[(slice(None),) + idx].contiguous(), self.e[idx].contiguous())

    @property
    def T(self):
        """transpose of the last two dimensions"""
        return MPF(self.m.transpose(-1, -2).contiguous(), self.e.transpose(-1, -2).contiguous())

    def reshape(self, *s):
        return MPF(self.m.reshape(self.L, *s), self.e.reshape(*s))

    def clone(self):
        return MPF(self.m.clone(), self.e.clone())

    def __neg__(self):
        return add(zeros(self.shape, self.L), self, -1)

    def __add__(self, o):
        return add(self, o, 1)

    def __sub__(self, o):
        return add(self, o, -1)

    def shift(self, k):
        """multiply by 2^k (k: int or tensor broadcastable to shape) -- exact"""
        e = self.e + k
        return MPF(self.m, torch.where(self.e == EZ, EZ, e))

    def to_mp(self):
        """-> numpy object array of mpmath mpf (host; tests / scalars)"""
        L = self.L
        a = self.m.reshape(L, -1).t().contiguous().cpu().numpy().astype(np.uint32)
        ex = self.e.reshape(-1).cpu().numpy()
        out = np.empty(a.shape[0], dtype=object)
        for i in range(a.shape[0]):
            v = int.from_bytes(a[i].tobytes(), "little", signed=True)
            out[i] = mp.mpf(0) if v == 0 else mp.mpf((v, int(ex[i])))
        return out.reshape(self.shape)

    def to_float(self):
        """approximate float64 values (with exponent clamping); host numpy"""
        if self.L > 1:
            top = self.m[-1].double() * 2.0 ** 32 + (self.m[-2].double() % 2.0 ** 32)
        else:
            top = self.m[-1].double()
        sc = (self.e + 32 * (self.L - 2)).clamp(-1100, 1100).double()
        v = torch.where(self.e == EZ, torch.zeros_like(top), top * torch.pow(2.0, sc))
        return v.cpu().numpy()


def zeros(shape, L):
    return MPF(torch.zeros((L, *shape), dtype=torch.int32, device=dev),
               torch.full(shape, EZ, dtype=torch.int64, device=dev))


def NBITS(L):
    return 32 * L - 2


def from_ints(ints, exps, L, shape):
    """Python ints (mantissas) and exponents (flat lists) -> normalised MPF"""
    n = len(ints)
    nb = 4 * L
    buf = bytearray(nb * n)
    for i, v in enumerate(ints):
        buf[i * nb:(i + 1) * nb] = int(v).to_bytes(nb, "little", signed=True)
    m = torch.from_numpy(np.frombuffer(bytes(buf), dtype=np.int32).reshape(n, L).T.copy()).to(dev)
    e = torch.tensor(exps, dtype=torch.int64, device=dev)
    return normalize(m, e, L).reshape(*shape)


def _dec_to_bin(t, NBb):
    """decimal string -> (signed mantissa with <= NBb bits, binary exponent) (sdpvibe/mpf.py:238-261)"""
    t = t.strip()
    neg = t.startswith("-")
    if t[0] in "+-":
        t = t[1:]
    e10 = 0
    if "e" in t or "E" in t:
        t, ex = t.replace("E", "e").split("e")
        e10 = int(ex)
    if "." in t:
        ip, fp = t.split(".")
        e10 -= len(fp)
        t = ip + fp
    man = int(t) if t else 0
    if man == 0:
        return 0, EZ
    if e10 >= 0:
        v = man * 10 ** e10
        bl = v.bit_length()
        if bl <= NBb:
            return (-v if neg else v), 0
        sh = bl - NBb
        v = (v + (1 << (sh - 1))) >> sh
        return (-v if neg else v), sh
    den = 10 ** (-e10)
    sh = NBb + den.bit_length() - man.bit_length() + 1
    q = ((man << sh) + den // 2) // den
    ex = -sh
    while q.bit_length() > NBb:
        q = (q + 1) >> 1
        ex += 1
    return (-q if neg else q), ex


def from_strings(strs, L, shape=None):
    NBb = NBITS(L)
    ints, exps = [], []
    for t in strs:
        m, e = _dec_to_bin(t, NBb)
        ints.append(m)
        exps.append(e)
    return from_ints(ints, exps, L, shape or (len(ints),))


def strings_to_host(strs, L):
    """decimal strings -> (limbs int32 (n, L) entry-major numpy, exps int64 numpy); CPU only"""
    NBb = NBITS(L)
    nb = 4 * L
    n = len(strs)
    buf = bytearray(nb * n)
    exps = np.empty(n, dtype=np.int64)
    for i, t in enumerate(strs):
        m, e = _dec_to_bin(t, NBb)
        buf[i * nb:(i + 1) * nb] = m.to_bytes(nb, "little", signed=True)
        exps[i] = e
    return np.frombuffer(bytes(buf), dtype=np.int32).reshape(n, L), exps


def host_to_mpf(limbs, exps, L, shape):
    m = torch.from_numpy(np.ascontiguousarray(limbs.T)).to(dev)
    e = torch.from_numpy(exps).to(dev)
    return normalize(m, e, L).reshape(*shape)


def from_mp(vals, L, shape=None):
    """iterable of mpmath numbers / strings -> MPF (rounded to NB bits, half up on magnitude)"""
    vals = list(vals)
    NBb = NBITS(L)
    ints, exps = [], []
    for v in vals:
        v = mp.mpf(v)
        if v == 0:
            ints.append(0)
            exps.append(EZ)
            continue
        sign, man, ex, bc = v._mpf_
        if bc > NBb:
            sh = bc - NBb
            man = (man + (1 << (sh - 1))) >> sh
            ex += sh
        ints.append(-man if sign else man)
        exps.append(ex)
    return from_ints(ints, exps, L, shape or (len(vals),))


# ------------------------------------------------------------------ elementwise kernels
def from_float(V, L):
    """float64 array (numpy, or a torch tensor on the device) -> MPF, exactly: the significand shifted to
    NB bits on the device (sdpvibe/solver.py:1012-1018).  A non-finite value becomes zero and sets the
    overflow bit of the device error word (``_lib.device_error_flags``)."""
    if torch.is_tensor(V):
        Vd = V.to(device=dev, dtype=torch.float64).contiguous()
    else:
        Vd = torch.from_numpy(np.ascontiguousarray(V, dtype=np.float64)).to(dev)
    shape = tuple(Vd.shape)
    n = Vd.numel()
    O = torch.empty((L, n), dtype=torch.int32, device=dev)
    eO = torch.empty((n,), dtype=torch.int64, device=dev)
    _lib.call("sdpv_mpf_from_f64", L, n, _lib.ptr(Vd), _lib.ptr(O), _lib.ptr(eO), _lib.stream())
    return MPF(O, eO).reshape(*shape)


def normalize(Xw, ein, L):
    """Xw: (LI, n) int32 wide two's complement, ein (n,) -> normalised MPF (n,) (sdpvibe/mpf.py:307-313)"""
    LI, n = Xw.shape
    assert LI <= LMAX_WIDE
    Xw = Xw.contiguous()
    ein = ein.contiguous()
    O = torch.empty((L, n), dtype=torch.int32, device=dev)
    eO = torch.empty((n,), dtype=torch.int64, device=dev)
    _lib.call("sdpv_mpf_norm", L, LI, n, _lib.ptr(Xw), _lib.ptr(ein), _lib.ptr(O), _lib.ptr(eO), _lib.stream())
    return MPF(O, eO)


def mul(A, B):
    """entrywise product; B may be a single entry (broadcast) (sdpvibe/mpf.py:316-323)"""
    L = A.L
    n = A.e.numel()
    bs = B.e.numel() == 1
    assert bs or B.shape == A.shape
    Am, Ae, Bm, Be = A.m.contiguous(), A.e.contiguous(), B.m.contiguous(), B.e.contiguous()
    O = torch.empty_like(Am)
    eO = torch.empty_like(Ae)
    _lib.call("sdpv_mpf_mul", L, n, _lib.ptr(Am), _lib.ptr(Ae), _lib.ptr(Bm), _lib.ptr(Be), int(bs), _lib.ptr(O),
              _lib.ptr(eO), _lib.stream())
    return MPF(O, eO)


def add(A, B, sgn=1):
    """entrywise A + sgn*B (sdpvibe/mpf.py:326-331)"""
    assert A.shape == B.shape, (A.shape, B.shape)
    L = A.L
    n = A.e.numel()
    Am, Ae, Bm, Be = A.m.contiguous(), A.e.contiguous(), B.m.contiguous(), B.e.contiguous()
    O = torch.empty_like(Am)
    eO = torch.empty_like(Ae)
    _lib.call("sdpv_mpf_add", L, n, _lib.ptr(Am), _lib.ptr(Ae), _lib.ptr(Bm), _lib.ptr(Be), int(sgn), _lib.ptr(O),
              _lib.ptr(eO), _lib.stream())
    return MPF(O, eO)


def scalar(v, L):
    return from_mp([v], L, (1,))


def eye(n, L, val=1):
    A = zeros((n, n), L)
    d = from_mp([val], L, (1,))
    idx = torch.arange(n, device=dev)
    A.m[:, idx, idx] = d.m[:, :1]
    A.e[idx, idx] = d.e[0]
    return A


# ------------------------------------------------------------------ reductions (host results)
def _top(A):
    """per-entry e + bitlen (log2 of magnitude, roughly); EZ for zeros (sdpvibe/mpf.py:348-351)"""
    bl = bitlen_words(A.m.reshape(A.L, -1)).view(A.shape)
    return torch.where(A.e == EZ, torch.full_like(A.e, EZ), A.e + bl)


def total(A):
    """exact-ish sum of all entries -> mpmath mpf (sdpvibe/mpf.py:354-366)"""
    L = A.L
    n = A.e.numel()
    if n == 0:
        return mp.mpf(0)
    t = int(A.e.max()) - 32
    if t < EZ // 2:
        return mp.mpf(0)
    s = (t - A.e.reshape(-1))
    W = shift_round(A.m.reshape(L, -1), s, L + 2)
    S = (W.to(torch.int64) & 0xFFFFFFFF).sum(1)
    top = W[-1].to(torch.int64).sum()
    S = S.cpu().tolist()
    top = int(top)
    v = sum(int(S[k]) << (32 * k) for k in range(L + 1)) + (top << (32 * (L + 1)))
    return mp.mpf((v, t)) if v else mp.mpf(0)


def dot(A, B):
    return total(mul(A, B))


def max_abs(A):
    if A.e.numel() == 0:
        return mp.mpf(0)
    tp = _top(A).reshape(-1)
    t = int(tp.max())
    if t <= EZ // 2:
        return mp.mpf(0)
    cand = torch.nonzero(tp >= t - 1).reshape(-1)
    Af = A.reshape(-1)
    vals = MPF(Af.m[:, cand], Af.e[cand]).shift(-t).to_float()
    i = int(cand[int(np.argmax(np.abs(vals)))])
    return abs(Af[i:i + 1].to_mp()[0])


def trace(A):
    n = A.shape[0]
    idx = torch.arange(n, device=dev)
    return total(MPF(A.m[:, idx, idx], A.e[idx, idx]))


# ------------------------------------------------------------------ GEMM
def _dims3(A):
    """(nb, R, C) view sizes of a 2-D or 3-D MPF."""
    sh = A.shape
    return (1,) + tuple(sh) if len(sh) == 2 else tuple(sh)


def top_max(A, over_rows):
    """max of top = e + bitlen over the rows (over_rows=True -> per column, (nb, C)) or over the
    columns (-> per row, (nb, R)) of a 2-D / 3-D MPF, in one kernel."""
    nb, R, C = _dims3(A)
    m, e = A.m.contiguous(), A.e.contiguous()
    out = torch.empty((nb, C if over_rows else R), dtype=torch.int64, device=m.device)
    _lib.call("sdpv_top_max", _lib.ptr(m), _lib.ptr(e), A.L, nb, R, C, 0 if over_rows else 1, _lib.ptr(out),
              _lib.stream())
    return out


def aligned(A, target, per_col, transpose, Lout=None, ld=None):
    """Mantissas of A rounded to the exponents target (nb, R) per row or (nb, C) per column, as Lout
    limbs, optionally transposed to (Lout, nb, C, R) -- or (Lout, nb, C, ld), ld >= R, with rows R .. ld - 1
    unset; zero entries give 0 (one kernel)."""
    nb, R, C = _dims3(A)
    Lout = Lout or A.L
    m, e = A.m.contiguous(), A.e.contiguous()
    if transpose and ld is not None:
        out = torch.empty((Lout, nb, C, ld), dtype=torch.int32, device=m.device)
        _lib.call("sdpv_align_t", _lib.ptr(m), _lib.ptr(e), A.L, nb, R, C, _lib.ptr(target.contiguous()), int(per_col),
                  Lout, ld, _lib.ptr(out), _lib.stream())
        return out
    out = torch.empty((Lout, nb, C, R) if transpose else (Lout, nb, R, C), dtype=torch.int32, device=m.device)
    _lib.call("sdpv_align", _lib.ptr(m), _lib.ptr(e), A.L, nb, R, C, _lib.ptr(target.contiguous()), int(per_col),
              int(transpose), Lout, _lib.ptr(out), _lib.stream())
    return out


def aligned_rows(A, target, per_col, Lout, Rp):
    """aligned(A, target, per_col, transpose=True, Lout) as operand rows for RNS.residues_rows: (nb, C, Rp,
    rb) uint8, row (b, c, r) = the Lout limbs' bytes, a sign byte, zeros (rb = 128 bytes for Lout <= 31, 256
    for Lout <= 63); rows R .. Rp - 1 zero (one kernel)."""
    nb, R, C = _dims3(A)
    rb = 128 if Lout <= 31 else 256
    m, e = A.m.contiguous(), A.e.contiguous()
    out = torch.empty((nb, C, Rp, rb), dtype=torch.uint8, device=m.device)
    _lib.call("sdpv_align_rows", _lib.ptr(m), _lib.ptr(e), A.L, nb, R, C, _lib.ptr(target.contiguous()), int(per_col),
              Lout, Rp, _lib.ptr(out), _lib.stream())
    return out


def _row_exponents(tmax, L):
    """mpf.py:394-395: common exponent max(top) - NB per row, 0 for all-zero rows."""
    E = tmax - NBITS(L)
    return torch.where(E < EZ // 2, torch.zeros_like(E), E)


def _align_rows(A):
    """A (..., R, K) -> (mantissas (L, ..., R, K) with a common exponent per row, row exps (..., R))
    (sdpvibe/mpf.py:390-398)."""
    E = _row_exponents(top_max(A, over_rows=False), A.L)
    out = aligned(A, E, per_col=False, transpose=False)
    return out.view(A.m.shape), E.view(A.shape[:-1])


def gemm(A, B, transA=False, transB=False):
    """C = op(A) op(B) (2-d, or batched 3-d (nb, ., .)); exact products, every entry rounded once
    (operands aligned per row of op(A) / column of op(B)) (sdpvibe/mpf.py:401-452)."""
    if A.e.dim() == 2:
        A1 = MPF(A.m[:, None], A.e[None])
        B1 = MPF(B.m[:, None], B.e[None])
        C = gemm(A1, B1, transA, transB)
        return MPF(C.m[:, 0], C.e[0])
    # op(A) rows and op(B) columns aligned to their own exponents; the transposes are fused into the
    # alignment kernel (stored A is (nb, K, M) when transA; stored B is (nb, K, N) unless transB)
    nb = A.shape[0]
    M = A.shape[2] if transA else A.shape[1]
    K = A.shape[1] if transA else A.shape[2]
    N = B.shape[1] if transB else B.shape[2]
    K2 = B.shape[2] if transB else B.shape[1]
    assert K == K2 and B.shape[0] == nb, (A.shape, B.shape)
    L = A.L
    rA = _row_exponents(top_max(A, over_rows=transA), L)            # (nb, M)
    Am = aligned(A, rA, per_col=transA, transpose=transA)          # (L, nb, M, K)
    cB = _row_exponents(top_max(B, over_rows=not transB), L)        # (nb, N)
    Bm = aligned(B, cB, per_col=not transB, transpose=not transB)  # (L, nb, N, K)
    R = lib_ctx(L)
    acc = (torch.empty if K else torch.zeros)((R.n, nb * M, N), dtype=torch.int16, device=dev)
    if K:
        from .mpmat import residue_product
        residue_product(R, Am.view(L, nb * M, K), Bm.view(L, nb * N, K), acc, nb=nb, fresh=True)
    Om, Oe = R.crt_norm(acc, N, 0, N, nb * M, rA.reshape(-1), cB, L, rows_per_block=M)
    return MPF(Om.view(L, nb, M, N), Oe.view(nb, M, N))


def symmetrize(A):
    """(A + A^T)/2"""
    return add(A, A.T).shift(-1)


# ------------------------------------------------------------------ Gram accumulation (Q = sum_c P_c^T P_c)
class GramAcc:
    """Q = sum over chunks of P_c^T P_c, accumulated exactly in residues (lower-triangle tiles only)
    against running column reference exponents E_j, reconstructed by one CRT
    (sdpvibe/mpf.py:536-630).  A column that outgrows its HEAD bits of headroom forces a flush (CRT of
    the partial sum, added in MPF).  Only the lower triangle of the result is defined.

    The flush decision is taken on the device (one bookkeeping kernel per chunk computes the predicate and the
    exponents; a predicated CRT, a predicated in-place MPF add and a predicated zeroing instead of a host
    branch), so ``add`` never waits for the GPU and a whole accumulation can be captured in a CUDA graph; the
    arithmetic, and so every bit of the result, is that of the host-branch formulation."""
    HEAD = 28
    OPERAND_ROWS = False       # True: align to operand rows and decompose them (sdpv_align_rows / _residues_rows)

    def __init__(self, N, L, E_ref=None):
        self.N, self.L = N, L
        self.R = lib_ctx(L + 1)
        self.E = (E_ref.to(torch.int64).contiguous().clone() if E_ref is not None
                  else torch.full((N,), EZ, dtype=torch.int64, device=dev))
        self.Tmax = torch.full((N,), EZ, dtype=torch.int64, device=dev)
        self.acc = None
        self.part = None                       # sum of the flushed partial sums (zero until the first flush)
        self._nflush = torch.zeros((), dtype=torch.int64, device=dev)
        self._f = torch.zeros((), dtype=torch.int32, device=dev)          # this chunk's flush predicate
        self._rE = torch.empty((N,), dtype=torch.int64, device=dev)       # the flush's CRT exponents
        self._target = torch.empty((1, N), dtype=torch.int64, device=dev)  # the chunk's alignment targets

    @property
    def flushes(self):
        return int(self._nflush)

    def add(self, P):
        """P: MPF (rows, N)."""
        L, N, R = self.L, self.N, self.R
        tp = top_max(P, over_rows=True)[0]                           # column tops (mpf.py:563)
        # flush predicate, the flush's CRT exponents (old E), the E / Tmax updates and the alignment targets
        # (mpf.py:564-575) in one launch; the flush itself runs predicated on the device
        had_acc = self.acc is not None
        _lib.call("sdpv_gram_columns", N, _lib.ptr(tp), _lib.ptr(self.E), _lib.ptr(self.Tmax), self.HEAD, NBITS(L),
                  int(had_acc), _lib.ptr(self._rE), _lib.ptr(self._target), _lib.ptr(self._f),
                  _lib.ptr(self._nflush), _lib.stream())
        if had_acc:
            self._flush_if()
        rows = P.shape[0]
        if self.acc is None:
            # rows padded to a multiple of 8 entries (16 bytes) for the vectorised GEMM epilogue
            self.acc = torch.zeros((R.n, N, -(-N // 8) * 8), dtype=torch.int16, device=dev)
        if not rows:
            return
        target = self._target
        if self.OPERAND_ROWS and L + 1 <= 63:
            # columns aligned to E_j - NB in L+1 limbs as operand rows (column j's rows padded to a multiple of
            # 128), decomposed straight from them
            from .mpmat import residue_product_rows
            Rp = -(-rows // 128) * 128
            Xr = aligned_rows(P, target, per_col=True, Lout=L + 1, Rp=Rp)
            residue_product_rows(R, Xr, N, Rp, rows, self.acc)
        else:
            # columns aligned in L+1 limbs and transposed to (N, rows) limb planes (row length padded to a
            # multiple of 4: 16-byte aligned rows for the decomposition's bulk copies), one kernel
            from .mpmat import residue_product
            ld = -(-rows // 4) * 4
            X = aligned(P, target, per_col=True, transpose=True, Lout=L + 1, ld=ld).view(L + 1, N, ld)
            residue_product(R, X, None, self.acc, syrk=True, kvalid=rows)

    def _crt(self, pred=None, rE=None):
        L, N, R = self.L, self.N, self.R
        if rE is None:
            rE = torch.where(self.E > EZ // 2, self.E - NBITS(L), torch.zeros_like(self.E))
        Om, Oe = R.crt_norm(self.acc, self.acc.shape[2], 0, N, N, rE, rE[None, :], L, pred=pred)
        return MPF(Om.view(L, N, N), Oe.view(N, N))

    def _flush_if(self):
        """where the chunk's flush predicate holds (device int32): part += CRT(acc) at the previous reference
        exponents, acc = 0 (the flush count was advanced by sdpv_gram_columns).  part starts at zero, and
        0 + q is q itself (q is normalised), so the first flush gives the reference's part = q."""
        fi = self._f
        q = self._crt(pred=fi, rE=self._rE)
        if self.part is None:
            self.part = zeros((self.N, self.N), self.L)
        n = self.N * self.N
        _lib.call("sdpv_mpf_add_if", self.L, n, _lib.ptr(self.part.m), _lib.ptr(self.part.e), _lib.ptr(q.m),
                  _lib.ptr(q.e), 1, _lib.ptr(self.part.m), _lib.ptr(self.part.e), _lib.ptr(fi), _lib.stream())
        _lib.call("sdpv_zero_if", _lib.ptr(self.acc), self.acc.numel() * 2, _lib.ptr(fi), _lib.stream())

    def next_reference(self, margin=4):
        return torch.where(self.Tmax > EZ // 2, self.Tmax + margin, self.Tmax)

    def precision_loss(self):
        ok = (self.Tmax > EZ // 2) & (self.E > EZ // 2)
        return int((self.E - self.Tmax)[ok].max()) if bool(ok.any()) else 0

    def result(self):
        if self.acc is None:
            return self.part
        q = self._crt()
        self.acc = None
        return q if self.part is None else add(self.part, q)


# ------------------------------------------------------------------ Cholesky (equilibrated, batched)
def fx_exp(L):
    """exponent of the equilibrated fixed-point format (sdpvibe/linalg.py:19)"""
    return -(32 * L - 40)


_FX_ONE = {}


def _fx_one(L, efx):
    """the fixed-point 1 (L limbs at exponent efx) on this device, made once"""
    key = (L, efx, torch.cuda.current_device())
    if key not in _FX_ONE:
        one = from_mp([1], L, (1,))
        _FX_ONE[key] = shift_round(one.m, torch.tensor([efx - int(one.e[0])], device=dev), L)[:, 0].clone()
    return _FX_ONE[key]


class _Prepared:
    """One batch (nb, n, n) equilibrated as sdpvibe/mpf.py:467-492 does: k_i = floor((top_ii + 1) / 2), the
    fixed-point matrix A_ij 2^-(k_i + k_j) at exponent fx_exp(L), padded to npad (a multiple of 32) with the
    fixed-point identity."""

    def __init__(self, A, bt):
        L = A.L
        nb, n, _ = A.shape
        self.nb, self.n, self.L = nb, n, L
        idx = torch.arange(n, device=dev)
        tpd = _top(A)[:, idx, idx]                                  # (nb, n)
        self.bad = ((A.m[-1][:, idx, idx] < 0) | (tpd <= EZ // 2)).any()
        self.k = torch.div(tpd + 1, 2, rounding_mode="floor")      # A_ii < 2^(2k)
        self.npad = max(bt, (n + bt - 1) // bt * bt)
        efx = fx_exp(L)
        s = (efx - (A.e - self.k[:, :, None] - self.k[:, None, :])).reshape(-1)
        s = torch.where(A.e.reshape(-1) == EZ, torch.full_like(s, 1 << 30), s)
        Af = shift_round(A.m.reshape(L, -1), s, L).view(L, nb, n, n)
        P = torch.zeros((L, nb, self.npad, self.npad), dtype=torch.int32, device=dev)
        P[:, :, :n, :n] = Af
        if self.npad > n:
            ii = torch.arange(n, self.npad, device=dev)
            P[:, :, ii, ii] = _fx_one(L, efx)[:, None, None]
        self.P = P


class CholGroup:
    """Cholesky factors of several batches of blocks of different sizes, A_b = L_b L_b^T with L_b = D^-1 Lt_b,
    D = diag(2^-k) (sdpvibe/mpf.py:461-532), factored together by the grouped work-list engine
    (``grouped``): one launch sequence for all blocks, each block's factor bit-identical to the reference's
    Chol of its own batch.  As: list of MPF (nb_i, n_i, n_i) (or (n, n))."""

    SOLVE_REFINE = int(os.environ.get("SDPB_GPU_SOLVE_REFINE", "0"))

    def __init__(self, As, bt=32, refine=1, defer_check=False):
        from . import grouped
        if bt != 32:
            raise ValueError("the base tiles are 32 x 32")
        if self.SOLVE_REFINE:
            raise ValueError("SDPB_GPU_SOLVE_REFINE: the grouped triangular solves implement refine = 0 only")
        self.two_d = [A.e.dim() == 2 for A in As]
        As = [MPF(A.m[:, None], A.e[None]) if t else A for A, t in zip(As, self.two_d)]
        self.L = L = As[0].L
        self.bt, self.refine = bt, refine
        self.efx = fx_exp(L)
        self.prep = [_Prepared(A, bt) for A in As]
        self.bad = torch.stack([p.bad for p in self.prep]).any() if len(self.prep) > 1 else self.prep[0].bad
        if not defer_check and bool(self.bad):                      # one host sync
            raise ValueError("matrix is not positive definite (diagonal)")
        self.fac = grouped.Factorisation([p.P for p in self.prep], self.efx, refine)

    def _solve_all(self, lower, Bs):
        """L^-1 B (lower) or L^-T B for one right-hand-side batch per factored batch, all in one grouped solve"""
        from . import grouped
        Bs = [MPF(B.m[:, None], B.e[None]) if t else B for B, t in zip(Bs, self.two_d)]
        m = Bs[0].shape[-1]
        assert all(B.shape[-1] == m for B in Bs), "one right-hand-side count per grouped solve"
        L = self.L
        state = [self.fac.Fa, self.fac.Xa, self.fac.xe]
        ins = [t for B, p in zip(Bs, self.prep) for t in (B.m.contiguous(), B.e.contiguous(), p.k)] + state
        shapes = tuple((p.nb, p.n, p.npad) for p in self.prep)

        def fn(ins):
            rhs = []
            for q, p in enumerate(self.prep):
                Bm, Be, k = ins[3 * q:3 * q + 3]
                B = MPF(Bm, Be).shift(-k[:, :, None]) if lower else MPF(Bm, Be)
                Am, cE = _align_rows(B.T)                          # per column: (L, nb, m, n)
                Pm = torch.zeros((L, p.nb, p.npad, m), dtype=torch.int32, device=dev)
                Pm[:, :, :p.n] = Am.transpose(2, 3)
                rhs.append((Pm, cE))
            Fa, Xa, xe = ins[3 * len(self.prep):]
            outs = grouped.solve(self.fac, rhs, lower, Fa, Xa, xe)
            res = []
            for p, (Pm, pe) in zip(self.prep, outs):
                X = Pm[:, :, :p.n].reshape(L, -1)
                ein = pe[:, None, :].expand(p.nb, p.n, m).reshape(-1)
                Y = normalize(X.contiguous(), ein.contiguous(), L).reshape(p.nb, p.n, m)
                res.append(Y.m)
                res.append(Y.e)
            return res

        def post(q, Y):
            return Y if lower else Y.shift(-self.prep[q].k[:, :, None])
        key = ("gsolve", lower, L, shapes, m, self.efx)
        flat = graphs.run(key, fn, ins)
        out = []
        for q, t in enumerate(self.two_d):
            Y = post(q, MPF(flat[2 * q], flat[2 * q + 1]))
            out.append(MPF(Y.m[:, 0], Y.e[0]) if t else Y)
        return out

    def solve_lower(self, Bs):
        """L^-1 B = Lt^-1 (D B) for each batch"""
        return self._solve_all(True, Bs)

    def solve_upper(self, Bs):
        """L^-T B = D (Lt^-T B) for each batch"""
        return self._solve_all(False, Bs)

    def solve(self, Bs):
        """A^-1 B for each batch"""
        return self.solve_upper(self.solve_lower(Bs))


class Chol(CholGroup):
    """A = L L^T per block, with L = D^-1 Lt, D = diag(2^-k): Lt fixed point, k integer
    (sdpvibe/mpf.py:461-532).  A: MPF (n, n) or batched (nb, n, n); padded internally to a multiple of
    bt with the fixed-point identity.  defer_check: instead of raising here (one host synchronisation),
    leave the positivity flag of the diagonal in self.bad (a device bool) for the caller to test later."""

    def __init__(self, A, bt=32, refine=1, defer_check=False):
        super().__init__([A], bt, refine, defer_check)
        p = self.prep[0]
        self.nb, self.n, self.npad, self.k = p.nb, p.n, p.npad, p.k
        if self.two_d[0]:
            self.k = p.k                                           # (1, n): as the reference's 3-d view

    @property
    def Lt(self):
        """the fixed-point factor as a BMP (L, nb, npad, npad) at exponent fx_exp(L) (zero above the diagonal)"""
        from .batched import BMP
        return BMP(self.fac.dense(0), self.efx)

    @property
    def tiles(self):
        """the diagonal tiles' factors and inverses, in order (each a BTile: X with one exponent per block)"""
        from .batched import BMP, BTile
        out = []
        for j in range(self.npad // 32):
            Xm, xe, Lm = self.fac.diag_tile(0, j)
            t = BTile()
            t.X = BMP(Xm, xe[:, None].expand(self.nb, 32).contiguous())
            t.Lmp = BMP(Lm, self.efx)
            out.append(t)
        return out

    def diag_limbs(self):
        """limbs of the diagonal of the fixed-point factor, (L, nb, n)"""
        return self.fac.diagonal(0)[:, :, :self.n]

    def solve_lower(self, B):
        """L^-1 B = Lt^-1 (D B)"""
        return self._solve_all(True, [B])[0]

    def solve_upper(self, B):
        """L^-T B = D (Lt^-T B)"""
        return self._solve_all(False, [B])[0]

    def solve(self, B):
        """A^-1 B"""
        return self.solve_upper(self.solve_lower(B))


def chol_solve_many(pairs):
    """[(A_b, B_b)] -> [A_b^-1 B_b] for independent batched systems of different block sizes (the reference's
    callers make one Chol + solve per bucket of blocks of equal padded size).  All batches are factored and
    solved together by the grouped engine -- one work-list launch sequence, no buckets; the results are those
    of the separate calls.  The positivity checks are read at the end, in one transfer (ValueError as Chol
    raises it)."""
    if not pairs:
        return []
    ch = CholGroup([A for A, _ in pairs], defer_check=True)
    out = ch.solve([B for _, B in pairs])
    if bool(ch.bad):
        raise ValueError("matrix is not positive definite (diagonal)")
    return out
