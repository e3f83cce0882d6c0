"""SDPB's primal-dual interior point iteration on the B200 multiprecision kernels: drop-in for the
hot-path call sites of ``sdpvibe.solver`` (sdpvibe/solver.py).

The solver itself is host orchestration: every matrix operation is an ``mpf`` call (GEMM through
the residue kernels, Cholesky / triangular solves through the batched recursion and the base-case
tiles, elementwise arithmetic through the limb kernels), and scalars (objectives, mu, step lengths)
are mpmath numbers on the host, as in the reference.  Operations are issued in the reference's
order, so that with bit-identical kernels every iterate is bit-identical.

Contents:
  batched-MPF helpers (put, sub, masked, copy_lower_to_upper, diag_of, add_diag, set_diag_where,
  col_scale, bexpand, dup, fold, flat_rows)                      sdpvibe/solver.py:24-116
  step length: min_eig, refine_min_eig, step_from_eig, ...       sdpvibe/solver.py:996-1103
  SDP (synthetic block structures) and Solver.run                sdpvibe/solver.py:424-982
"""
import os
import sys
import time

import mpmath as mp
import numpy as np
import torch

from . import mpf as F
from .mpf import MPF, mul, add, gemm, symmetrize, total, dot, max_abs, Chol, EZ
from .rns import dev


# ------------------------------------------------------------------ batched MPF helpers (nb, R, C)
def put(dst, r0, c0, src):
    """write src into dst[..., r0:, c0:] (in place)"""
    r1, c1 = r0 + src.shape[-2], c0 + src.shape[-1]
    dst.m[..., r0:r1, c0:c1] = src.m
    dst.e[..., r0:r1, c0:c1] = src.e


def sub(A, r0, r1, c0, c1):
    """contiguous copy of A[..., r0:r1, c0:c1]"""
    return MPF(A.m[..., r0:r1, c0:c1].contiguous(), A.e[..., r0:r1, c0:c1].contiguous())


def masked(A, M):
    """A with the entries where the boolean M (broadcast to A's shape) is False set to zero"""
    keep = M.expand(A.shape)
    return MPF(A.m * keep[None].to(A.m.dtype), torch.where(keep, A.e, torch.full_like(A.e, EZ)))


def copy_lower_to_upper(A):
    """symmetric matrix from the lower triangle of each (.., n, n) slice"""
    n = A.shape[-1]
    low = torch.tril(torch.ones(n, n, dtype=torch.bool, device=A.e.device))
    mT, eT = A.m.transpose(-1, -2), A.e.transpose(-1, -2)
    return MPF(torch.where(low, A.m, mT).contiguous(), torch.where(low, A.e, eT).contiguous())


def _diag_idx(A):
    return torch.arange(A.shape[-1], device=A.e.device)


def diag_of(A):
    """diagonal of each (.., n, n) slice as a column (.., n, 1)"""
    i = _diag_idx(A)
    return MPF(A.m[..., i, i].unsqueeze(-1).contiguous(), A.e[..., i, i].unsqueeze(-1).contiguous())


def _with_diag(A, dm, de):
    i = _diag_idx(A)
    m, e = A.m.clone(), A.e.clone()
    m[..., i, i] = dm
    e[..., i, i] = de
    return MPF(m, e)


def add_diag(A, s, dmask=None):
    """A + s on the diagonal (only where dmask (nb, n) is True); s an MPF scalar"""
    i = _diag_idx(A)
    dm, de = A.m[..., i, i].contiguous(), A.e[..., i, i].contiguous()
    sm = s.m.reshape(s.L, *([1] * de.dim())).expand(dm.shape).contiguous()
    se = s.e.reshape([1] * de.dim()).expand(de.shape).contiguous()
    sv = MPF(sm, se)
    if dmask is not None:
        sv = masked(sv, dmask)
    d = add(MPF(dm, de), sv)
    return _with_diag(A, d.m, d.e)


def set_diag_where(A, val, dmask):
    """diagonal entries set to the MPF scalar val where dmask (nb, n) is True"""
    i = _diag_idx(A)
    dm = torch.where(dmask[None], val.m.reshape(-1, 1, 1), A.m[..., i, i])
    de = torch.where(dmask, val.e.reshape(1, 1), A.e[..., i, i])
    return _with_diag(A, dm, de)


def col_scale(V, v):
    """V (nb, h, K) with column k multiplied by v[:, k] (v: (nb, K, 1))"""
    nb, h, K = V.shape
    vm = v.m.reshape(v.L, nb, 1, K).expand(v.L, nb, h, K).contiguous()
    ve = v.e.reshape(nb, 1, K).expand(nb, h, K).contiguous()
    return mul(V, MPF(vm, ve))


def bexpand(v, nb):
    """(R, C) -> (nb, R, C) copies"""
    return MPF(v.m.unsqueeze(1).expand(v.L, nb, *v.shape).contiguous(),
               v.e.unsqueeze(0).expand(nb, *v.shape).contiguous())


def dup(a):
    """(nb, R, C) -> (2 nb, R, C): the same data for both parity batches"""
    return MPF(a.m.repeat(1, 2, 1, 1), a.e.repeat(2, 1, 1))


def fold(A, nb):
    """sum of the two parity halves (2 nb, ...) -> (nb, ...)"""
    return add(A[:nb], A[nb:])


def flat_rows(A):
    """(nb, R, C) -> (nb R, C)"""
    nb, R, C = A.shape
    return A.reshape(nb * R, C)


# ------------------------------------------------------------------ step length (sdpvibe/solver.py:996-1103)
EIG_TOL = float(os.environ.get("SDPB_GPU_EIG_TOL", "1e-10"))    # relative accuracy of the step lengths
_EPS = 2.0 ** -52
_DEFLATE = 2.0 ** -20          # refine_min_eig: eigenvalues above this * ||A||_F are deflated


def _eig_err(Mf):
    """per block bound on |computed - exact| for the float64 eigenvalues of Mf (nb, n, n): the rounding
    to float64 plus the eigensolver's backward error, (n + 2) eps ||Mf||_F (sdpvibe/solver.py:1001-1004)"""
    return (Mf.shape[-1] + 2) * _EPS * np.sqrt(np.einsum("bij,bij->b", Mf, Mf))


def step_from_eig(lam, gamma):
    """gamma * (-1 / lambda_min), capped at 1 (sdpvibe/solver.py:1096-1099)"""
    if lam is None or lam > -gamma:
        return mp.mpf(1)
    return -gamma / lam


def _resolved(lam, err, gamma):
    """every value in [lam - err, lam + err] gives the same step length to EIG_TOL"""
    return step_from_eig(lam - err, gamma) >= (1 - EIG_TOL) * step_from_eig(lam + err, gamma)


def _mpf_from_float(V, L):
    """float64 array -> MPF, exactly (sdpvibe/solver.py:1012-1018)"""
    return F.from_float(V, L)


EIG_DEVICE = os.environ.get("SDPV_EIG", "device") != "host"    # min_eig's float64 eigenvalues on the GPU
EIG_DEVICE_NMAX = 128


def _scaled(M):
    """(per block scale s, ok mask, M * 2^-s as an MPF): s is the largest entry top of each block (0 for
    all-zero blocks), so the float64 copy is O(1) and cannot overflow"""
    tp = F._top(M)
    s = tp.reshape(tp.shape[0], -1).amax(1)
    ok = s > EZ // 2
    s = torch.where(ok, s, torch.zeros_like(s))
    return s, ok, M.shift(-s[:, None, None])


def _scaled_float(M):
    """(s, ok, symmetric float64 copy of M * 2^-s on the host)"""
    s, ok, Ms = _scaled(M)
    Mf = Ms.to_float()
    return s, ok, (Mf + np.swapaxes(Mf, 1, 2)) / 2


def _device_float(A):
    """float64 values of an MPF on the device (the formula of MPF.to_float)"""
    L = A.L
    top = A.m[-1].double() * 2.0 ** 32 + (A.m[-2].double() % 2.0 ** 32) if L > 1 else A.m[-1].double()
    sc = (A.e + 32 * (L - 2)).clamp(-1100, 1100).double()
    return torch.where(A.e == EZ, torch.zeros_like(top), top * torch.pow(2.0, sc))


def _eig_min_device(Ms):
    """(lambda_min (nb,), error bound (nb,)) of the symmetric float64 copies of the blocks of Ms, by the
    batched Jacobi kernel (sdpv_eig_sym_f64), returned to the host"""
    w, err = _eig_device(Ms)
    return w.cpu().numpy(), err.cpu().numpy()


def _eig_device(Ms):
    """as _eig_min_device, the results left on the device"""
    from . import _lib
    Af = _device_float(Ms)
    Af = ((Af + Af.transpose(1, 2)) / 2).contiguous()
    nb, n, _ = Af.shape
    w = torch.empty((nb, n), dtype=torch.float64, device=Af.device)
    err = torch.empty((nb,), dtype=torch.float64, device=Af.device)
    _lib.call("sdpv_eig_sym_f64", _lib.ptr(Af), nb, n, _lib.ptr(w), _lib.ptr(err), None, _lib.stream())
    return w[:, 0], err


def refine_min_eig(A, gamma, levels=64):
    """lambda_min of each symmetric MPF block A[b] (nb, n, n) to the accuracy the step length needs, for
    blocks whose float64 copy cannot resolve it (sdpvibe/solver.py:1021-1061).

    Each level diagonalises the float64 copy (V its eigenvectors), forms W = V^T A V in multiprecision
    (congruent to A: same inertia, eigenvalues within a factor 1 + O(n eps)), deflates the eigenvalues
    above _DEFLATE ||A||_F (rows b) and continues on the Schur complement W_ss - W_sb W_bb^-1 W_bs, kept
    at full size with zero rows and columns at the deflated positions (its extra zero eigenvalues do not
    change the step length).  Returns (values, number of blocks left unresolved, whose value is the lower
    end of their error interval: a shorter, safe step)."""
    L = A.L
    out, idx, unresolved = [None] * A.shape[0], list(range(A.shape[0])), set()
    one = F.scalar(1, L)
    for _ in range(levels):
        s, ok, Af = _scaled_float(A)
        zero = (~ok).tolist()
        w, V = np.linalg.eigh(Af)
        err = _eig_err(Af)
        big = w > _DEFLATE * np.sqrt(np.einsum("bij,bij->b", Af, Af))[:, None]
        keep = []
        for j, q in enumerate(idx):
            sc = mp.mpf(2) ** int(s[j])
            lam, e = mp.mpf(float(w[j, 0])) * sc, mp.mpf(float(err[j])) * sc
            unresolved.discard(q)
            if zero[j]:
                out[q] = mp.mpf(0)
            elif _resolved(lam, e, gamma):
                out[q] = lam
            else:
                out[q] = lam - e
                unresolved.add(q)
                if big[j].any() and not big[j].all():
                    keep.append(j)
        if not keep:
            break
        A, idx = A[torch.tensor(keep, device=dev)], [idx[j] for j in keep]
        Pb = torch.from_numpy(big[keep]).to(dev)
        Ps = ~Pb
        Vm = _mpf_from_float(V[keep], L)
        W = symmetrize(gemm(Vm, gemm(A, Vm), transA=True))
        Wbb = add_diag(masked(W, Pb[:, :, None] & Pb[:, None, :]), one, Ps)
        Y = Chol(Wbb).solve_lower(masked(W, Pb[:, :, None] & Ps[:, None, :]))
        A = symmetrize(add(masked(W, Ps[:, :, None] & Ps[:, None, :]), gemm(Y, Y, transA=True), -1))
    return out, len(unresolved)


def min_eig_start(ch, D):
    """the device part of min_eig for one factor: M = L^-1 dM L^-T, its scaling and (EIG_DEVICE) the
    eigenvalue kernel, with nothing read back; min_eig_finish takes the results"""
    T = ch.solve_lower(D)
    M = ch.solve_lower(T.T)                                         # L^-1 dM L^-T (dM symmetric)
    if EIG_DEVICE and M.shape[-1] <= EIG_DEVICE_NMAX:
        s, ok, Ms = _scaled(M)
        return M, s, ok, _eig_device(Ms)
    s, ok, Mf = _scaled_float(M)
    return M, s, ok, (np.linalg.eigvalsh(Mf)[:, 0], _eig_err(Mf))


def min_eig(chols, dMs, lam=None, gamma=None, stats=None):
    """min over blocks of lambda_min(L^-1 dM L^-T), combined with lam (sdpvibe/solver.py:1064-1093).
    The eigenvalues come from a float64 copy of each block: on the GPU by the batched Jacobi kernel with
    its own error bound (EIG_DEVICE, blocks up to 128), else LAPACK on the host with the reference's bound
    (n + 2) eps ||M||_F, which reproduces the reference's steps bit for bit.  With gamma
    (stepLengthReduction) the blocks whose error bound could move the step length by more than EIG_TOL
    are recomputed in multiprecision (refine_min_eig), counted in stats."""
    return min_eig_finish([min_eig_start(ch, D) for ch, D in zip(chols, dMs)], lam, gamma, stats)


def min_eig_finish(pending, lam=None, gamma=None, stats=None):
    """the host part of min_eig over the results of min_eig_start, in order"""
    for M, s, ok, (ev, err) in pending:
        if torch.is_tensor(ev):
            ev, err = ev.cpu().numpy(), err.cpu().numpy()
        s_h, ok_h = s.tolist(), ok.tolist()                        # one transfer each
        flag = []
        for q in (q for q in range(len(ok_h)) if ok_h[q]):
            sc = mp.mpf(2) ** int(s_h[q])
            lq = mp.mpf(float(ev[q])) * sc
            if gamma is not None and not _resolved(lq, mp.mpf(float(err[q])) * sc, gamma):
                flag.append(q)
                continue
            lam = lq if lam is None else min(lam, lq)
        if flag:
            vals, nu = refine_min_eig(M[torch.tensor(flag, device=dev)], gamma)
            for v in vals:
                lam = v if lam is None else min(lam, v)
            if stats is not None:
                stats["eig_refined"] = stats.get("eig_refined", 0) + len(flag)
                stats["eig_unresolved"] = stats.get("eig_unresolved", 0) + nu
    return lam


def step_length(chols, dMs, gamma):
    return step_from_eig(min_eig(chols, dMs), gamma)


# ------------------------------------------------------------------ SDP input (sdpvibe/solver.py:399-521)
class Group:
    """one chunk of blocks of equal dim, zero-padded to common K (points) and h (bilinear basis size)"""


def _chunks_by_dim(blocks):
    """single-GPU resident plan: one chunk per dim, blocks ordered by (K, max(he, ho)) inside it
    (sdpvibe/solver.py:277-279, the unchunked branch of Layout)"""
    bydim = {}
    for j, b in enumerate(blocks):
        bydim.setdefault(b["dim"], []).append(j)
    for d in bydim:
        bydim[d].sort(key=lambda j: (blocks[j]["K"], max(blocks[j]["he"], blocks[j]["ho"])))
    return [bydim[d] for d in sorted(bydim)]


def _host_mpf(H, L):
    """host data of one MPF array -> device MPF.  H is (limbs (L, *shape) int32, exps (*shape) int64)
    of normalised entries, a float64 numpy array (converted exactly) or already an MPF."""
    if isinstance(H, MPF):
        return H
    if isinstance(H, np.ndarray):
        return F.from_float(H, L)
    m, e = H
    return MPF(torch.from_numpy(np.ascontiguousarray(m)).to(dev), torch.from_numpy(np.ascontiguousarray(e)).to(dev))


def _shape(H):
    if isinstance(H, (MPF, np.ndarray)):
        return H.shape
    return H[1].shape


def _rand_host_mpf(rng, shape, L, spread=4):
    """random normalised MPF host data: |mantissa| of exactly 32L-2 bits, random sign, |value| in
    [2^u, 2^(u+1)) with u ~ U[-spread, spread] (numpy generator)"""
    n = int(np.prod(shape))
    mag = rng.integers(0, 1 << 32, size=(L, n), dtype=np.uint64).astype(np.uint32)
    mag[L - 1] = (mag[L - 1] & np.uint32((1 << 29) - 1)) | np.uint32(1 << 29)
    neg = rng.random(n) < 0.5
    m = mag.copy()
    m[:, neg] = ~m[:, neg]
    carry = neg.copy()
    for k in range(L):                                     # two's complement: +1 with carry
        v = m[k].astype(np.uint64) + carry
        m[k] = v.astype(np.uint32)
        carry = carry & (v > 0xffffffff)
    e = rng.integers(-spread, spread + 1, size=n).astype(np.int64) - (32 * L - 3)
    return m.view(np.int32).reshape(L, *shape), e.reshape(shape)


class SDP:
    """SDP in SDPB's block form, batched by dim (one chunk per dim, every array resident on the GPU).

    Block j: dim, K points, even / odd bilinear bases V_e (he, K), V_o (ho, K), c_j (K npair, 1),
    B_j (K npair, N) with npair = dim (dim + 1) / 2; then b (N, 1) and const.  Arrays are MPF, host MPF
    data (limbs, exps) or float64 numpy arrays (exact)."""

    def __init__(self, blocks, b, const, L):
        """blocks: [dict(dim, K, Ve, Vo, c, B)] (Ve / Vo None for an empty basis)"""
        mp.mp.prec = F.NBITS(L) + 64
        shapes = []
        for bl in blocks:
            he = 0 if bl.get("Ve") is None else _shape(bl["Ve"])[0]
            ho = 0 if bl.get("Vo") is None else _shape(bl["Vo"])[0]
            shapes.append(dict(dim=bl["dim"], K=bl["K"], he=he, ho=ho))
        self._build(shapes, lambda j: (blocks[j].get("Ve"), blocks[j].get("Vo"), blocks[j]["c"], blocks[j]["B"]),
                    _host_mpf(b, L), mp.mpf(const), L)

    @classmethod
    def synthetic(cls, blocks, N, L, seed=0):
        """random SDP with the given block shapes [dict(dim, K, he, ho)] (benchmarks)"""
        self = cls.__new__(cls)
        mp.mp.prec = F.NBITS(L) + 64
        rng = np.random.default_rng(seed)
        b = _rand_host_mpf(rng, (N, 1), L)
        data = []
        for bl in blocks:
            npair = bl["dim"] * (bl["dim"] + 1) // 2
            data.append((_rand_host_mpf(rng, (bl["he"], bl["K"]), L) if bl["he"] else None,
                         _rand_host_mpf(rng, (bl["ho"], bl["K"]), L) if bl["ho"] else None,
                         _rand_host_mpf(rng, (bl["K"] * npair, 1), L), _rand_host_mpf(rng, (bl["K"] * npair, N), L)))
        self._build(blocks, lambda j: data[j], _host_mpf(b, L), mp.mpf(0), L)
        return self

    def _build(self, blocks, data, b, const, L):
        self.const, self.b, self.N, self.L = const, b, b.shape[0], L
        N = self.N
        self.groups = []
        for c in _chunks_by_dim(blocks):
            g = Group()
            nb, dim = len(c), blocks[c[0]]["dim"]
            K = max(blocks[j]["K"] for j in c)
            h = max(max(blocks[j]["he"], blocks[j]["ho"]) for j in c)
            npair = dim * (dim + 1) // 2
            P = K * npair
            g.idx, g.nb, g.dim, g.K, g.h, g.nbp, g.P = list(c), nb, dim, K, [h], 2 * nb, P
            g.psd_rows = sum(blocks[j]["dim"] * (blocks[j]["he"] + blocks[j]["ho"]) for j in c)
            V = F.zeros((2 * nb, h, K), L)
            xm = torch.zeros((2 * nb, dim * h), dtype=torch.bool, device=dev)
            g.c = F.zeros((nb, P, 1), L)
            B = F.zeros((nb, P, N), L)
            g.xmask = torch.zeros((nb, P), dtype=torch.bool, device=dev)
            for q, j in enumerate(c):
                Kj = blocks[j]["K"]
                Ve, Vo, cj, Bj = data(j)
                for par, v in enumerate((Ve, Vo)):
                    z = par * nb + q
                    hj = 0
                    if v is not None:
                        v = _host_mpf(v, L)
                        hj = v.shape[0]
                        V.m[:, z, :hj, :Kj] = v.m
                        V.e[z, :hj, :Kj] = v.e
                    for cc in range(dim):
                        xm[z, cc * h:cc * h + hj] = True
                cj, Bj = _host_mpf(cj, L), _host_mpf(Bj, L)
                for s in range(npair):                      # pair segment s: Kj points -> K slots
                    rows = slice(s * Kj, (s + 1) * Kj)
                    g.c.m[:, q, s * K:s * K + Kj] = cj.m[:, rows]
                    g.c.e[q, s * K:s * K + Kj] = cj.e[rows]
                    B.m[:, q, s * K:s * K + Kj] = Bj.m[:, rows]
                    B.e[q, s * K:s * K + Kj] = Bj.e[rows]
                    g.xmask[q, s * K:s * K + Kj] = True
            Vx = F.zeros((2 * nb, dim * h, dim * K), L)
            for cc in range(dim):
                put(Vx, cc * h, cc * K, V)
            g.Xmask = [xm]
            g.B = B
            g.V = dict(V=[V], Vx=[Vx])
            assert g.psd_rows == int(xm.sum())
            self.groups.append(g)
        self.total_psd_rows = sum(g.psd_rows for g in self.groups)
        self.nblocks = len(blocks)


# ------------------------------------------------------------------ solver (sdpvibe/solver.py:524-982)
DEFAULTS = dict(maxIterations=500, findPrimalFeasible=False, findDualFeasible=False,
                detectPrimalFeasibleJump=False, detectDualFeasibleJump=False,
                dualityGapThreshold="1e-30", primalErrorThreshold="1e-30", dualErrorThreshold="1e-30",
                initialMatrixScalePrimal="1e20", initialMatrixScaleDual="1e20",
                feasibleCenteringParameter="0.1", infeasibleCenteringParameter="0.3",
                stepLengthReduction="0.7", maxComplementarity="1e100", minPrimalStep="0", minDualStep="0")


def fmt_big(v, digits):
    """a number printed the way SDPB prints a BigFloat: C++ defaultfloat (%g style) with `digits`
    significant digits and an exponent of at least two digits with its sign (sdpvibe/solver.py:533-546)"""
    v = mp.mpf(v)
    if v == 0:
        return "0"
    txt = mp.nstr(v, digits, min_fixed=-5, max_fixed=digits, strip_zeros=True)
    mant, _, ex = txt.partition("e")
    if mant.endswith(".0"):
        mant = mant[:-2]
    if not ex:
        return mant
    sign = "-" if ex.startswith("-") else "+"
    ex = ex.lstrip("+-").lstrip("0") or "0"
    return f"{mant}e{sign}{ex.zfill(2)}"


def chol_log2_cond_parts(ch):
    """(max, min) over the diagonal of L (log2) of a factorisation (sdpvibe/solver.py:548-555)"""
    L = ch.L
    d = ch.diag_limbs()
    top = d[-1].double() * 2.0 ** 32 + (d[-2].double() % 2.0 ** 32) if L > 1 else d[-1].double()
    lg = torch.log2(torch.clamp(top, min=1e-300)) + (ch.efx + 32 * (L - 2)) + ch.k.double()
    return float(lg.max()), float(lg.min())


def chol_log2_cond(ch, mask=None):
    """per block log2 of SDPB's Cholesky condition estimate (max / min diagonal of L)^2, over the rows
    where mask (nb, n) is True (sdpvibe/solver.py:563-576)"""
    L = ch.L
    d = ch.diag_limbs()
    top = d[-1].double() * 2.0 ** 32 + (d[-2].double() % 2.0 ** 32) if L > 1 else d[-1].double()
    lg = torch.log2(torch.clamp(top, min=1e-300)) + (ch.efx + 32 * (L - 2)) + ch.k.double()
    if mask is None:
        mask = torch.ones_like(lg, dtype=torch.bool)
    hi = torch.where(mask, lg, torch.full_like(lg, -1e300)).amax(1)
    lo = torch.where(mask, lg, torch.full_like(lg, 1e300)).amin(1)
    return torch.where(mask.any(1), 2 * (hi - lo), torch.zeros_like(hi))


class PhaseTimer:
    """per-phase device time of Solver.run: CUDA events on the current stream, read after the run"""

    def __init__(self, on):
        self.on, self.marks = on, []

    def __call__(self, name):
        if not self.on:
            return
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        self.marks.append((name, ev))

    def totals(self):
        if not self.on or len(self.marks) < 2:
            return {}
        torch.cuda.synchronize()
        out = {}
        for (name, a), (_, b) in zip(self.marks, self.marks[1:]):
            out[name] = out.get(name, 0.0) + a.elapsed_time(b) * 1e-3
        return out


CONCURRENT = os.environ.get("SDPV_CONCURRENT", "1") != "0"


class _ChunkStreams:
    """Streams for independent per-chunk work.  Tensors made on a chunk stream and used afterwards on the
    main stream are safe to free there: a chunk stream only runs new work after waiting for the main stream
    at the next entry, so a freed block is never reused while the main stream still reads it."""

    def __init__(self, solver, n):
        self.solver, self.n = solver, n

    def __enter__(self):
        self.main = torch.cuda.current_stream()
        if not CONCURRENT:
            return lambda i: _NullCtx()
        pool = getattr(self.solver, "_streams", None)
        if pool is None or len(pool) < self.n:
            pool = self.solver._streams = [torch.cuda.Stream() for _ in range(self.n)]
        start = torch.cuda.Event()
        start.record(self.main)
        for st in pool[:self.n]:
            st.wait_event(start)
        self.pool = pool
        return lambda i: torch.cuda.stream(pool[i])

    def __exit__(self, *exc):
        if CONCURRENT:
            for st in self.pool[:self.n]:
                self.main.wait_stream(st)
        return False


class _NullCtx:
    def __enter__(self):
        return None

    def __exit__(self, *exc):
        return False


class Solver:
    """SDPB's Mehrotra predictor-corrector iteration (sdpvibe/solver.py:579-982) on one GPU with every
    chunk resident.  Per chunk the iteration keeps x, X, Y, their Cholesky factors, the residues, the
    pairings, the Schur complement factor and P = L_S^-1 B; y, b and Q are global."""

    def __init__(self, sdp, L, precision=None, timing=False, **params):
        self.sdp, self.L = sdp, L
        mp.mp.prec = F.NBITS(L) + 64
        self.precision = precision or (32 * (L - 1) - 2)
        self.digits = int(mp.ceil(self.precision * mp.log10(2))) + 1      # SDPB's stream precision
        p = dict(DEFAULTS)
        p.update(params)
        self.p = {k: (mp.mpf(v) if isinstance(v, str) else v) for k, v in p.items()}
        self.S = lambda v: F.scalar(v, L)
        self.st = []
        for g in sdp.groups:
            I = bexpand(F.eye(g.dim * g.h[0], L, 1), g.nbp)
            X = [set_diag_where(I, self.S(self.p["initialMatrixScalePrimal"]), g.Xmask[0])]
            Y = [set_diag_where(I, self.S(self.p["initialMatrixScaleDual"]), g.Xmask[0])]
            self.st.append(dict(xs=dict(x=F.zeros((g.nb, g.P, 1), L), X=X, Y=Y)))
        self.y = F.zeros((sdp.N, 1), L)
        self.timer = PhaseTimer(timing)
        self.eig_refined = self.eig_unresolved = 0

    # -- chunk concurrency
    def _chunk_streams(self):
        """context manager: inside it, `on(i)` runs chunk i's work on stream i (after everything issued before
        on the current stream); on exit the current stream waits for all chunk streams.  SDPV_CONCURRENT=0
        keeps every chunk on the current stream."""
        return _ChunkStreams(self, len(self.sdp.groups))

    # -- per-chunk pieces (sdpvibe/solver.py:622-665)
    @staticmethod
    def segments(g):
        return [(c, r, (c * (c + 1) // 2 + r) * g.K) for c in range(g.dim) for r in range(c + 1)]

    def cmws(self, g, Vs, a):
        """sum_p a_p A_p per parity batch (constraint_matrix_weighted_sum)"""
        a2 = dup(a)
        h = g.h[0]
        R = F.zeros((g.nbp, g.dim * h, g.dim * h), self.L)
        V = Vs["V"][0]
        for c, r, off in self.segments(g):
            s = gemm(V, col_scale(V, sub(a2, off, off + g.K, 0, 1)), transB=True)
            if r != c:
                s = s.shift(-1)
            put(R, r * h, c * h, s)
            if r != c:
                put(R, c * h, r * h, s.T)
        return [R]

    def pairings(self, g, Vs, cholX, Y):
        Vx = Vs["Vx"][0]
        T = cholX[0].solve_lower(Vx)
        AXI = copy_lower_to_upper(gemm(T, T, transA=True))
        AY = copy_lower_to_upper(gemm(Vx, gemm(Y[0], Vx), transA=True))
        return [AXI], [AY]

    def schur(self, g, AXI, AY):
        """S_pq = Tr(A_p X^-1 A_q Y) of the chunk from its pairings, in one launch (sdpv_schur_assemble:
        the operations of schur_composed, fused, bit for bit)"""
        from . import _lib
        A, Yp = AXI[0], AY[0]
        L, nb, P = self.L, g.nb, g.P
        S = MPF(torch.empty((L, nb, P, P), dtype=torch.int32, device=dev),
                torch.empty((nb, P, P), dtype=torch.int64, device=dev))
        one, one_e = self._one()
        _lib.call("sdpv_schur_assemble", L, nb, P, g.K, g.dim, _lib.ptr(A.m.contiguous()), _lib.ptr(A.e.contiguous()),
                  _lib.ptr(Yp.m.contiguous()), _lib.ptr(Yp.e.contiguous()), _lib.ptr(g.xmask.contiguous()),
                  _lib.ptr(one.m), one_e, _lib.ptr(S.m), _lib.ptr(S.e), _lib.stream())
        return S

    def _one(self):
        """the MPF scalar 1 and its exponent (made once)"""
        if getattr(self, "_one_c", None) is None:
            o = self.S(1)
            self._one_c = (o, int(o.e[0]))
        return self._one_c

    def schur_composed(self, g, AXI, AY):
        """the reference's composition of the Schur complement out of elementwise MPF operations"""
        K = g.K
        if g.dim == 1:
            S = fold(mul(AXI[0], AY[0]), g.nb)
        else:
            def sb(M, c, r):                                  # A_X_inv[c][r]
                return sub(M, c * K, (c + 1) * K, r * K, (r + 1) * K)

            def sy(M, c, r):                                  # A_Y[c][r]
                return sub(M, r * K, (r + 1) * K, c * K, (c + 1) * K)
            S = F.zeros((g.nb, g.P, g.P), self.L)
            A, Yp = AXI[0], AY[0]
            for c0, r0, ro in self.segments(g):
                for c1, r1, co in self.segments(g):
                    if co > ro:
                        break
                    el = None
                    for t in (mul(sb(A, c0, r1), sy(Yp, c1, r0)), mul(sb(A, r0, r1), sy(Yp, c1, c0)),
                              mul(sb(A, c0, c1), sy(Yp, r1, r0)), mul(sb(A, r0, c1), sy(Yp, r1, c0))):
                        el = t if el is None else add(el, t)
                    put(S, ro, co, fold(el, g.nb).shift(-2))
        S = copy_lower_to_upper(S)
        return set_diag_where(S, self.S(1), ~g.xmask)

    def seg_diag(self, g, Ms, hs):
        v = F.zeros((g.nb, g.P, 1), self.L)
        for c, r, off in self.segments(g):
            d = diag_of(sub(Ms[0], r * hs[0], (r + 1) * hs[0], c * hs[0], (c + 1) * hs[0]))
            put(v, off, 0, fold(d, g.nb))
        return v

    # -- the iteration (sdpvibe/solver.py:680-982)
    def run(self, max_iter=None, log=None, verbose=False, on_iteration=None, record=None):
        """iterate until a termination criterion holds; returns the result dict.  record(it, solver,
        info) is called after each iteration's update of y (tests read the iterates there)."""
        p, sdp, S = self.p, self.sdp, self.S
        G = sdp.groups
        tm = self.timer
        alphaP = alphaD = mp.mpf(0)
        t0 = time.time()
        it = 0
        update = None
        pobj = dobj = gap = primal_err = dual_err = mp.mpf(0)

        def mk2(g):
            return g.Xmask[0][:, :, None] & g.Xmask[0][:, None, :]

        def result(reason, iterations):
            return dict(terminateReason=reason, primalObjective=pobj, dualObjective=dobj, dualityGap=gap,
                        primalError=primal_err, dualError=dual_err, iterations=iterations, time=time.time() - t0)
        while True:
            it += 1
            ti = time.time()
            cond = [mp.mpf(0), ""]

            def upd_cond(lg2, name):
                if lg2 > float(mp.log(cond[0], 2) if cond[0] > 0 else -1):
                    cond[0] = mp.mpf(2) ** mp.mpf(lg2)
                    cond[1] = name
            # condition estimates and positivity flags stay on the device until the end of the iteration
            # (read there in one transfer, applied in this order): no host synchronisation per factorisation
            conds, bads = [], []

            def chol(A):
                ch = Chol(A, defer_check=True)
                bads.append(ch.bad)
                return ch

            def resolve(extra=()):
                """read the pending flags, estimates and `extra` tensors in one transfer; apply them in order"""
                parts = [b.reshape(1).to(torch.float64) for b in bads] + [c.reshape(-1).to(torch.float64)
                                                                          for c, _ in conds]
                parts += [x.reshape(-1).to(torch.float64) for x in extra]
                vals = torch.cat(parts).cpu().tolist() if parts else []
                if any(vals[:len(bads)]):
                    raise ValueError("matrix is not positive definite (diagonal)")
                o = len(bads)
                for c, name in conds:
                    lg = vals[o:o + c.numel()]
                    o += c.numel()
                    z = max(range(len(lg)), key=lambda i: lg[i])
                    upd_cond(lg[z], name(z))
                out = []
                for x in extra:
                    out.append(vals[o:o + x.numel()])
                    o += x.numel()
                bads.clear()
                conds.clear()
                return out
            tm("residues")
            dobj = sdp.const + dot(sdp.b, self.y)
            psum = musum = mp.mpf(0)
            dual_err = primal_err_P = mp.mpf(0)
            pvec = sdp.b
            pgs = []
            with self._chunk_streams() as on:                    # chunks concurrent, as in the Schur phase
                for gi, g in enumerate(G):
                    with on(gi):
                        o = self.st[gi]
                        xs = o["xs"]
                        if update:
                            aP, aD = update
                            dc = o.pop("dc")
                            xs = dict(x=add(xs["x"], mul(dc["dx"], aP)),
                                      X=[add(X, mul(d, aP)) for X, d in zip(xs["X"], dc["dX"])],
                                      Y=[add(Y, mul(d, aD)) for Y, d in zip(xs["Y"], dc["dY"])])
                        cX = [chol(X) for X in xs["X"]]
                        cY = [chol(Y) for Y in xs["Y"]]
                        for tag, chs in (("X", cX), ("Y", cY)):
                            conds.append((chol_log2_cond(chs[0], g.Xmask[0]),
                                          lambda z, tag=tag, g=g: f"{tag}_cholesky.block_{g.idx[z % g.nb]}_{z // g.nb}"))
                        Vs = g.V
                        a, y_ = self.pairings(g, Vs, cX, xs["Y"])
                        d = -self.seg_diag(g, y_, [g.K])
                        o["AXI"], o["AY"] = a, y_
                        B = g.B
                        By = gemm(B, bexpand(self.y, g.nb))
                        d = add(d, By, -1)
                        dres = add(d, g.c)
                        pgs.append(gemm(flat_rows(B), flat_rows(xs["x"]), transA=True))
                        Ax = self.cmws(g, Vs, xs["x"])
                        Pres = [masked(add(Ax[0], xs["X"][0], -1), mk2(g))]
                        mXY = [masked(-gemm(X, Y), mk2(g)) for X, Y in zip(xs["X"], xs["Y"])]
                        o["xs"], o["ch"] = xs, dict(X=cX, Y=cY)
                        o["res"] = dict(dres=dres, Pres=Pres, mXY=mXY)
            for gi, g in enumerate(G):                           # sums and host scalars in chunk order
                o = self.st[gi]
                res = o["res"]
                psum += dot(g.c, o["xs"]["x"])
                pvec = add(pvec, pgs[gi], -1)
                dual_err = max(dual_err, max_abs(res["dres"]))
                primal_err_P = max([primal_err_P] + [max_abs(P) for P in res["Pres"]])
                for M in res["mXY"]:
                    musum += total(diag_of(M))
            del pgs
            resolve()
            update = None
            pobj = sdp.const + psum
            gap = abs(pobj - dobj) / max(abs(pobj) + abs(dobj), mp.mpf(1))
            primal_err_p = max_abs(pvec)
            primal_err = max(primal_err_P, primal_err_p)
            dual_feas = dual_err < p["dualErrorThreshold"]
            primal_feas = primal_err < p["primalErrorThreshold"]
            pd_feas = dual_feas and primal_feas
            reason = None
            if pd_feas and gap < p["dualityGapThreshold"]:
                reason = "found primal-dual optimal solution"
            elif dual_feas and p["findDualFeasible"]:
                reason = "found dual feasible solution"
            elif primal_feas and p["findPrimalFeasible"]:
                reason = "found primal feasible solution"
            elif alphaD == 1 and p["detectDualFeasibleJump"]:
                reason = "dual feasible jump detected"
            elif alphaP == 1 and p["detectPrimalFeasibleJump"]:
                reason = "primal feasible jump detected"
            elif it > (max_iter or p["maxIterations"]):
                reason = "maxIterations exceeded"
            elif it > 1 and alphaP < p["minPrimalStep"]:
                reason = "primal step too small"
            elif it > 1 and alphaD < p["minDualStep"]:
                reason = "dual step too small"
            if reason:
                self.result = result(reason, it - 1)
                break
            mu = -musum / sdp.total_psd_rows
            if mu > p["maxComplementarity"]:
                self.result = result("maxComplementarity exceeded", it - 1)
                break
            # Schur complement, its Cholesky factor, Q = sum_g P_g^T P_g (all chunks resident: P kept).  The
            # chunks are independent until the sum: each runs on its own stream, the sum in chunk order.
            tm("schur: S, chol(S), P = L^-1 B, P^T P")
            qgs = []
            with self._chunk_streams() as on:
                for gi, g in enumerate(G):
                    with on(gi):
                        o = self.st[gi]
                        Sg = self.schur(g, o.pop("AXI"), o.pop("AY"))
                        cs = chol(Sg)
                        conds.append((chol_log2_cond(cs, g.xmask),
                                      lambda q, g=g: f"schur_complement_cholesky.block_{g.idx[q]}"))
                        P = cs.solve_lower(g.B)
                        qgs.append(gemm(flat_rows(P), flat_rows(P), transA=True))
                        o["cholS"], o["Pm"] = cs, P
            Q = qgs[0]
            for qg in qgs[1:]:
                Q = add(Q, qg)
            del qgs
            # chol(Q) on a stream of its own: the first half of the predictor does not need it, so the two
            # overlap; _direction waits for it before its solve with Q
            tm("chol(Q) + direction (predictor) 1")
            main = torch.cuda.current_stream()
            qstream = self._q_stream() if CONCURRENT else main
            qstream.wait_stream(main)
            qb = self._q_block(sdp.N)
            with torch.cuda.stream(qstream):
                if qb:                                         # tiled: ~Q/2 instead of ~9 Q at the peak
                    from .blockchol import BlockChol
                    cholQ, q_lg = BlockChol([Q], qb), None
                    q_cond_lg = cholQ.log2_cond()
                else:
                    cholQ = chol(copy_lower_to_upper(Q))
                    q_lg = chol_log2_cond(cholQ)
                q_ready = torch.cuda.Event()
                q_ready.record(qstream)
            for t in (Q.m, Q.e):
                t.record_stream(qstream)                       # freed below while the Q stream may read it
            del Q
            dy, acc = self._direction(mu, pvec, cholQ, corr=False,
                                      beta=mp.mpf(0) if pd_feas else p["infeasibleCenteringParameter"],
                                      q_ready=q_ready)
            R_err = acc["Rerr"]
            r = acc["fr"] / (mu * sdp.total_psd_rows)
            beta = r * r if r < 1 else r
            if pd_feas:
                beta_c = min(max(p["feasibleCenteringParameter"], beta), mp.mpf(1))
            else:
                beta_c = max(p["infeasibleCenteringParameter"], beta)
            dy, acc = self._direction(mu, pvec, cholQ, corr=True, beta=beta_c)
            if acc.get("eig_refined"):
                self.eig_refined += acc["eig_refined"]
                self.eig_unresolved += acc.get("eig_unresolved", 0)
            for o in self.st:
                o.pop("cholS", None)
                o.pop("Pm", None)
            del cholQ
            gm = p["stepLengthReduction"]
            alphaP = step_from_eig(acc["lamP"], gm)
            alphaD = step_from_eig(acc["lamD"], gm)
            if pd_feas:
                alphaP = alphaD = min(alphaP, alphaD)
            tm("update")
            aP, aD = S(alphaP), S(alphaD)
            update = (aP, aD)
            self.y = add(self.y, mul(dy, aD))
            if q_lg is None:
                resolve()
                Q_cond = mp.mpf(2) ** mp.mpf(q_cond_lg)
            else:
                Q_cond = mp.mpf(2) ** mp.mpf(resolve([q_lg])[0][0])
            row = dict(iteration=it, total_time=round(time.time() - t0, 3), iter_time=round(time.time() - ti, 3),
                       mu=mu, pobj=pobj, dobj=dobj, gap=gap, P_err=primal_err_P, p_err=primal_err_p, D_err=dual_err,
                       R_err=R_err, P_step=alphaP, D_step=alphaD, beta=beta_c, Q_cond=Q_cond,
                       max_block_cond=cond[0], block_name=cond[1])
            self.last_mu, self.last_steps = mu, (alphaP, alphaD, beta_c)
            if log is not None:
                log.append(row)
            if on_iteration is not None:
                on_iteration(row)
            if record is not None:
                record(it, self, dict(dy=dy, aP=aP, aD=aD, row=row))
            if verbose:
                f = lambda v: mp.nstr(v, 3)
                print(f"{it:4d} {time.time() - t0:7.2f} mu {f(mu)} P-obj {f(pobj)} D-obj {f(dobj)} gap {f(gap)} "
                      f"P-err {f(primal_err_P)} D-err {f(dual_err)} steps {f(alphaP)} {f(alphaD)} beta {f(beta_c)}",
                      flush=True)
        self._pending_update = update
        return self.result

    def _q_block(self, N):
        """tile size of the tiled Cholesky of Q, or 0 for the monolithic one (sdpvibe/solver.py:594-606):
        SDPB_GPU_QBLOCK=<tile> forces it; else 2048 when the monolithic factorisation (about 9 N^2 MPF
        entries) would take more than 35% of the GPU's memory and N > 2048"""
        forced = int(os.environ.get("SDPB_GPU_QBLOCK", 0))
        if forced:
            return forced if forced < N else 0
        E = 4 * self.L + 8
        budget = torch.cuda.get_device_properties(torch.cuda.current_device()).total_memory
        return 2048 if 9.0 * N * N * E > 0.35 * budget and N > 2048 else 0

    def _q_stream(self):
        if getattr(self, "_qs", None) is None:
            self._qs = torch.cuda.Stream()
        return self._qs

    def _direction(self, mu, pvec, cholQ, corr, beta, q_ready=None):
        """predictor (corr=False) or corrector search direction (sdpvibe/solver.py:870-933): dy, and per
        chunk dp (predictor) or dc (corrector) with the step-length eigenvalues"""
        p, S, G = self.p, self.S, self.sdp.groups
        tm = self.timer
        bm, muS = S(beta * mu), S(mu)

        def mk2(g):
            return g.Xmask[0][:, :, None] & g.Xmask[0][:, None, :]
        acc = dict(Rerr=mp.mpf(0), fr=mp.mpf(0), lamP=None, lamD=None)
        if corr:
            tm("direction (corrector) 1")
        tgs = []
        with self._chunk_streams() as on:                        # chunks concurrent; sums in chunk order below
            for gi, g in enumerate(G):
                with on(gi):
                    o = self.st[gi]
                    xs, res, cX = o["xs"], o["res"], o["ch"]["X"]
                    Rb = res["mXY"][0] if not corr else add(res["mXY"][0], gemm(o["dp"]["dX"][0], o["dp"]["dY"][0]), -1)
                    Rb = add_diag(Rb, bm, g.Xmask[0])
                    Z = symmetrize(cX[0].solve(add(gemm(res["Pres"][0], xs["Y"][0]), Rb, -1)))
                    Vx = g.V["Vx"][0]
                    VZV = gemm(Vx, gemm(Z, Vx), transA=True)
                    rhs = add(-res["dres"], self.seg_diag(g, [VZV], [g.K]), -1)
                    w = o["cholS"].solve_lower(rhs)
                    o["dir"] = dict(R=[Rb], W=w)
                    tgs.append(gemm(flat_rows(o["Pm"]), flat_rows(w), transA=True))
        dy = pvec
        for gi, g in enumerate(G):
            if not corr:
                acc["Rerr"] = max([acc["Rerr"]] + [max_abs(add_diag(M, muS, g.Xmask[0]))
                                                   for M in self.st[gi]["res"]["mXY"]])
            dy = add(dy, tgs[gi], -1)
        del tgs
        if q_ready is not None:
            torch.cuda.current_stream().wait_event(q_ready)
        dy = cholQ.solve(dy)
        tm("direction (corrector) 2 + step length" if corr else "direction (predictor) 2")
        with self._chunk_streams() as on:
            for gi, g in enumerate(G):
                with on(gi):
                    o = self.st[gi]
                    xs, res, cX, dr = o["xs"], o["res"], o["ch"]["X"], o.pop("dir")
                    Pdy = gemm(o["Pm"], bexpand(dy, g.nb))
                    dxg = o["cholS"].solve_upper(add(dr["W"], Pdy))
                    Ad = self.cmws(g, g.V, dxg)
                    dXg = [add(Ad[0], res["Pres"][0])]
                    dYg = [masked(-symmetrize(cX[0].solve(add(gemm(dXg[0], xs["Y"][0]), dr["R"][0], -1))), mk2(g))]
                    o["step"] = (dxg, dXg, dYg)
                    if corr:                                     # the device part of the step lengths too
                        o["eig"] = ([min_eig_start(c, D) for c, D in zip(o["ch"]["X"], dXg)],
                                    [min_eig_start(c, D) for c, D in zip(o["ch"]["Y"], dYg)])
        for gi, g in enumerate(G):                               # host scalars / step lengths in chunk order
            o = self.st[gi]
            xs = o["xs"]
            dxg, dXg, dYg = o.pop("step")
            if not corr:
                acc["fr"] += dot(masked(add(xs["X"][0], dXg[0]), mk2(g)), masked(add(xs["Y"][0], dYg[0]), mk2(g)))
                o["dp"] = dict(dX=dXg, dY=dYg)
            else:
                gm = p["stepLengthReduction"]
                st = {}
                pend_P, pend_D = o.pop("eig")
                lamP = min_eig_finish(pend_P, gamma=gm, stats=st)
                lamD = min_eig_finish(pend_D, gamma=gm, stats=st)
                for k, v in (("lamP", lamP), ("lamD", lamD)):
                    if v is not None:
                        acc[k] = v if acc[k] is None else min(acc[k], v)
                for k in ("eig_refined", "eig_unresolved"):
                    acc[k] = acc.get(k, 0) + st.get(k, 0)
                o.pop("dp", None)
                o["dc"] = dict(dx=dxg, dX=dXg, dY=dYg)
        return dy, acc
