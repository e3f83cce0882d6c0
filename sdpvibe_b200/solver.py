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


def _scaled_float(M):
    """(per block scale s, ok mask, symmetric float64 copy of M * 2^-s): s is the largest entry top of
    each block (0 for all-zero blocks), so the copy is O(1) and cannot overflow"""
    tp = F._top(M)
    s = tp.reshape(tp.shape[0], -1).amax(1)
    ok = s > EZ // 2
    s = torch.where(ok, s, torch.zeros_like(s))
    Mf = M.shift(-s[:, None, None]).to_float()
    return s, ok, (Mf + np.swapaxes(Mf, 1, 2)) / 2


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


def min_eig(chols, dMs, lam=None, gamma=None, stats=None):
    """min over blocks of lambda_min(L^-1 dM L^-T), combined with lam (sdpvibe/solver.py:1064-1093).
    The eigenvalues come from a float64 copy of each block (LAPACK on the host, as the reference);
    with gamma (stepLengthReduction) the blocks whose float64 error bound could move the step length by
    more than EIG_TOL are recomputed in multiprecision (refine_min_eig), counted in stats."""
    for ch, D in zip(chols, dMs):
        T = ch.solve_lower(D)
        M = ch.solve_lower(T.T)                                     # L^-1 dM L^-T (dM symmetric)
        s, ok, Mf = _scaled_float(M)
        ev = np.linalg.eigvalsh(Mf)[:, 0]
        err = _eig_err(Mf)
        flag = []
        for q in torch.nonzero(ok).reshape(-1).tolist():
            sc = mp.mpf(2) ** int(s[q])
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
