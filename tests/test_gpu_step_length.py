"""Step-length eigenvalues (solver.min_eig / refine_min_eig) against exact spectra, following the
reference's own known-answer construction (tests/test_step_length.py of the reference): with an integer
matrix V, X = V V^T and dM = V diag(lam) V^T, the eigenvalues of L^-1 dM L^-T (X = L L^T) are exactly
lam.  Spectra with large positive eigenvalues next to the smallest one defeat the float64 copy; the
checked path (gamma given) must still give the exact step length to EIG_TOL, with the reference's
number of refined blocks."""
from fractions import Fraction

import mpmath as mp
import numpy as np
import pytest
import torch

from oracle import mp as OM

pytestmark = pytest.mark.gpu

L = 40                              # 1278 bits: room for spectra spread over 2^700
GAMMA = mp.mpf("0.7")


def _mpf_exact(Q, K):
    from sdpvibe_b200 import mpf as F
    n = len(Q)
    ints = [int(v) for row in Q for v in row]
    return F.from_ints(ints, [-K if v else F.EZ for v in ints], L, (n, n))


def _case(n, lam, seed):
    rng = np.random.default_rng(seed)
    V = rng.integers(-3, 4, size=(n, n)).astype(object)
    while abs(np.linalg.det(V.astype(float))) < 1:
        V = rng.integers(-3, 4, size=(n, n)).astype(object)
    K = max(0, max(-int(np.floor(np.log2(abs(float(v))))) for v in lam if v) + 8)
    den = max(v.denominator for v in lam)
    K = max(K, den.bit_length() - 1)
    D = [int(v * (1 << K)) for v in lam]
    dM = (V * np.array(D, dtype=object)[None, :]).dot(V.T)
    return _mpf_exact(V.dot(V.T), 0), _mpf_exact(dM, K)


def _spectrum(n, big, small, lo, seed=0):
    rng = np.random.default_rng(100 + seed)
    lam = [Fraction(int(rng.integers(1, 8))) * (Fraction(2) ** k) for k in big]
    lam += [Fraction(int(rng.integers(1, 25)), 8) for _ in range(small)]
    lam += [lo]
    lam += [Fraction(int(rng.integers(1, 25)), 8) for _ in range(n - len(lam))]
    rng.shuffle(lam)
    return lam


def _run(blocks, expect_refined):
    from sdpvibe_b200.mpf import MPF, Chol
    from sdpvibe_b200.solver import min_eig, step_from_eig, EIG_TOL
    mp.mp.prec = 32 * L
    Xs, Ds = zip(*[_case(len(lam), lam, seed) for seed, lam in enumerate(blocks)])
    X = MPF(torch.stack([x.m for x in Xs], 1), torch.stack([x.e for x in Xs]))
    D = MPF(torch.stack([d.m for d in Ds], 1), torch.stack([d.e for d in Ds]))
    ch = Chol(X)
    exact = min(mp.mpf(v.numerator) / v.denominator for lam in blocks for v in lam)
    a_ex = step_from_eig(exact, GAMMA)
    st = {}
    got = min_eig([ch], [D], gamma=GAMMA, stats=st)
    err = abs(step_from_eig(got, GAMMA) / a_ex - 1)
    assert err <= EIG_TOL, (float(err), st)
    if expect_refined is not None:
        assert st.get("eig_refined", 0) == expect_refined, st
    return ch, D


CASES = {
    "ordinary": (lambda n: [_spectrum(n, [], n - 1, Fraction(-11, 8))], 0),
    "big_positive": (lambda n: [_spectrum(n, [100] * 5 + [60] * 3, 4, Fraction(-11, 8))], 1),
    "big_positive_step1": (lambda n: [_spectrum(n, [100] * 5, 4, Fraction(-1, 2))], None),
    "multiscale": (lambda n: [_spectrum(n, [700, 500, 300, 200, 120, 60, 30], 4, Fraction(-5, 2))], 1),
    "cluster": (lambda n: [_spectrum(n, [100] * 5, 0, Fraction(-11, 8))[:-3]
                           + [Fraction(-11, 8) - Fraction(1, 2 ** 40), Fraction(-11, 8) + Fraction(1, 2 ** 40),
                              Fraction(-11, 8) + Fraction(1, 2 ** 20)]], None),
    "big_negative": (lambda n: [_spectrum(n, [90] * 3, 4, -Fraction(2) ** 100)], 0),
    "three_of_four": (lambda n: [_spectrum(n, [100] * 5, 4, Fraction(-11, 8), 0),
                                 _spectrum(n, [700, 400, 100], 4, Fraction(-5, 2), 1),
                                 _spectrum(n, [], n - 1, Fraction(-3, 4), 2),
                                 _spectrum(n, [300] * 2, 4, Fraction(-1, 2), 3)], 3),
    "one_of_four": (lambda n: [_spectrum(n, [], n - 1, Fraction(-3, 4), s) for s in range(3)]
                    + [_spectrum(n, [200] * 4, 4, Fraction(-9, 4), 3)], 1),
}


@pytest.mark.parametrize("eig", ["host", "device"])
@pytest.mark.parametrize("n", [40, 144])
@pytest.mark.parametrize("name", sorted(CASES))
def test_min_eig_exact_spectra(name, n, eig, monkeypatch):
    """host: LAPACK with the reference's bound (the reference's refined-block counts); device: the Jacobi
    kernel with its own, wider bound (as many refinements or more, the same step accuracy).  n = 144 is
    beyond the device kernel's 128 and runs on the host in both modes."""
    from sdpvibe_b200 import solver
    monkeypatch.setattr(solver, "EIG_DEVICE", eig == "device")
    make, refined = CASES[name]
    _run(make(n), refined if eig == "host" or n > solver.EIG_DEVICE_NMAX else None)


@pytest.mark.parametrize("n", [1, 2, 3, 7, 21, 42, 63, 64, 100, 128])
def test_eig_sym_f64_kernel(n):
    """sdpv_eig_sym_f64 against LAPACK: every eigenvalue within the kernel's bound plus LAPACK's."""
    from sdpvibe_b200 import _lib
    rng = np.random.default_rng(n)
    nb = 5
    A = rng.standard_normal((nb, n, n)) * 2.0 ** rng.integers(-3, 4, size=(nb, 1, 1))
    A[1] = A[1] @ A[1].transpose() if n > 1 else A[1]                 # semidefinite, clustered small ones
    A = (A + np.swapaxes(A, 1, 2)) / 2
    A[2] = np.diag(np.arange(n, dtype=np.float64))                      # already diagonal
    Ad = torch.from_numpy(A).cuda()
    w = torch.empty((nb, n), dtype=torch.float64, device="cuda")
    err = torch.empty((nb,), dtype=torch.float64, device="cuda")
    sw = torch.empty((nb,), dtype=torch.int32, device="cuda")
    _lib.call("sdpv_eig_sym_f64", _lib.ptr(Ad), nb, n, _lib.ptr(w), _lib.ptr(err), _lib.ptr(sw), _lib.stream())
    ref = np.linalg.eigvalsh(A)
    lap = (n + 2) * 2.0 ** -52 * np.sqrt((A * A).sum(axis=(1, 2)))
    wd, ed = w.cpu().numpy(), err.cpu().numpy()
    assert (sw.cpu().numpy() < 40).all()
    assert np.all(np.abs(wd - ref) <= (ed + lap)[:, None])
    assert np.all(np.diff(wd, axis=1) >= 0)


def test_min_eig_matrix_matches_oracle():
    """M = L^-1 dM L^-T, the matrix whose float64 copy feeds the eigensolver, is bit-identical to the
    oracle's (so the float64 eigenvalues, and the step, are the reference's)."""
    from sdpvibe_b200.mpf import MPF, Chol
    blocks = [_spectrum(24, [100] * 3, 4, Fraction(-11, 8), s) for s in range(3)]
    Xs, Ds = zip(*[_case(len(lam), lam, seed) for seed, lam in enumerate(blocks)])
    X = MPF(torch.stack([x.m for x in Xs], 1), torch.stack([x.e for x in Xs]))
    D = MPF(torch.stack([d.m for d in Ds], 1), torch.stack([d.e for d in Ds]))
    ch = Chol(X)
    M = ch.solve_lower(ch.solve_lower(D).T)
    ref = OM.Chol(X.m.cpu().numpy(), X.e.cpu().numpy())
    tm, te = ref.solve_lower(D.m.cpu().numpy(), D.e.cpu().numpy())
    rm, re_ = ref.solve_lower(np.ascontiguousarray(np.swapaxes(tm, -1, -2)),
                              np.ascontiguousarray(np.swapaxes(te, -1, -2)))
    assert np.array_equal(M.m.cpu().numpy(), rm) and np.array_equal(M.e.cpu().numpy(), re_)


def test_step_from_eig_unconstrained():
    from sdpvibe_b200.solver import min_eig, step_from_eig
    from sdpvibe_b200.mpf import MPF, Chol
    mp.mp.prec = 32 * L
    X, D = _case(16, [Fraction(k + 1, 4) for k in range(16)], 5)          # dM positive definite
    ch = Chol(MPF(X.m[:, None], X.e[None]))
    lam = min_eig([ch], [MPF(D.m[:, None], D.e[None])], gamma=GAMMA)
    assert abs(lam - mp.mpf(1) / 4) < 1e-13                                # float64 eigenvalue
    assert step_from_eig(lam, GAMMA) == 1
