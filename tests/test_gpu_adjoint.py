"""Adjoints of the multiprecision building blocks (sdpvibe_b200.adjoint; no counterpart in the reference):
the GEMM vector-Jacobian products satisfy <G, dA B> = <gemm_vjp_A, dA> to working precision; the
Cholesky-solve adjoint matches central finite differences at working precision; the objective's linear
response equals its defining formula evaluated in mpmath."""
import mpmath as mp
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rand(rng, shape, L, lo=-3, hi=3):
    from sdpvibe_b200.solver import _rand_host_mpf, _host_mpf
    return _host_mpf(_rand_host_mpf(rng, shape, L, spread=hi), L)


def _inner(A, B):
    a, b = A.to_mp().reshape(-1), B.to_mp().reshape(-1)
    return mp.fsum(x * y for x, y in zip(a, b))


@pytest.mark.parametrize("tA,tB", [(False, False), (True, False), (False, True), (True, True)])
def test_gemm_vjp_identity(tA, tB):
    from sdpvibe_b200.adjoint import gemm_vjp
    from sdpvibe_b200.mpf import gemm
    L = 8
    mp.mp.prec = 32 * L + 64
    rng = np.random.default_rng(int(tA) * 2 + int(tB))
    M, K, N = 6, 9, 5
    A = _rand(rng, (K, M) if tA else (M, K), L)
    B = _rand(rng, (N, K) if tB else (K, N), L)
    G = _rand(rng, (M, N), L)
    dA = _rand(rng, A.shape, L)
    dB = _rand(rng, B.shape, L)
    gA, gB = gemm_vjp(A, B, G, tA, tB)
    assert gA.shape == A.shape and gB.shape == B.shape
    lhsA = _inner(G, gemm(dA, B, tA, tB))
    lhsB = _inner(G, gemm(A, dB, tA, tB))
    for lhs, rhs in ((lhsA, _inner(gA, dA)), (lhsB, _inner(gB, dB))):
        assert abs(lhs - rhs) <= mp.mpf(2) ** -(32 * L - 20) * (abs(lhs) + 1)


def test_chol_solve_vjp_central_differences():
    from sdpvibe_b200.adjoint import chol_solve_vjp
    from sdpvibe_b200.mpf import MPF, Chol, add, from_float, gemm
    L = 26
    mp.mp.prec = 32 * L + 64
    rng = np.random.default_rng(3)
    nb, n, m = 2, 40, 3
    G = rng.standard_normal((nb, n, n))
    S = from_float(G @ np.swapaxes(G, 1, 2) + n * np.eye(n), L)
    r = from_float(rng.standard_normal((nb, n, m)), L)
    gx = from_float(rng.standard_normal((nb, n, m)), L)
    D = rng.standard_normal((nb, n, n))
    dS = from_float((D + np.swapaxes(D, 1, 2)) / 2, L)
    dr = from_float(rng.standard_normal((nb, n, m)), L)
    ch = Chol(S)
    x = ch.solve(r)
    gr, gS = chol_solve_vjp(ch, x, gx)
    h = 2 ** -120

    def obj(Sm, rm):
        return _inner(gx, Chol(Sm).solve(rm))
    fd_S = (obj(add(S, dS.shift(-120)), r) - obj(add(S, dS.shift(-120), -1), r)) / (2 * mp.mpf(h))
    fd_r = (obj(S, add(r, dr.shift(-120))) - obj(S, add(r, dr.shift(-120), -1))) / (2 * mp.mpf(h))
    for fd, an in ((fd_S, _inner(gS, dS)), (fd_r, _inner(gr, dr))):
        assert abs(fd - an) <= mp.mpf(2) ** -200 * (abs(an) + 1), (float(fd), float(an))


def test_objective_sensitivity_formula():
    from conftest import golden
    from test_gpu_solver import _sdp_from_fixture
    from sdpvibe_b200.adjoint import objective_sensitivity, random_directions
    from sdpvibe_b200.solver import Solver
    g = golden("solver_tiny")
    sdp, L = _sdp_from_fixture(g)
    sol = Solver(sdp, L)
    sol.run(max_iter=2)
    dirs = random_directions(sdp, 3, seed=1)
    got = objective_sensitivity(sol, dirs)
    y = sol.y.to_mp().reshape(-1)
    for d, v in zip(dirs, got):
        ref = mp.mpf(0)
        for gi, (dB, dc) in enumerate(d):
            x = sol.st[gi]["xs"]["x"].to_mp()
            B = dB.to_mp()
            c = dc.to_mp()
            for b in range(x.shape[0]):
                for p in range(x.shape[1]):
                    ref += c[b, p, 0] * x[b, p, 0] - x[b, p, 0] * mp.fsum(B[b, p, k] * y[k] for k in range(len(y)))
        assert abs(v - ref) <= mp.mpf(2) ** -(32 * L - 40) * (abs(ref) + 1)
