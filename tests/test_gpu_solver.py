"""The SDPB iteration (sdpvibe_b200.solver.Solver) on the GPU against the reference's own iterates.

tests/golden/solver_tiny.npz holds a tiny SDP (4 blocks of dims 1, 1, 2, 3; N = 5; L = 8) and, for its
first iterations, what the reference's Solver.run produced (tests/golden/make_solver_golden.py): the
printed scalars, the step lengths, y, and each chunk's corrector direction.  The GPU run must reproduce
them bit for bit when the step-length eigenvalues come from LAPACK on the host, as in the reference (both
runs use numpy's, on bit-identical input matrices), and to 1e-13 relative with the GPU eigenvalue kernel.""" 
import mpmath as mp
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _mpstr(v):
    s, man, ex, _ = mp.mpf(v)._mpf_
    return f"{'-' if s else ''}{int(man)}*2^{int(ex)}"


def _sdp_from_fixture(g):
    from sdpvibe_b200.solver import SDP
    L = int(g["L"])
    blocks = []
    for j, (dim, K) in enumerate(zip(g["blk_dim"].tolist(), g["blk_K"].tolist())):

        def arr(name):
            key = f"blk{j}_{name}"
            return (g[key + "_m"], g[key + "_e"]) if key + "_m" in g.files else None
        blocks.append(dict(dim=dim, K=K, Ve=arr("Ve"), Vo=arr("Vo"), c=arr("c"), B=arr("B")))
    return SDP(blocks, (g["b_m"], g["b_e"]), 0, L), L


def test_solver_iterates_match_reference(monkeypatch):
    """with the step-length eigenvalues from LAPACK on the host, as the reference: bit-identical"""
    from sdpvibe_b200 import solver
    from sdpvibe_b200.solver import Solver, fmt_big
    monkeypatch.setattr(solver, "EIG_DEVICE", False)
    g = golden("solver_tiny")
    iters = int(g["iters_done"])
    sdp, L = _sdp_from_fixture(g)
    assert [j for grp in sdp.groups for j in grp.idx] == g["chunk_blocks"].tolist()
    sol = Solver(sdp, L)
    seen = []
    names = {"mu": "mu", "P-obj": "pobj", "D-obj": "dobj", "gap": "gap", "P-err": "P_err", "p-err": "p_err",
             "D-err": "D_err", "R-err": "R_err", "P-step": "P_step", "D-step": "D_step", "beta": "beta"}

    def rec(it, s, info):
        row = info["row"]
        for ref_key, key in names.items():
            assert fmt_big(row[key], s.digits) == str(g[f"it{it}_{ref_key}"]), (it, ref_key)
        assert _mpstr(s.last_steps[0]) == str(g[f"it{it}_aP"]) and _mpstr(s.last_steps[1]) == str(g[f"it{it}_aD"])
        assert np.array_equal(s.y.m.cpu().numpy(), g[f"it{it}_y_m"]), it
        assert np.array_equal(s.y.e.cpu().numpy(), g[f"it{it}_y_e"]), it
        for gi, o in enumerate(s.st):
            dc = o["dc"]
            for name, M in (("dx", dc["dx"]), ("dX", dc["dX"][0]), ("dY", dc["dY"][0])):
                assert np.array_equal(M.m.cpu().numpy(), g[f"it{it}_g{gi}_{name}_m"]), (it, gi, name)
                assert np.array_equal(M.e.cpu().numpy(), g[f"it{it}_g{gi}_{name}_e"]), (it, gi, name)
        seen.append(it)
    res = sol.run(max_iter=iters, record=rec)
    assert seen == list(range(1, iters + 1))
    if "terminate" in g.files:
        assert res["terminateReason"] == str(g["terminate"])


def test_solver_ising_like_small_runs():
    """a small instance of the Ising-structured benchmark SDP: two iterations, finite objectives,
    steps in (0, 1]"""
    from sdpvibe_b200.solver import Solver
    from sdpvibe_b200.synthetic import ising_like_sdp
    sdp, blocks = ising_like_sdp(12, nblocks=10, N=20)
    log = []
    Solver(sdp, 12).run(max_iter=2, log=log)
    assert len(log) == 2
    for row in log:
        assert 0 < row["P_step"] <= 1 and 0 < row["D_step"] <= 1
        assert mp.isfinite(row["pobj"]) and mp.isfinite(row["dobj"])


def test_solver_iterates_device_eigenvalues_near_reference():
    """with the step-length eigenvalues from the GPU Jacobi kernel: the float64 lambda_min may differ from
    LAPACK's in the last bits, so the steps (and the iterates after them) agree to 1e-13 relative"""
    from sdpvibe_b200 import solver
    from sdpvibe_b200.mpf import MPF
    from sdpvibe_b200.solver import Solver
    assert solver.EIG_DEVICE
    g = golden("solver_tiny")
    iters = int(g["iters_done"])
    sdp, L = _sdp_from_fixture(g)
    sol = Solver(sdp, L)
    worst = [0.0]

    def close(M, key):
        got = M.to_mp().reshape(-1)
        ref = MPF(torch.from_numpy(g[key + "_m"]).cuda(), torch.from_numpy(g[key + "_e"]).cuda()).to_mp().reshape(-1)
        scale = max(abs(v) for v in ref) or mp.mpf(1)
        d = max(abs(a - b) for a, b in zip(got, ref)) / scale
        worst[0] = max(worst[0], float(d))
        assert d <= mp.mpf("1e-13"), (key, float(d))

    def rec(it, s, info):
        for k, v in zip(("aP", "aD"), s.last_steps[:2]):
            man, ex = str(g[f"it{it}_{k}"]).split("*2^")
            ref = mp.mpf(int(man)) * mp.mpf(2) ** int(ex)
            assert abs(v / ref - 1) <= mp.mpf("1e-13"), (it, k)
        close(s.y, f"it{it}_y")
        for gi, o in enumerate(s.st):
            close(o["dc"]["dx"], f"it{it}_g{gi}_dx")
    sol.run(max_iter=iters, record=rec)


@pytest.mark.parametrize("dims,K,L", [((1, 2, 3), 5, 8), ((2, 3), 9, 26), ((1, 4), 3, 12)])
def test_schur_kernel_matches_composition(dims, K, L):
    """the fused Schur assembly (sdpv_schur_assemble) gives the bits of the composed elementwise operations,
    on random pairings with zeros and padding rows"""
    from sdpvibe_b200 import mpf as F
    from sdpvibe_b200.mpf import MPF
    from sdpvibe_b200.solver import SDP, Solver
    rng = np.random.default_rng(K + L)
    blocks = []
    for d in dims:
        for kk in (K, K - 1):
            npair = d * (d + 1) // 2
            blocks.append(dict(dim=d, K=kk, Ve=rng.standard_normal((2, kk)), Vo=rng.standard_normal((1, kk)),
                               c=rng.standard_normal((kk * npair, 1)), B=rng.standard_normal((kk * npair, 3))))
    sdp = SDP(blocks, rng.standard_normal((3, 1)), 0, L)
    sol = Solver(sdp, L)
    for g in sdp.groups:
        W = g.dim * g.K
        shape = (2 * g.nb, W, W)

        def sym():
            v = rng.standard_normal(shape) * 2.0 ** rng.integers(-30, 30, size=shape)
            v[rng.random(shape) < 0.1] = 0
            return F.from_float((v + np.swapaxes(v, 1, 2)) / 2, L)
        A, Y = sym(), sym()
        got = sol.schur(g, [A], [Y])
        ref = sol.schur_composed(g, [A], [Y])
        assert torch.equal(got.m, ref.m) and torch.equal(got.e, ref.e), g.dim
