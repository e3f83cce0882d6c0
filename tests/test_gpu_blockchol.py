"""The tiled Cholesky of Q (sdpvibe_b200.blockchol.BlockChol) against the reference's own BlockChol run on
CPU (tests/golden/blockchol_n70_b32.npz: N = 70 in tiles of 32, 32 and 6, L = 8): the three solves bit for
bit and the condition estimate; and the solver with the tiled factorisation forced."""
import mpmath as mp
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def test_blockchol_matches_reference():
    from sdpvibe_b200.blockchol import BlockChol
    from sdpvibe_b200.mpf import MPF
    g = golden("blockchol_n70_b32")
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ch = BlockChol([MPF(cu(g["Qm"]), cu(g["Qe"]))], int(g["b"]))
    B = MPF(cu(g["Bm"]), cu(g["Be"]))
    for name, X in (("lo", ch.solve_lower(B)), ("up", ch.solve_upper(B)), ("x", ch.solve(B))):
        assert np.array_equal(X.m.cpu().numpy(), g[f"{name}_m"]), name
        assert np.array_equal(X.e.cpu().numpy(), g[f"{name}_e"]), name
    assert ch.log2_cond() == float(g["log2_cond"])


def test_solver_with_tiled_q_factorisation(monkeypatch):
    """SDPB_GPU_QBLOCK forces the tiled factorisation of Q: the run agrees with the monolithic one to
    working precision (different rounding order)"""
    from sdpvibe_b200.solver import Solver
    from sdpvibe_b200.synthetic import ising_like_sdp
    logs = {}
    for qb in (0, 8):
        monkeypatch.setenv("SDPB_GPU_QBLOCK", str(qb))
        sdp, _ = ising_like_sdp(12, nblocks=10, N=20)
        log = []
        Solver(sdp, 12).run(max_iter=3, log=log)
        logs[qb] = log
    for a, b in zip(logs[0], logs[8]):
        for k in ("pobj", "dobj", "P_step", "D_step"):
            assert abs(a[k] - b[k]) <= mp.mpf(10) ** -60 * (abs(a[k]) + 1), k
