"""Parity at the benchmarked configurations, on the benchmark's own inputs.

* Gram accumulation (bench.py's default workload): GramAcc(274, 26) over the 400 blocks m_b ~ U[20, 120]
  (seed 0) in 4 chunks with E_ref = None -- the lower triangle of Q bit-exact against the oracle's GramAcc
  (the restatement of sdpvibe/mpf.py:536-630); and a pair of chunks whose second chunk outgrows the
  column references, so the flush path (CRT of the partial sum, MPF add) runs at full N = 274.
* Batched Cholesky + solve (bench.py --workload cholsolve): blocks of every padded size 32 ... 160 taken
  from the benchmark's 600-block input, factored and solved as the benchmark does, bit-exact against the
  oracle's Chol (sdpvibe/mpf.py:461-532, sdpvibe/batched.py:274-352).
"""
import numpy as np
import pytest
import torch

import bench
from oracle import mp as OM

pytestmark = pytest.mark.gpu


def np_(t):
    return t.detach().cpu().numpy()


def _lower(a):
    n = a.shape[-1]
    return np.where(np.tril(np.ones((n, n), bool)), a, 0)


def _gram_gpu(chunks, N, L, E_ref=None):
    from sdpvibe_b200 import mpf
    acc = mpf.GramAcc(N, L, E_ref=E_ref)
    for m, e in chunks:
        acc.add(mpf.MPF(torch.from_numpy(m).cuda(), torch.from_numpy(e).cuda()))
    Q = acc.result()
    return np_(Q.m), np_(Q.e), acc.flushes


def _gram_oracle(chunks, N, L):
    ref = OM.GramAcc(N, L)
    for m, e in chunks:
        ref.add(m, e)
    qm, qe = ref.result()
    return qm, qe, ref.flushes


def test_gram_configuration_full_size_vs_oracle():
    """The Gram configuration exactly as bench.py times it (rank 0's data), E_ref = None."""
    _, rows = bench.workload_shape()
    rng = np.random.default_rng(100)                       # bench.run_b200's generator on rank 0
    chunks = [bench.gen_chunk(rng, r, bench.NCOLS, bench.L) for r in rows]
    gm, ge, gf = _gram_gpu(chunks, bench.NCOLS, bench.L)
    om, oe, of = _gram_oracle(chunks, bench.NCOLS, bench.L)
    assert gf == of
    assert np.array_equal(_lower(gm), _lower(om))
    assert np.array_equal(_lower(ge), _lower(oe))


def test_gram_full_width_flush_vs_oracle():
    """Two chunks at N = 274, L = 26; the second chunk's columns 0, 100 and 273 are 2^40 larger, past the
    HEAD = 28 bits of headroom of the references the first chunk set: one flush, then one more CRT."""
    rng = np.random.default_rng(5)
    a = bench.gen_chunk(rng, 300, bench.NCOLS, bench.L)
    bm, be = bench.gen_chunk(rng, 250, bench.NCOLS, bench.L)
    be = be.copy()
    be[:, [0, 100, 273]] += 40
    chunks = [a, (bm, be)]
    gm, ge, gf = _gram_gpu(chunks, bench.NCOLS, bench.L)
    om, oe, of = _gram_oracle(chunks, bench.NCOLS, bench.L)
    assert of == 1 and gf == 1
    assert np.array_equal(_lower(gm), _lower(om))
    assert np.array_equal(_lower(ge), _lower(oe))


def test_cholsolve_configuration_every_padded_size_vs_oracle():
    """Two blocks of each padded size 32, 64, 96, 128, 160 from the benchmark's 600-block input (n up to
    160, 8 right-hand sides, L = 26), through the benchmark's call, against the oracle per size."""
    from sdpvibe_b200 import mpf
    from sdpvibe_b200.kernel_bench import cholsolve_inputs, cholsolve_buckets
    cases = cholsolve_inputs(bench.CS_BLOCKS, bench.CS_NMIN, bench.CS_NMAX, bench.CS_NRHS)
    pick, seen = [], {}
    for i, (n, _, _) in enumerate(cases):
        p = max(32, -(-n // 32) * 32)
        if seen.get(p, 0) < 2:
            seen[p] = seen.get(p, 0) + 1
            pick.append(cases[i])
    assert sorted(seen) == [32, 64, 96, 128, 160] and max(c[0] for c in pick) > 128
    buckets = cholsolve_buckets(pick, bench.CS_L)
    outs = mpf.chol_solve_many([(A, B) for _, _, A, B in buckets])
    for (npad, idx, A, B), X in zip(buckets, outs):
        ref = OM.Chol(np_(A.m), np_(A.e))
        rm, re_ = ref.solve(np_(B.m), np_(B.e))
        assert np.array_equal(np_(X.m), rm) and np.array_equal(np_(X.e), re_), npad
