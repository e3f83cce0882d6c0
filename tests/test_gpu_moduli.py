"""The prime split chosen by the autotuner (the moduli group G of the library's own RNS contexts) never changes
a bit: every product is exact for any moduli set with M > 4 kmax 2^(2(32 L - 1)) (sdpvibe/rns.py:166-173),
so mp GEMMs, Gram accumulations (with flushes) and grouped Cholesky solves give the same results for every
G, and the reference-format context RNS(L) keeps its 16-moduli groups."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def _results(L):
    from sdpvibe_b200 import mpf
    from sdpvibe_b200.kernel_bench import cholsolve_inputs, cholsolve_buckets
    rng = np.random.default_rng(5)
    A = mpf.from_float(rng.standard_normal((70, 90)), L)
    B = mpf.from_float(rng.standard_normal((90, 50)), L)
    # three chunks whose scales grow past the accumulator's headroom: the later ones force flushes
    V = [mpf.from_float(rng.standard_normal((r, 40)) * s, L) for r, s in ((60, 1.0), (45, 2.0 ** 20), (80, 2.0 ** 45))]
    pairs = [(Ab, Bb) for _, _, Ab, Bb in cholsolve_buckets(cholsolve_inputs(12, 8, 100, 4, seed=3), L)]
    C = mpf.gemm(A, B)
    acc = mpf.GramAcc(40, L)
    for v in V:
        acc.add(v)
    Q = acc.result()
    low = torch.tril(torch.ones((40, 40), dtype=torch.bool, device="cuda"))
    X = mpf.chol_solve_many(pairs)
    out = [C.m, C.e, Q.m[:, low], Q.e[low]] + [t for x in X for t in (x.m, x.e)]
    return [t.clone() for t in out], acc.flushes


@pytest.mark.parametrize("L", [8, 26])
def test_moduli_group_same_bits(L):
    from sdpvibe_b200 import autotune, mpmat
    from sdpvibe_b200.rns import RNS
    default = autotune.get_knob("moduli_group")
    outs, mods, fl = {}, {}, {}
    try:
        for G in (16, 8, 4, 1):
            autotune.set_knob("moduli_group", G)
            mods[G] = list(mpmat.lib_ctx(L).mods)
            outs[G], fl[G] = _results(L)
    finally:
        autotune.set_knob("moduli_group", default)
    # the moduli of the reference's rule with groups of G primes (the oracle's restatement of rns.py:166-173)
    want = {G: [int(m) for m in O.RNSTables(L, G=G).mods] for G in (16, 8, 4, 1)}
    assert mods == want and len(mods[1]) < len(mods[16])
    assert fl[16] > 0 and len(set(fl.values())) == 1
    for G in (8, 4, 1):
        for a, b in zip(outs[16], outs[G]):
            assert torch.equal(a, b)
    assert list(RNS(L).mods) == want[16]              # the API's contexts keep the reference's moduli
    assert list(mpmat.ctx(L).mods) == want[16]


def test_moduli_group_knob_range():
    from sdpvibe_b200 import autotune
    from sdpvibe_b200 import _lib
    default = autotune.get_knob("moduli_group")
    for bad in (0, 3, 32):
        with pytest.raises(ValueError):
            _lib.call("sdpv_tune_set", 4, bad)
    assert autotune.get_knob("moduli_group") == default
