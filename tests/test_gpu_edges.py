"""Edge cases of the C-ABI path on the GPU: empty operands (zero rows, columns, K, entries), invalid
arguments (refused with a status that maps to ValueError, before any launch), and the largest sizes the
entry points accept (K = 65536 in one residue GEMM, L = 160 in the elementwise kernels), each against the
oracle or the documented result."""
import numpy as np
import pytest
import torch

import oracle as O
from test_gpu_kernels import _rand_mpf_np, _rand_residues, cu, np_

pytestmark = pytest.mark.gpu


def test_empty_operands():
    from sdpvibe_b200 import mpf
    from sdpvibe_b200.mpmat import ctx
    L = 26
    R = ctx(L)
    # decomposition of zero rows / zero K
    for rows, K in ((0, 48), (5, 0)):
        Rhi, Rlo = R.residues(torch.zeros((L, rows, K), dtype=torch.int32, device="cuda"), 0, K)
        assert Rhi.shape[1] == rows and Rlo.shape == Rhi.shape
    # residue GEMM with M, N or K zero leaves the accumulator as it is
    acc0 = torch.randint(0, 1000, (R.n, 7, 9), dtype=torch.int16, device="cuda")
    for M, N, K in ((0, 9, 16), (7, 0, 16), (7, 9, 0)):
        acc = acc0[:, :max(M, 1), :max(N, 1)].clone()
        keep = acc.clone()
        A = torch.zeros((R.n, M, K), dtype=torch.int8, device="cuda")
        B = torch.zeros((R.n, N, K), dtype=torch.int8, device="cuda")
        R.accumulate(A, A, B, B, acc)
        assert torch.equal(acc, keep)
    # CRT of no entries
    Wd, bl, n = R.crt_block(acc0, 9, 0, 9, 0)
    assert n == 0 and Wd.shape[1] == 0 and bl.numel() == 0
    # MPF: elementwise on no entries, a GEMM with K = 0 is exact zero
    Z = mpf.zeros((0,), L)
    assert mpf.add(Z, Z).shape == (0,) and mpf.mul(Z, Z).shape == (0,)
    A = mpf.from_float(np.ones((3, 0)), L)
    B = mpf.from_float(np.ones((0, 4)), L)
    C = mpf.gemm(A, B)
    assert C.shape == (3, 4)
    assert bool((C.m == 0).all()) and bool((C.e == mpf.EZ).all())
    assert mpf.total(Z) == 0 and mpf.max_abs(Z) == 0


def test_invalid_arguments_raise():
    from sdpvibe_b200 import _lib
    from sdpvibe_b200.mpmat import ctx
    R = ctx(26)
    _lib.device_error_flags()                                        # start from a clear error word
    A = torch.zeros((R.n, 8, 48), dtype=torch.int8, device="cuda")
    acc = torch.zeros((R.n, 8, 8), dtype=torch.int16, device="cuda")
    with pytest.raises(ValueError):                                  # K not a multiple of 16
        _lib.call("sdpv_rns_gemm", R._h, _lib.ptr(A), _lib.ptr(A), _lib.ptr(A), _lib.ptr(A), 0, 0, _lib.ptr(acc), 8,
                  0, R.n, 1, 8, 8, 40, 0, _lib.stream())
    with pytest.raises(ValueError):                                  # moduli beyond the context
        _lib.call("sdpv_rns_gemm", R._h, _lib.ptr(A), _lib.ptr(A), _lib.ptr(A), _lib.ptr(A), 0, 0, _lib.ptr(acc), 8,
                  1, R.n, 1, 8, 8, 48, 0, _lib.stream())
    with pytest.raises(ValueError):                                  # column block beyond N
        R.crt_block(acc, 8, 4, 5, 8)
    v = torch.zeros(4, dtype=torch.float64, device="cuda")
    m = torch.empty((1, 4), dtype=torch.int32, device="cuda")
    e = torch.empty(4, dtype=torch.int64, device="cuda")
    with pytest.raises(ValueError):                                  # one limb cannot hold a double exactly
        _lib.call("sdpv_mpf_from_f64", 1, 4, _lib.ptr(v), _lib.ptr(m), _lib.ptr(e), _lib.stream())
    assert _lib.device_error_flags() == 0                            # nothing was launched


def test_residue_gemm_largest_k():
    """K = 65536, the largest K one launch accepts (int32 accumulation exact: |hh| <= K 2^14 = 2^30),
    on the narrow path (3 x 70 block)"""
    from sdpvibe_b200.mpmat import ctx
    L, M, N, K = 26, 3, 70, 65536
    rng = np.random.default_rng(11)
    T = O.tables(L)
    R = ctx(L)
    Ah, Al = _rand_residues(rng, T, T.n, M, K)
    Bh, Bl = _rand_residues(rng, T, T.n, N, K)
    m = T.m32.astype(np.int64)[:, None, None]
    acc0 = (rng.integers(0, 1 << 30, size=(T.n, M, N)) % m).astype(np.int16)
    acc = cu(acc0).clone()
    R.accumulate(cu(Ah), cu(Al), cu(Bh), cu(Bl), acc)
    assert np.array_equal(np_(acc), O.accumulate(T, Ah, Al, Bh, Bl, acc0, 0))


def test_elementwise_largest_limb_count():
    """L = 160, the largest limb count of the elementwise MPF kernels"""
    from sdpvibe_b200.mpf import MPF, add, mul
    L = 160
    rng = np.random.default_rng(5)
    am, ae = _rand_mpf_np(rng, L, (97,))
    bm, be = _rand_mpf_np(rng, L, (97,))
    A, B = MPF(cu(am), cu(ae)), MPF(cu(bm), cu(be))
    for got, (rm, re_) in ((mul(A, B), O.mpf_mul(am, ae, bm, be)), (add(A, B), O.mpf_add(am, ae, bm, be)),
                           (add(A, B, -1), O.mpf_add(am, ae, bm, be, -1))):
        assert np.array_equal(np_(got.m), rm) and np.array_equal(np_(got.e), re_)
