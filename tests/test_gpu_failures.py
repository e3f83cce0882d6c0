"""Failure paths on the GPU, made without a GPU fault.

* A bounded pipeline wait that nothing completes (sdpv_wait_probe with arrive = 0) gives up after its
  limit, the device error word reports SDPV_ETIMEOUT, and the context stays usable.
* A matrix whose diagonal is not positive raises the reference's ValueError (sdpvibe/mpf.py:475-476),
  eagerly and through the deferred check of chol_solve_many.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_stays_usable():
    from sdpvibe_b200 import _lib
    from sdpvibe_b200.limbops import add_same
    _lib.device_error_flags()                                  # start from a clear error word
    st = _lib.lib().sdpv_wait_probe(1000, 1, _lib.stream())   # the barrier completes: no timeout
    assert st == _lib.OK
    assert _lib.lib().sdpv_device_status(_lib.stream()) == _lib.OK
    st = _lib.lib().sdpv_wait_probe(20000, 0, _lib.stream())  # nothing completes it: gives up after 20 ms
    assert st == _lib.OK                                       # the launch itself is fine
    assert _lib.lib().sdpv_device_status(_lib.stream()) == _lib.ETIMEOUT
    assert _lib.lib().sdpv_device_status(_lib.stream()) == _lib.OK   # read and cleared
    _lib.lib().sdpv_wait_probe(20000, 0, _lib.stream())
    with pytest.raises(RuntimeError, match="timed out"):
        _lib.device_status()
    a = torch.arange(12, dtype=torch.int32, device="cuda").view(3, 4)
    assert torch.equal(add_same(a, a, 1), 2 * a)               # later kernels still run
    assert _lib.lib().sdpv_wait_probe(0, 0, _lib.stream()) == _lib.EINVAL


def test_non_positive_diagonal_raises_value_error():
    from sdpvibe_b200 import mpf
    A = np.eye(40)[None].repeat(2, 0) * 3.0
    A[1, 7, 7] = -1.0
    with pytest.raises(ValueError, match="not positive definite"):
        mpf.Chol(mpf.from_float(A, 26))
    A[1, 7, 7] = 0.0                                           # a zero pivot as well
    with pytest.raises(ValueError, match="not positive definite"):
        mpf.Chol(mpf.from_float(A, 26))
    B = mpf.from_float(np.ones((2, 40, 1)), 26)
    good = mpf.from_float(np.eye(40)[None].repeat(2, 0) * 2.0, 26)
    with pytest.raises(ValueError, match="not positive definite"):
        mpf.chol_solve_many([(good, B), (mpf.from_float(A, 26), B)])
