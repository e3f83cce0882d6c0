"""Load the reference package (SDPviBe) on CPU torch, for golden-vector generation only.

The reference's Triton kernels run under Triton's interpreter (TRITON_INTERPRET=1) and its CUDA C
kernel strings run as host code through the ``cupy`` stand-in of ``oracle/ref_build.py``.  Two
shims keep the reference's arithmetic unchanged:

* ``rns._crt_dot_kernel`` passes ``tl.dot(int8, int8, acc_int32)`` without ``out_dtype``, which the
  installed Triton 3.6 rejects (``sdpvibe/rns.py:157-158``); it is replaced by the exact int64
  product it computes, ``Z = Ct @ (128*Yhi + Ylo)^T``.
* ``libdevice.clz`` (``sdpvibe/limbops.py:150,209``) has no interpreter implementation; it is
  replaced by an exact numpy count of leading zeros.

This module must be imported before torch/triton are imported anywhere else in the process.
It reads the reference tree and is never used on the GPU box.
"""
import os
import sys

os.environ["TRITON_INTERPRET"] = "1"
HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE_ROOT = os.environ.get("SDPV_REFERENCE_ROOT")
if not REFERENCE_ROOT or not os.path.isdir(os.path.join(REFERENCE_ROOT, "sdpvibe")):
    raise RuntimeError("set SDPV_REFERENCE_ROOT to the reference (SDPviBe) source tree to generate golden vectors")
sys.path.insert(0, REPO)
sys.path.insert(0, REFERENCE_ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

torch.cuda.current_device = lambda: 0

from oracle.ref_build import install_cupy_shim  # noqa: E402

install_cupy_shim()

import triton.language as tl  # noqa: E402
from triton.runtime.interpreter import TensorHandle  # noqa: E402


def _clz(x, _semantic=None, **kw):
    v = x.handle.data.astype(np.uint32).astype(np.float64)
    bl = np.where(v == 0, 0, np.frexp(v)[1]).astype(np.int32)
    return tl.tensor(TensorHandle((32 - bl).astype(np.int32), tl.int32), tl.int32)


tl.extra.cuda.libdevice.clz = _clz

import sdpvibe.rns as rns  # noqa: E402

rns.dev = "cpu"
import sdpvibe.limbops as limbops  # noqa: E402

limbops.dev = "cpu"


class _CrtDot:
    """Exact restatement of rns._crt_dot_kernel: Z = Ct @ (128*Yhi + Ylo)^T (int32 result)."""

    def __getitem__(self, grid):
        def run(Ct, Yhi, Ylo, Z, E, B, N, **kw):
            y = 128 * Yhi[:B, :N].to(torch.int64) + Ylo[:B, :N].to(torch.int64)
            Z[:E, :B] = (Ct[:E, :N].to(torch.int64) @ y.T).to(torch.int32)
        return run


rns._crt_dot_kernel = _CrtDot()

import sdpvibe.mpmat as mpmat  # noqa: E402
import sdpvibe.basecase as basecase  # noqa: E402
import sdpvibe.linalg as linalg  # noqa: E402
import sdpvibe.batched as batched  # noqa: E402
import sdpvibe.mpf as mpf  # noqa: E402

for _m in (mpmat, basecase, linalg, batched, mpf):
    if hasattr(_m, "dev"):
        _m.dev = "cpu"
