"""SDPB's binary block files (pmp2sdp --outputFormat bin: a boost binary archive of El::BigFloat records),
read and written with the number records decoded and encoded on the GPU (drop-in for the binary paths of
``sdpvibe.sdp_io``, sdpvibe/sdp_io.py:143-297, and its C codec sdpvibe/_bigfloat.c).

  decode_bigfloats(buf, pos, n, nl, L) -> (MPF (n,) on the device, end position): offsets of the records
      from one pass over their zero flags on the host (sdpv_bigfloat_index), the bytes copied once, one GPU
      thread per record (sdpv_bigfloat_unpack) straight into limb planes
  encode_bigfloats(A, nl) -> bytes (sdpv_bigfloat_pack)
  BinReader(buf, L): the archive (header, El::Matrix<BigFloat> column-major with a leading dimension,
      std::vector<BigFloat>) with matrices and vectors as device MPFs
  read_block_bin(buf, L) / write_block_bin(path, blk, precision, L, N): block_data_<j>.bin

The archive layout (header bytes, class-information bytes, record format) is SDPB's file format and is
reproduced as such.  Decoded mantissas are rounded half up to at most 32 L - 2 bits and not renormalised,
as the reference's host arrays (``mpf.normalize`` makes them normalised MPFs).
"""
import ctypes
import struct

import numpy as np
import torch

from . import _lib
from .mpf import MPF, EZ
from .rns import dev

_SIG = b"serialization::archive"
_BIGFLOAT_CLASS = b"\0\x01\0\0\0"               # El::BigFloat class information, version 1


def limbs_for_precision(precision):
    """GMP limbs of an mpf_t of `precision` bits as the archive stores them (__GMPF_BITS_TO_PREC + 1)"""
    return (precision + 127) // 64 + 1


def decode_bigfloats(buf, pos, n, nl, L):
    arr = np.frombuffer(buf, dtype=np.uint8) if not isinstance(buf, np.ndarray) else buf
    if n == 0:
        return MPF(torch.zeros((L, 0), dtype=torch.int32, device=dev),
                   torch.zeros((0,), dtype=torch.int64, device=dev)), pos
    offs = np.empty(n, dtype=np.int64)
    end = ctypes.c_int64(0)
    st = _lib.lib().sdpv_bigfloat_index(arr.ctypes.data_as(ctypes.c_void_p), len(arr), pos, n, nl,
                                        offs.ctypes.data_as(ctypes.c_void_p), ctypes.addressof(end))
    if st != _lib.OK:
        raise ValueError("truncated or corrupt binary block data")
    lo, hi = int(offs[0]), int(end.value)
    dbuf = torch.from_numpy(np.array(arr[lo:hi])).to(dev)           # one copy of the records, then H2D
    doffs = torch.from_numpy(offs - lo).to(dev)
    m = torch.empty((L, n), dtype=torch.int32, device=dev)
    e = torch.empty((n,), dtype=torch.int64, device=dev)
    _lib.call("sdpv_bigfloat_unpack", _lib.ptr(dbuf), _lib.ptr(doffs), n, nl, L, _lib.ptr(m), _lib.ptr(e), _lib.stream())
    return MPF(m, e), hi


def encode_bigfloats(A, nl):
    """records of the entries of A (any shape, row-major order of its entries)"""
    L = A.L
    m = A.m.reshape(L, -1).contiguous()
    e = A.e.reshape(-1).contiguous()
    n = e.numel()
    if n == 0:
        return b""
    zero = (e == EZ) | (m == 0).all(0)
    lens = torch.where(zero, 1, 13 + 8 * nl).to(torch.int64)
    offs = torch.cumsum(lens, 0) - lens
    total = int(lens.sum())
    out = torch.empty((total,), dtype=torch.uint8, device=dev)
    _lib.device_error_flags()
    _lib.call("sdpv_bigfloat_pack", _lib.ptr(m), _lib.ptr(e), n, L, nl, _lib.ptr(offs), _lib.ptr(out), _lib.stream())
    if _lib.device_error_flags() & _lib.ERR_OVERFLOW:
        raise ValueError("cannot encode (mantissa larger than the archive precision)")
    return out.cpu().numpy().tobytes()


class BinReader:
    """a block_data archive read front to back (sdpvibe/sdp_io.py:143-199)"""

    def __init__(self, buf, L):
        self.b, self.L = buf, L
        p = 0
        n = struct.unpack_from("<Q", buf, p)[0]
        p += 8
        if buf[p:p + n] != _SIG:
            raise ValueError("not a boost binary archive")
        p += n + 2 + 4 + 4                              # signature, library version, sizes, endianness
        self.precision = struct.unpack_from("<Q", buf, p)[0]
        p += 8
        self.nl = limbs_for_precision(self.precision)
        self.p = p
        self.first_bigfloat = self.first_matrix = self.first_vector = True

    def _floats(self, n):
        if n and self.first_bigfloat:
            self.p += 5
            self.first_bigfloat = False
        A, self.p = decode_bigfloats(self.b, self.p, n, self.nl, self.L)
        return A

    def matrix(self):
        """El::Matrix<BigFloat> -> (h, w, MPF (h, w) row-major)"""
        if self.first_matrix:
            self.p += 5
            self.first_matrix = False
        h, w, ld = struct.unpack_from("<iii", self.b, self.p)
        self.p += 12
        A = self._floats(ld * w)
        L = self.L
        m = A.m.reshape(L, w, ld)[:, :, :h].transpose(1, 2).contiguous()
        e = A.e.reshape(w, ld)[:, :h].t().contiguous()
        return h, w, MPF(m, e)

    def vector(self):
        if self.first_vector:
            self.p += 5
            self.first_vector = False
        n = struct.unpack_from("<Q", self.b, self.p)[0]
        self.p += 8 + 4                                 # length, item version
        return self._floats(n)


def read_block_bin(buf, L):
    """block_data_<j>.bin -> dict(B (P, N), c (P,), bilinear_bases_even / _odd: (h, MPF (h, K) or None),
    precision) with every array an MPF on the device (sdpvibe/sdp_io.py:202-217)"""
    r = BinReader(buf, L)
    _, _, B = r.matrix()
    c = r.vector()
    out = {"B": B, "c": c, "precision": r.precision}
    for key in ("bilinear_bases_even", "bilinear_bases_odd"):
        h, _, V = r.matrix()
        out[key] = (h, V if h else None)
    if r.p != len(r.b):
        raise ValueError(f"{len(r.b) - r.p} unexpected trailing bytes")
    return out


def write_block_bin(path, blk, precision, L, N):
    """blk: dict(B MPF (P, N), c MPF (P,), K, bilinear_bases_even / _odd: (h, MPF (h, K) or None)) ->
    block_data_<j>.bin in pmp2sdp's binary format (sdpvibe/sdp_io.py:261-297)"""
    nl = limbs_for_precision(precision)
    hdr = struct.pack("<Q", len(_SIG)) + _SIG + struct.pack("<H", 19) + bytes([4, 8, 4, 8]) + struct.pack("<i", 1)
    parts = [hdr, struct.pack("<Q", precision)]
    first = [True]

    def records(A):
        head = b""
        if first[0]:
            head, first[0] = _BIGFLOAT_CLASS, False
        return head + encode_bigfloats(A, nl)

    def matrix(A, h, w, class_info):                    # row-major (h, w) -> column-major, ld = h
        out = (b"\0" * 5 if class_info else b"") + struct.pack("<iii", h, w, max(h, 1) if w == 0 else h)
        if h * w:
            out += records(MPF(A.m.transpose(-1, -2).contiguous(), A.e.t().contiguous()))
        return out

    B = blk["B"]
    parts.append(matrix(B, B.shape[0], N, True))
    c = blk["c"]
    v = b"\0" * 5 + struct.pack("<Q", c.e.numel()) + struct.pack("<I", 1)
    if c.e.numel():
        v += records(c)
    parts.append(v)
    for key in ("bilinear_bases_even", "bilinear_bases_odd"):
        h, V = blk[key]
        parts.append(struct.pack("<iii", 0, blk["K"], 0) if V is None else matrix(V, h, blk["K"], False))
    with open(path, "wb") as f:
        f.write(b"".join(parts))
