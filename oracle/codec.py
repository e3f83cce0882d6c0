"""TEST INFRASTRUCTURE ONLY: Python-integer restatement of SDPB's binary number records (boost-serialised
El::BigFloat, GMP mpf_t limbs), the checker of the device codec (sdpvibe_b200/csrc/codec.cu).

Record (sdpvibe/_bigfloat.c:1-12): byte is_zero; unless zero, int32 size, int64 exp and nl 64-bit limbs;
value = sign(size) M 2^(64 (exp - |size|)) with M the first |size| limbs.  decode (sdpvibe/_bigfloat.c:16-61,
sdpvibe/sdp_io.py:119-141): M rounded half up to at most 32L - 2 bits (right shift s), L 32-bit
two's-complement limbs, exponent 64 (exp - |size|) + s; zeros -> 0, EZ.  encode (sdpvibe/_bigfloat.c:63-111):
the inverse with the exponent's residue mod 64 moved into the mantissa and all |size| used limbs kept.
Entries are entry-major (n, L) here, as the reference's host arrays.
"""
import struct

import numpy as np

EZ = -(1 << 40)


def decode(buf, pos, n, nl, L):
    """-> (limbs (n, L) int32, exps (n,) int64, end position); ValueError on a short or corrupt buffer"""
    buf = bytes(buf)
    T = 32 * L - 2
    limbs = np.zeros((n, L), np.int32)
    exps = np.full(n, EZ, np.int64)
    for i in range(n):
        if pos >= len(buf):
            raise ValueError("truncated")
        zero = buf[pos]
        pos += 1
        if zero:
            continue
        if pos + 12 + 8 * nl > len(buf):
            raise ValueError("truncated")
        size, exp = struct.unpack_from("<iq", buf, pos)
        pos += 12
        asz = abs(size)
        if asz > nl:
            raise ValueError("corrupt record")
        M = int.from_bytes(buf[pos:pos + 8 * asz], "little")
        pos += 8 * nl
        if M == 0:
            continue
        s = max(0, M.bit_length() - T)
        if s:
            M = (M + (1 << (s - 1))) >> s
        v = -M if size < 0 else M
        limbs[i] = np.frombuffer(v.to_bytes(4 * L, "little", signed=True), np.int32)
        exps[i] = 64 * (exp - asz) + s
    return limbs, exps, pos


def encode(limbs, exps, nl):
    """(n, L) int32 two's-complement mantissas with exponents -> record bytes; ValueError if a mantissa
    needs more than nl 64-bit limbs"""
    out = bytearray()
    limbs = np.asarray(limbs, np.int32)
    for row, e in zip(limbs, np.asarray(exps, np.int64)):
        v = int.from_bytes(row.tobytes(), "little", signed=True)
        if v == 0 or e == EZ:
            out += b"\x01"
            continue
        r = int(e) % 64                                   # value = (|v| << r) 2^(64 base)
        base = (int(e) - r) // 64
        D = abs(v) << r
        size = (D.bit_length() + 63) // 64
        if size > nl:
            raise ValueError("mantissa larger than the archive precision")
        out += b"\x00" + struct.pack("<iq", -size if v < 0 else size, base + size)
        out += D.to_bytes(8 * nl, "little")
    return bytes(out)
