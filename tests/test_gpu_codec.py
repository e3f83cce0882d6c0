"""SDPB's binary records and block files on the GPU (sdpvibe_b200.sdp_io) against the reference's own C
codec and archive writer / reader run on CPU (tests/golden/bigfloat_*.npz, tests/golden/make_golden.py
case_bigfloat): decoded limbs and exponents bit for bit, encoded bytes byte for byte, a block file read
into device MPFs and written back to the same bytes; truncated and corrupt data refused."""
import numpy as np
import pytest
import torch

from conftest import golden, golden_names

pytestmark = pytest.mark.gpu


def _entry_major(A):
    return A.m.reshape(A.L, -1).t().cpu().numpy(), A.e.reshape(-1).cpu().numpy()


@pytest.mark.parametrize("name", golden_names("bigfloat_records_"))
def test_records_decode_encode(name):
    from sdpvibe_b200.mpf import MPF
    from sdpvibe_b200.sdp_io import decode_bigfloats, encode_bigfloats
    g = golden(name)
    n, nl, L = int(g["n"]), int(g["nl"]), int(g["L"])
    A, end = decode_bigfloats(g["raw"], 0, n, nl, L)
    m, e = _entry_major(A)
    assert np.array_equal(m, g["limbs"]) and np.array_equal(e, g["exps"]) and end == int(g["end"])
    B = MPF(torch.from_numpy(np.ascontiguousarray(g["limbs"].T)).cuda(), torch.from_numpy(g["exps"]).cuda())
    assert encode_bigfloats(B, nl) == g["enc"].tobytes()
    with pytest.raises(ValueError):                                  # truncated
        decode_bigfloats(g["raw"][:-1], 0, n, nl, L)


def test_records_refused():
    from sdpvibe_b200.mpf import from_float
    from sdpvibe_b200.sdp_io import decode_bigfloats, encode_bigfloats
    bad = np.frombuffer(b"\x00" + (5).to_bytes(4, "little") + bytes(8 + 8 * 4), np.uint8)   # |size| 5 > nl 4
    with pytest.raises(ValueError):
        decode_bigfloats(bad, 0, 1, 4, 8)
    with pytest.raises(ValueError):                                  # 60-bit-plus mantissas in one limb
        encode_bigfloats(from_float(np.array([1.0 + 2.0 ** -52, 3.0]), 8).shift(-3), 1)


@pytest.mark.parametrize("name", golden_names("bigfloat_block_"))
def test_block_file_roundtrip(name, tmp_path):
    from sdpvibe_b200.sdp_io import read_block_bin, write_block_bin
    g = golden(name)
    L, N, K, h = int(g["L"]), int(g["N"]), int(g["K"]), int(g["h"])
    blk = read_block_bin(g["raw"].tobytes(), L)
    for key, (mref, eref) in (("B", ("Bl", "Be")), ("c", ("cl", "ce"))):
        m, e = _entry_major(blk[key])
        assert np.array_equal(m, g[mref]) and np.array_equal(e, g[eref]), key
    hh, V = blk["bilinear_bases_even"]
    m, e = _entry_major(V)
    assert hh == h and np.array_equal(m, g["hl"]) and np.array_equal(e, g["he"])
    assert blk["bilinear_bases_odd"] == (0, None)
    assert blk["B"].shape == (g["Be"].size // N, N)
    blk["K"] = K
    out = tmp_path / "block.bin"
    write_block_bin(out, blk, int(g["precision"]), L, N)
    assert out.read_bytes() == g["raw"].tobytes()
