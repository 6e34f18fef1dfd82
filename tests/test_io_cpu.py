"""Output/input formats of libmm_b200.so (host code, no GPU): OVF 2.0 and OMF 1.0
(ovf/ovf2_output.go, ovf/omf_output.go, ovf/omf_input.go) and the dump format with its
CRC-64 (dump/writer.go, dump/reader.go, engine/format_dump.go)."""
import struct

import numpy as np
import pytest

from mumax2 import _native as nat


def _crc64_go_iso(data):
    """Go's hash/crc64 with the ISO table, written out independently for the check."""
    poly = 0xD800000000000000
    tab = []
    for i in range(256):
        c = i
        for _ in range(8):
            c = (c >> 1) ^ poly if c & 1 else c >> 1
        tab.append(c)
    crc = 0xFFFFFFFFFFFFFFFF
    for b in data:
        crc = tab[(crc ^ b) & 0xFF] ^ (crc >> 8)
    return crc ^ 0xFFFFFFFFFFFFFFFF


def test_crc64_iso_check_value():
    import ctypes as C
    buf = b"123456789"
    # published check value of CRC-64/GO-ISO
    assert nat.lib().mm_crc64_iso(C.c_char_p(buf), len(buf)) == 0xB90956C775A41001
    assert _crc64_go_iso(buf) == 0xB90956C775A41001


def _data(ncomp, n, seed=0):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(ncomp,) + tuple(n)).astype(np.float32)


@pytest.mark.parametrize("fmt,opts", [("ovf", []), ("ovf", ["Text"]), ("omf", []), ("omf", ["text"]),
                                      ("dump", [])])
@pytest.mark.parametrize("ncomp", [1, 3])
def test_round_trip(tmp_path, fmt, opts, ncomp):
    if fmt == "omf" and ncomp == 1:
        pytest.skip("OMF 1.0 files carry vector fields; the reader takes 3 components (omf_input.go:35)")
    n = (2, 3, 5)
    a = _data(ncomp, n, seed=ncomp)
    path = tmp_path / f"f.{fmt}"
    nat.write_field(path, nat.format_code(fmt, opts), a, n, (3e-9, 4e-9, 5e-9), 1.25e-11, "m", "")
    b, nn, t = nat.read_field(path)
    assert nn == n and b.shape == a.shape
    assert np.array_equal(a, b)  # binary is exact; text uses shortest round-trip digits
    if fmt != "omf":
        assert t == pytest.approx(1.25e-11)


def test_ovf2_header_and_byte_order(tmp_path):
    n = (1, 2, 4)  # internal (z, y, x): user 4 x 2 x 1
    a = np.arange(3 * 8, dtype=np.float32).reshape(3, *n)
    p = tmp_path / "m.ovf"
    nat.write_field(p, nat.format_code("ovf"), a, n, (3e-9, 2e-9, 1e-9), 5e-12, "m", "")
    raw = p.read_bytes()
    head, rest = raw.split(b"# Begin: Data Binary 4\n", 1)
    lines = head.decode().splitlines()
    assert lines[0] == "# OOMMF OVF 2.0"
    assert "# xnodes: 4" in lines and "# ynodes: 2" in lines and "# znodes: 1" in lines
    assert "# xstepsize: 1e-09" in lines and "# zstepsize: 3e-09" in lines
    assert "# valuelabels: m_x m_y m_z" in lines and "# valueunits: 1 1 1" in lines
    assert "# Desc: Total simulation time:  5e-12  s" in lines
    assert rest[:4] == struct.pack("<f", 1234567.0)
    vals = np.frombuffer(rest[4:4 + 4 * 24], dtype="<f4").reshape(8, 3)
    # cells x fastest, components in user order (internal component 2 first)
    assert np.array_equal(vals[:, 0], a[2].ravel()) and np.array_equal(vals[:, 2], a[0].ravel())
    assert rest[4 + 96:].decode() == "# End: Data Binary 4\n# End: Segment\n"


def test_omf_big_endian_control_number(tmp_path):
    n = (1, 1, 2)
    p = tmp_path / "m.omf"
    nat.write_field(p, nat.format_code("omf"), _data(3, n), n, (1e-9, 1e-9, 1e-9), 0.0, "m", "")
    raw = p.read_bytes()
    assert raw.startswith(b"# OOMMF: rectangular mesh v1.0\n")
    data = raw.split(b"# Begin: Data Binary 4\n", 1)[1]
    assert data[:4] == bytes([0x49, 0x96, 0xB4, 0x38])  # 1234567.0 big-endian


def test_dump_frame_layout_and_crc(tmp_path):
    """The frame of dump/dump_test.go (1 component, 2x4x9, steps 1,2,3 nm, t = 1e-15)."""
    n = (2, 4, 9)
    a = np.arange(72, dtype=np.float32).reshape(1, *n)
    p = tmp_path / "f.dump"
    nat.write_field(p, nat.format_code("dump"), a, n, (1e-9, 2e-9, 3e-9), 1e-15, "Msat", "A/m")
    raw = p.read_bytes()
    assert raw[:8] == b"#dump002"
    comps, s0, s1, s2 = struct.unpack("<4Q", raw[8:40])
    assert (comps, s0, s1, s2) == (1, 2, 4, 9)
    assert struct.unpack("<3d", raw[40:64]) == (1e-9, 2e-9, 3e-9)
    assert raw[64:72] == b"m" + b"\0" * 7
    assert struct.unpack("<d", raw[72:80])[0] == 1e-15
    assert raw[80:88] == b"s" + b"\0" * 7 and raw[88:96] == b"Msat" + b"\0" * 4
    assert raw[96:104] == b"A/m" + b"\0" * 5 and struct.unpack("<Q", raw[104:112])[0] == 4
    body = raw[:112 + 4 * 72]
    assert np.array_equal(np.frombuffer(raw[112:112 + 288], dtype="<f4"), a.ravel())
    assert struct.unpack("<Q", raw[400:408])[0] == _crc64_go_iso(body)
    # a second frame is appended; a flipped data byte fails the reader's CRC check
    nat.write_field(p, nat.format_code("dump"), a, n, (1e-9, 2e-9, 3e-9), 2e-15, "Msat", "A/m")
    assert len(p.read_bytes()) == 2 * 408
    bad = bytearray(raw)
    bad[200] ^= 1
    q = tmp_path / "bad.dump"
    q.write_bytes(bytes(bad))
    with pytest.raises(nat.MMError):
        nat.read_field(q)


def test_format_options():
    assert nat.format_code("ovf") == nat.FORMATS["ovf"]
    assert nat.format_code("omf", ["Text"]) == nat.FORMATS["omf_text"]
    with pytest.raises(ValueError):
        nat.format_code("dump", ["text"])
    with pytest.raises(ValueError):
        nat.format_code("ovf", ["binary 8"])
