"""EMS slice files (.sli): the product's reader and writer (JMS_Sli*) against
the reference bench driver's header code (prm_slice_file_info) and a golden
file written by it.  Needs no GPU."""
import os

import numpy as np
import pytest

from tests.golden import make_golden_sli as GS

GOLD = GS.OUT


@pytest.fixture(scope="module")
def jb():
    import jmultislicelib_b200 as jb

    jb.lib()
    return jb


def test_reads_reference_written_file(jb):
    h, g = jb.sli_read(GOLD)
    assert (h["nx"], h["ny"], h["nvar"], h["content"]) == (16, 12, 2, 0)
    assert h["version"] == 2020052801 and h["data_offset"] == 8192 and h["swapped"] == 0
    assert h["title"] == GS.PARAMS["title"]
    for k in ("thickness", "ekv", "sx", "sy"):
        assert h[k] == np.float32(GS.PARAMS[k]), k
    np.testing.assert_array_equal(g, GS.gratings())


def test_roundtrip_and_reference_reader(jb, tmp_path):
    rng = np.random.default_rng(3)
    g = (rng.normal(size=(3, 20, 24)) + 1j * rng.normal(size=(3, 20, 24))).astype(np.complex64)
    p = str(tmp_path / "w_001.sli")
    assert jb.sli_write(p, g, 0.2, 200.0, 1.1, 0.9, title="roundtrip") == 0
    h, g2 = jb.sli_read(p)
    np.testing.assert_array_equal(g2, g)
    assert (h["nx"], h["ny"], h["nvar"], h["title"]) == (24, 20, 3, "roundtrip")
    from oracle import ref

    if not ref.available():
        pytest.skip("oracle/_ref not built")
    r = ref.sli_read_header(p)
    assert (r["nx"], r["ny"], r["nvar"], r["content"]) == (24, 20, 3, 0)
    assert r["data_offset"] == 8192 and r["version"] == 2020052801
    assert (r["thickness"], r["ekv"], r["sx"], r["sy"]) == tuple(np.float32(v) for v in (0.2, 200.0, 1.1, 0.9))
    assert r["title"] == "roundtrip"


def test_other_byte_order(jb, tmp_path):
    """A big-endian file (every 4-byte field and datum swapped) reads the same."""
    raw = bytearray(open(GOLD, "rb").read())
    fields = [0x0, 0x4, 0x74, 0x78, 0x80, 0x88, 0x8C, 0x1034, 0x1040, 0x1044, 0x1048]
    for off in fields + list(range(8192, len(raw), 4)):
        raw[off:off + 4] = raw[off:off + 4][::-1]
    p = str(tmp_path / "be_001.sli")
    open(p, "wb").write(bytes(raw))
    h, g = jb.sli_read(p)
    assert h["swapped"] == 1 and (h["nx"], h["ny"], h["nvar"]) == (16, 12, 2)
    assert h["ekv"] == np.float32(300.0)
    np.testing.assert_array_equal(g, GS.gratings())


def test_bad_files(jb, tmp_path):
    import ctypes as C

    h = jb.JMSSliHeader()
    assert jb.lib().JMS_SliReadHeader(os.fsencode(str(tmp_path / "missing.sli")), C.byref(h)) == 2
    p = tmp_path / "short.sli"
    p.write_bytes(b"\x10\x00\x00\x00" * 8)
    assert jb.lib().JMS_SliReadHeader(os.fsencode(str(p)), C.byref(h)) == 3
    q = tmp_path / "trunc.sli"
    q.write_bytes(open(GOLD, "rb").read()[:9000])
    buf = np.zeros(2 * 16 * 12 * 2, np.float32)
    assert jb.lib().JMS_SliReadData(os.fsencode(str(q)), buf.ctypes.data_as(C.POINTER(C.c_float))) == 5
