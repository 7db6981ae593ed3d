"""CSR snapshot files: foreign, missing and truncated files are refused with
G500_E_IO before anything reaches the device."""
import struct

import pytest


def test_missing_file_is_refused(g500, tmp_path):
    with pytest.raises(g500.G500Error) as e:
        g500.Graph2DCSR.load(str(tmp_path / "nope.g500"))
    assert e.value.code == g500.G500_E_IO


def test_foreign_file_is_refused(g500, tmp_path):
    p = tmp_path / "junk.g500"
    p.write_bytes(b"not a snapshot" * 100)
    with pytest.raises(g500.G500Error) as e:
        g500.Graph2DCSR.load(str(p))
    assert e.value.code == g500.G500_E_IO and b"not a graph snapshot" in g500.lib().g500_last_error()


def test_inconsistent_header_is_refused(g500, tmp_path):
    # right magic and version, lengths that do not match the scalars
    hdr = b"G500CSR1" + struct.pack("<Iiii", 2, 2, 20, 1) + struct.pack("<8q", 16, 65536, 65536, 10, 100, 9, 0, 0)
    hdr += struct.pack("<2d", 0.0, 0.0) + struct.pack("<9Q", *([1] * 9))
    p = tmp_path / "bad.g500"
    p.write_bytes(hdr)
    with pytest.raises(g500.G500Error) as e:
        g500.Graph2DCSR.load(str(p))
    assert e.value.code == g500.G500_E_IO and b"inconsistent" in g500.lib().g500_last_error()
