"""FITS image I/O (host only): round trips, an independently written file with
BZERO/BSCALE scaling, 1-D images, and error reporting."""
import struct

import numpy as np
import pytest

import moao_b200 as M
from moao_b200.fits import read_fits, write_fits


def test_round_trip_float64(tmp_path):
    a = np.random.default_rng(0).standard_normal((13, 7))
    p = str(tmp_path / "a.fits")
    write_fits(p, a)
    b = read_fits(p)
    assert b.shape == (13, 7) and np.array_equal(a, b)
    raw = open(p, "rb").read()
    assert len(raw) % 2880 == 0
    assert raw[:80].startswith(b"SIMPLE  =")
    assert b"NAXIS1  =                    7" in raw[:2880]


def test_round_trip_int64_exact(tmp_path):
    a = (np.arange(-20, 22, dtype=np.int64) * 987654321987).reshape(6, 7)
    p = str(tmp_path / "i.fits")
    write_fits(p, a)
    assert np.array_equal(read_fits(p, np.int64), a)


def _card(text):
    return text.ljust(80).encode()


def test_reads_scaled_int16_written_independently(tmp_path):
    """A file built here card by card (BITPIX 16, BZERO 32768, BSCALE 0.5, 1-D)."""
    vals = np.array([-32768, -1, 0, 1, 32767], dtype=">i2")
    hdr = b"".join([_card("SIMPLE  =                    T"), _card("BITPIX  =                   16"),
                    _card("NAXIS   =                    1"), _card("NAXIS1  =                    5"),
                    _card("BZERO   =              32768.0 / offset"),
                    _card("BSCALE  =                  0.5"), _card("END")])
    hdr += b" " * (2880 - len(hdr))
    data = vals.tobytes()
    data += b"\0" * (2880 - len(data))
    p = tmp_path / "s.fits"
    p.write_bytes(hdr + data)
    got = read_fits(str(p))
    assert got.shape == (1, 5)
    np.testing.assert_array_equal(got[0], 32768.0 + 0.5 * vals.astype(np.float64))


def test_reads_float32_big_endian(tmp_path):
    vals = np.array([[1.5, -2.25], [3.0, 1e-3]], dtype=">f4")
    hdr = b"".join([_card("SIMPLE  =                    T"), _card("BITPIX  =                  -32"),
                    _card("NAXIS   =                    2"), _card("NAXIS1  =                    2"),
                    _card("NAXIS2  =                    2"), _card("END")])
    hdr += b" " * (2880 - len(hdr))
    p = tmp_path / "f.fits"
    p.write_bytes(hdr + vals.tobytes() + b"\0" * (2880 - 16))
    np.testing.assert_array_equal(read_fits(str(p)), vals.astype(np.float64))


def test_errors(tmp_path):
    with pytest.raises(M.MoaoError):
        read_fits(str(tmp_path / "missing.fits"))
    bad = tmp_path / "bad.fits"
    bad.write_bytes(b"NOT A FITS FILE".ljust(2880))
    with pytest.raises(M.MoaoError):
        read_fits(str(bad))
    short = tmp_path / "short.fits"
    write_fits(str(short), np.ones((40, 40)))
    short.write_bytes(short.read_bytes()[:2880 + 100])
    with pytest.raises(M.MoaoError):
        read_fits(str(short))
