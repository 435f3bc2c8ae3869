"""FITS images through the library's reader/writer (host only, no GPU needed).

Arrays follow the file's order: element ``[j, i]`` of the returned array is
pixel ``(NAXIS1 index i, NAXIS2 index j)``, i.e. NAXIS1 varies fastest, which
is the column-major layout the reference's matrices use when read with
``readFits`` (common/io/fits.cpp:66-104).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib


def _dims(path: str):
    n1, n2 = C.c_long(), C.c_long()
    check(lib().moao_fits_read_f64(path.encode(), C.byref(n1), C.byref(n2), None, 0), "fits dims")
    return int(n1.value), int(n2.value)


def read_fits(path: str, dtype=np.float64) -> np.ndarray:
    """Image as an (NAXIS2, NAXIS1) array of float64 or int64."""
    n1, n2 = _dims(path)
    out = np.empty((n2, n1), dtype=np.int64 if np.dtype(dtype) == np.int64 else np.float64)
    a1, a2 = C.c_long(), C.c_long()
    f = lib().moao_fits_read_i64 if out.dtype == np.int64 else lib().moao_fits_read_f64
    check(f(path.encode(), C.byref(a1), C.byref(a2), out.ctypes.data, out.size), "read_fits")
    return out


def write_fits(path: str, data) -> None:
    """Writes a 1-D or 2-D array (float64 as BITPIX -64, int64 as BITPIX 64);
    a 2-D array's last axis becomes NAXIS1."""
    a = np.asarray(data)
    if a.ndim == 1:
        a = a[None, :]
    if a.ndim != 2:
        raise ValueError("write_fits: 1-D or 2-D arrays only")
    if np.issubdtype(a.dtype, np.integer):
        a = np.ascontiguousarray(a, dtype=np.int64)
        check(lib().moao_fits_write_i64(path.encode(), a.shape[1], a.shape[0], a.ctypes.data),
              "write_fits")
    else:
        a = np.ascontiguousarray(a, dtype=np.float64)
        check(lib().moao_fits_write_f64(path.encode(), a.shape[1], a.shape[0], a.ctypes.data),
              "write_fits")
