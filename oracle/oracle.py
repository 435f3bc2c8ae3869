"""TEST INFRASTRUCTURE ONLY — the CPU oracle of the reconstructor path.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module, and only as the checker; the product (``moao_b200``) never
does. Pieces:

* ``matcov``          covariance tiles from the plain-C restatement
                      (oracle/moao_oracle.c, pinned bit-for-bit against the
                      reference's own common/ code compiled in oracle/_ref).
* ``RefTomo``         the reference's Tomo_struct + matcov_tile themselves
                      (oracle/_ref/libmoao_ref.so, built from the reference's
                      sources by oracle/Makefile) when that library exists.
* ``reconstructor``   lapack/compute/reconstructor.cpp:32-58 with LAPACK/BLAS
                      (scipy's OpenBLAS): dpotrf('L'); dtrsm(R,L,T,N);
                      dtrsm(R,L,N,N).
* ``cee_cvv``         lapack/compute/cee_cvv.cpp:50-125, the nine BLAS/LAPACK
                      steps in order (dsyr2k, dsymm, laset, lacpy, geadd,
                      scal, dgemm, dsymm, dgemm).
* ``intersample``     common/tomo_struct/intersample.cpp:74-170 in numpy; the
                      unnormalised FFTW r2c/c2r become numpy FFTs times N^2.
* ``compare_matrices`` common/compute/check_utils.cpp:20-58.
* ``RefDense``        the reference's own MOAO_LAPACK::reconstructor / Cee_Cvv and
                      intersample_prepare/_init/_process/_free, compiled
                      unchanged (oracle/_ref/libmoao_ref_dense.so) against
                      oracle/shim/: CBLAS/LAPACKE from scipy's OpenBLAS, FFTW's
                      2-D real transforms and cfitsio's image reads supplied by
                      oracle/ref_dense_shim.cpp. tests/test_oracle.py pins
                      ``reconstructor``, ``cee_cvv`` and ``intersample`` to it.

The reference tree has no golden vectors for the LAPACK and PSF steps (its
golden FITS files are not distributed with it); those steps are pinned by
running the reference's own code (RefDense) on the same inputs.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.linalg.blas as blas
import scipy.linalg.lapack as lapack

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libmoao_ref.so")
REF_DENSE_LIB = os.path.join(HERE, "_ref", "libmoao_ref_dense.so")

_TABLES = ["Nsubap", "Nssp", "u", "v", "sspSizeL", "L0diff", "cn2", "X", "Y", "noiseNGS",
           "noiseLGSxx", "noiseLGSyy", "noiseLGSxy"]


class _Geom(C.Structure):
    _fields_ = ([("nW", C.c_int), ("nLgs", C.c_int), ("nLayer", C.c_int), ("Nx", C.c_int)] +
                [(n, C.c_void_p) for n in ["Nsubap", "Nssp", "u", "v", "sspSizeL", "L0", "cn2", "X",
                                           "Y", "noiseNGS", "noiseLGSxx", "noiseLGSyy",
                                           "noiseLGSxy"]] +
                [("lgsCst", C.c_double), ("diam", C.c_double)])


_olib = None


def oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_LIB):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(ORACLE_LIB)
        L.oracle_matcov_tile.argtypes = [C.c_void_p] + [C.c_int] * 5 + [C.c_void_p, C.c_int]
        L.oracle_matcov_tile_mt.argtypes = [C.c_void_p] + [C.c_int] * 5 + [C.c_void_p, C.c_int, C.c_int]
        L.oracle_dphi.argtypes = [C.c_double] * 3
        L.oracle_dphi.restype = C.c_double
        _olib = L
    return _olib


class Geometry:
    """Geometry tables of one system, from any object with ``table(name)``
    (moao_b200.Tomo or RefTomo) plus nW, nLgs, nLayer, Nx, lgsCst, diam."""

    def __init__(self, tables: dict, nW: int, nLgs: int, nLayer: int, Nx: int, lgsCst: float,
                 diam: float):
        self.t = {k: np.ascontiguousarray(v, dtype=np.int64 if k in ("Nsubap", "Nssp") else np.float64)
                  for k, v in tables.items()}
        self.nW, self.nLgs, self.nLayer, self.Nx = nW, nLgs, nLayer, Nx
        self.lgsCst, self.diam = lgsCst, diam
        t = self.t
        self._g = _Geom(nW, nLgs, nLayer, Nx, *[t[k].ctypes.data for k in _TABLES], lgsCst, diam)
        self.nmeas = int(2 * (Nx - t["Nsubap"][nW - 1]))
        self.nmeasts = int(2 * t["Nsubap"][nW - 1])

    @classmethod
    def from_tomo(cls, tomo) -> "Geometry":
        info = tomo.info
        tables = {k: tomo.table(k) for k in _TABLES}
        return cls(tables, info.nW, info.nLgs, info.nLayer, info.Nx, info.lgsCst, info.diam)


def matcov(geom: Geometry, nrows: int, ncols: int, xoffset: int, yoffset: int, type_mat: int,
           out: np.ndarray | None = None, nthreads: int = 1) -> np.ndarray:
    if out is None:
        out = np.zeros((nrows, ncols), order="F")
    assert out.flags.f_contiguous and out.dtype == np.float64
    r = oracle_lib().oracle_matcov_tile_mt(out.ctypes.data, nrows, ncols, xoffset, yoffset, nrows,
                                           C.byref(geom._g), type_mat, nthreads)
    if r:
        raise ValueError(f"unrecognized type_mat {type_mat}")
    return out


def dphi(x: float, y: float, L0: float) -> float:
    return oracle_lib().oracle_dphi(x, y, L0)


# ---------------------------------------------------------------- reference itself
class _RefInfo:
    pass


class RefTomo:
    """The reference's own Tomo_struct<double> and matcov_tile (oracle/_ref)."""
    _lib = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REF_LIB)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = C.CDLL(REF_LIB)
            L.ref_tomo_create.restype = C.c_void_p
            L.ref_tomo_create.argtypes = [C.c_char_p, C.c_char_p]
            L.ref_tomo_destroy.argtypes = [C.c_void_p]
            L.ref_tomo_update_atm.argtypes = [C.c_void_p, C.c_char_p]
            L.ref_tomo_set_target.argtypes = [C.c_void_p, C.c_int]
            L.ref_tomo_info.argtypes = [C.c_void_p, C.c_void_p]
            L.ref_tomo_table.restype = C.c_long
            L.ref_tomo_table.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_long]
            L.ref_matcov_tile.argtypes = [C.c_void_p, C.c_void_p] + [C.c_int] * 6
            L.ref_matcov_tiled_mt.argtypes = [C.c_void_p, C.c_void_p] + [C.c_int] * 6
            cls._lib = L
        return cls._lib

    def __init__(self, sys_file: str, atm_file: str):
        self.h = self.lib().ref_tomo_create(os.fsencode(sys_file), os.fsencode(atm_file))
        if not self.h:
            raise IOError("reference Tomo_struct construction failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().ref_tomo_destroy(self.h)
            self.h = None

    def updateAtm(self, atm_file):
        if self.lib().ref_tomo_update_atm(self.h, os.fsencode(atm_file)):
            raise IOError(atm_file)

    def setTarget(self, i):
        self.lib().ref_tomo_set_target(self.h, i)

    @property
    def info(self):
        a = (C.c_long * 8)()
        self.lib().ref_tomo_info(self.h, a)
        i = _RefInfo()
        i.nW, i.nLgs, i.nNgs, i.nLayer, i.Nx, i.nmeas, i.nmeasts, i.nTarget = [int(x) for x in a]
        s = self.table("scalars")
        i.diam, i.lgsCst = float(s[0]), float(s[1])
        return i

    def table(self, name: str) -> np.ndarray:
        n = self.lib().ref_tomo_table(self.h, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        self.lib().ref_tomo_table(self.h, name.encode(), out.ctypes.data, n)
        if name == "L0diff":
            out = out[: self.info.nLayer]
        return out

    def matcov_tile(self, data: np.ndarray, nrows, ncols, xoffset, yoffset, lda, type_mat):
        self.lib().ref_matcov_tile(self.h, data.ctypes.data, nrows, ncols, xoffset, yoffset, lda,
                                   type_mat)

    def matcov_full(self, nrows, ncols, type_mat, nthreads=1, ts=128) -> np.ndarray:
        out = np.zeros((nrows, ncols), order="F")
        self.lib().ref_matcov_tiled_mt(self.h, out.ctypes.data, nrows, ncols, nrows, type_mat, ts,
                                       nthreads)
        return out


# ---------------------------------------------------------------- reference dense code
class RefDense:
    """The reference's lapack/compute and intersample code (oracle/_ref)."""
    _lib = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REF_DENSE_LIB)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = C.CDLL(REF_DENSE_LIB)
            L.ref_reconstructor.argtypes = [C.c_long, C.c_long, C.c_void_p, C.c_long, C.c_void_p,
                                            C.c_long, C.c_long]
            L.ref_cee_cvv.argtypes = [C.c_long] * 3 + [C.c_void_p, C.c_long] * 8
            L.ref_intersample.argtypes = [C.c_long, C.c_long, C.c_double, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_long, C.c_void_p, C.c_void_p]
            L.ref_intersample.restype = C.c_long
            cls._lib = L
        return cls._lib

    @classmethod
    def reconstructor(cls, Cmm, Ctm):
        """(L, R): the reference's in-place potrf + two trsm on copies."""
        L = np.array(Cmm, dtype=np.float64, order="F", copy=True)
        R = np.array(Ctm, dtype=np.float64, order="F", copy=True)
        nm, nts = L.shape[0], R.shape[0]
        cls.lib().ref_reconstructor(nm, nts, L.ctypes.data, nm, R.ctypes.data, nts, 1)
        return L, R

    @classmethod
    def cee_cvv(cls, Cmm, Ctt, Ctm, R, Dx):
        """(Cee, Cvv, Cpp_after, Cpm_after, Tmp) from the reference's nine steps
        (leading dimensions equal to the sizes, as the reference assumes)."""
        f = lambda A: np.array(A, dtype=np.float64, order="F", copy=True)
        Cmm, Cpp, Cpm, R, Dx = f(Cmm), f(Ctt), f(Ctm), f(R), f(Dx)
        nm, nts, nact = Cmm.shape[0], Cpp.shape[0], Dx.shape[0]
        Cee = np.zeros((nts, nts), order="F")
        Cvv = np.zeros((nact, nact), order="F")
        Tmp = np.zeros((nact, nts), order="F")
        args = []
        for A, ld in ((Cmm, nm), (Cpp, nts), (Cpm, nts), (R, nts), (Dx, nact), (Cee, nts),
                      (Cvv, nact), (Tmp, nact)):
            args += [A.ctypes.data, ld]
        cls.lib().ref_cee_cvv(nm, nts, nact, *args)
        return Cee, Cvv, Cpp, Cpm, Tmp

    @classmethod
    def intersample(cls, Cvv, idx, abs2fi, otf, np_, Dtel):
        """PSF (N x N, flat C order like isample->dphi) from the reference's code."""
        N = int(max(512, 8 * 2 ** int(np.log(np_) + 0.5)))
        c = np.ascontiguousarray(np.asarray(Cvv, dtype=np.float64).flatten("F"))
        ix = np.ascontiguousarray(idx, dtype=np.int64)
        a = np.ascontiguousarray(np.asarray(abs2fi, dtype=np.float64).reshape(-1))
        o = np.ascontiguousarray(np.asarray(otf, dtype=np.float64).reshape(-1))
        assert a.size == N * N and o.size == N * N and ix.size == c.size
        out = np.zeros(N * N)
        got = cls.lib().ref_intersample(ix.size, np_, Dtel, ix.ctypes.data, a.ctypes.data,
                                        o.ctypes.data, N, c.ctypes.data, out.ctypes.data)
        if got != N:
            raise ValueError("intersample: N differs from the tables' size")
        return out.reshape(N, N)


# ---------------------------------------------------------------- LAPACK steps
def reconstructor(Cmm: np.ndarray, Ctm: np.ndarray):
    """Returns (L, R, info): dpotrf('L', Cmm) then the two right-side dtrsm.
    Cmm and Ctm are not modified."""
    L, info = lapack.dpotrf(np.asfortranarray(Cmm), lower=1, clean=0)
    if info != 0:
        return L, None, info
    X = blas.dtrsm(1.0, L, np.asfortranarray(Ctm), side=1, lower=1, trans_a=1, diag=0)
    R = blas.dtrsm(1.0, L, X, side=1, lower=1, trans_a=0, diag=0)
    return L, R, 0


def geadd_t_inplace(B: np.ndarray):
    """MOAO_LAPACK::geadd('T', M, N, 1, B, ld, 1, B, ld) with A aliasing B,
    executed in the reference's loop order (lapack/compute/cee_cvv.cpp:144-160)."""
    M, N = B.shape
    for i in range(M):
        for j in range(N):
            B[j, i] = B[i, j] + B[j, i]


def cee_cvv(Cmm, Ctt, Ctm, R, Dx, literal_geadd: bool = False):
    """Returns (Cee, Cvv, Cpp_after, Cpm_after, Tmp) following the reference's
    nine steps. Cmm is read through its lower triangle only."""
    Cpp = np.array(Ctt, order="F", copy=True)
    Cpm = np.asfortranarray(Ctm)
    R = np.asfortranarray(R)
    Cpp = blas.dsyr2k(-1.0, Cpm, R, beta=1.0, c=Cpp, trans=0, lower=1)
    Cpm = blas.dsymm(1.0, np.asfortranarray(Cmm), R, beta=0.0, side=1, lower=1)
    n = Cpp.shape[0]
    Cee = np.zeros((n, n), order="F")
    il = np.tril_indices(n)
    Cee[il] = Cpp[il]                      # laset('U',0,0) then lacpy('L')
    if literal_geadd:
        geadd_t_inplace(Cee)
    else:                                   # same result: lower mirrored, diagonal doubled
        d = np.diag(Cee).copy()
        Cee = Cee + np.tril(Cee, -1).T
        Cee[np.diag_indices(n)] = d + d
    Cee[np.diag_indices(n)] *= 0.5           # scal(diag, 0.5)
    Cee = blas.dgemm(1.0, Cpm, R, beta=1.0, c=np.asfortranarray(Cee), trans_b=1)
    Tmp = blas.dsymm(1.0, Cee, np.asfortranarray(Dx), beta=0.0, side=1, lower=1)
    Cvv = blas.dgemm(1.0, Tmp, np.asfortranarray(Dx), trans_b=1)
    return Cee, Cvv, Cpp, Cpm, Tmp


# ---------------------------------------------------------------- intersample
def intersample(Cvv: np.ndarray, idx: np.ndarray, abs2fi: np.ndarray, otf: np.ndarray, np_: int):
    """PSF (N x N, C-ordered flat like the reference's isample->dphi)."""
    N = int(max(512, 8 * 2 ** int(np.log(np_) + 0.5)))
    dp = N // (3 * (np_ - 1)) + 1
    ncov = 2 * np_ - 1
    nmap = ncov * ncov
    flat = np.asarray(Cvv, dtype=np.float64).flatten("F")
    Map = np.zeros(nmap)
    np.add.at(Map, idx - 1, flat)               # sequential scatter in index order
    div = np.bincount(idx - 1, minlength=nmap).astype(np.float64)
    nz = div > 0
    Map[nz] /= div[nz]
    ncmap = N // 2 + 1
    nelem = (ncov - 1) // 2
    a = ncmap - nelem * dp - 1
    grid = np.zeros((N, N))
    grid[a:a + ncov * dp:dp, a:a + ncov * dp:dp] = Map.reshape(ncov, ncov)
    H = N // 2 + 1
    A2 = np.asarray(abs2fi, dtype=np.float64).reshape(N, N)
    spec = np.fft.rfft2(grid).real * A2.T[:, :H]
    dphi = np.fft.irfft2(spec.astype(np.complex128), s=(N, N)) * (N * N)
    fact = 2 * (2 * 3.14159 / 1.65e-06) ** 2
    fact2 = N * N * float(dp) * float(dp)
    norm = dphi[ncmap - 1, ncmap - 1] / fact2 * fact
    dphi = np.exp(-0.5 * (norm - dphi / fact2 * fact))
    dphi = np.roll(dphi, (N // 2, N // 2), axis=(0, 1))
    O2 = np.asarray(otf, dtype=np.float64).reshape(N, N)
    spec2 = (O2 * dphi).T[:, :H]
    psf = np.fft.irfft2(spec2.astype(np.complex128), s=(N, N)) * (N * N)
    return np.roll(psf, (N // 2, N // 2), axis=(0, 1))


def compare_matrices(A: np.ndarray, B: np.ndarray, uplo: str = "N"):
    """compareMatrices (check_utils.cpp:20-58) with trans='N': max elementwise
    relative error and absolute Frobenius norm (off-diagonal terms doubled for
    a triangle)."""
    A = np.asarray(A)
    B = np.asarray(B)
    if uplo == "L":
        mask = np.tril(np.ones(A.shape, bool), -1)
    elif uplo == "U":
        mask = np.triu(np.ones(A.shape, bool))
    else:
        mask = np.ones(A.shape, bool)
    a, b = A[mask], B[mask]
    with np.errstate(divide="ignore", invalid="ignore"):
        d = np.where(a == 0, -b, 1 - b / np.where(a == 0, 1, a))
    maxerr = float(np.max(np.abs(d))) if d.size else 0.0
    w = np.ones(A.shape)
    if uplo in ("L", "U"):
        w = np.where(np.eye(*A.shape, dtype=bool), 1.0, 2.0)
    fro = float(np.sqrt(np.sum(((B - A) ** 2 * w)[mask])))
    return maxerr, fro


def rel_fro(A, B) -> float:
    """||A - B||_F / ||B||_F."""
    return float(np.linalg.norm(np.asarray(A) - np.asarray(B)) / np.linalg.norm(np.asarray(B)))
