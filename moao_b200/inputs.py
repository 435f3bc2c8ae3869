"""Inputs of the intersample stage and the actuator projection Dx.

The reference ships these as FITS files produced by its Python tooling
(cython/pipeline). They are synthesised here with the same formulas:

* ``make_dm``        deformable-mirror actuator grid   cython/pipeline/commande.py:57-79
* ``make_idx``       Cvv -> covariance-map index       cython/pipeline/generate_file.py:57-76
* ``fourier_space``  FFT support, pixel size, pitch    cython/pipeline/intersample.pyx:3-39
* ``make_abs2fi``    |FT(influence function)|^2        cython/pipeline/generate_file.py:79-86
                     influence function                cython/pipeline/commande.py:160-174
* ``otf_telescope``  telescope OTF (pupil autocorr.)   cython/pipeline/intersample.pyx:151-200

``Dx`` is a seeded N(0, 1) matrix of shape nact x nmeasts (column-major), the
synthetic command matrix the benchmark configurations specify.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class DM:
    nactu: int
    ndiam: int
    x0: float
    csX: np.ndarray
    csY: np.ndarray
    csI: np.ndarray


def make_dm(nssp: int, couplage: float = 0.2, obs: float = 0.2) -> DM:
    x = np.tile(np.linspace(-1, 1, nssp + 1), (nssp + 1, 1))
    y = x.T.copy()
    r = np.sqrt(x * x + y * y).flatten()
    nn = np.where((r < (1.0 + 1.4 / nssp)) & (r > (obs - 1.0 / nssp)))[0]
    x0 = math.sqrt(-2 / math.log(couplage)) / nssp
    return DM(nactu=nn.size, ndiam=nssp + 1, x0=x0, csX=x.flatten()[nn], csY=y.flatten()[nn], csI=nn)


def make_idx(dm: DM) -> np.ndarray:
    """1-based index of every Cvv element (column-major flat) in the
    (2 Ndiam - 1)^2 covariance map."""
    Np = dm.ndiam
    xx = np.tile(np.arange(Np), (Np, 1)).flatten("C")[dm.csI]
    xx = -np.tile(xx, (xx.size, 1))
    dx = xx - xx.T
    yy = np.tile(np.arange(Np), (Np, 1)).flatten("F")[dm.csI]
    yy = -np.tile(yy, (yy.size, 1))
    dy = yy - yy.T
    dx += Np
    dy += Np
    return (dx.flatten("F") + (Np * 2 - 1) * (dy.flatten("F") - 1)).astype(np.int64)


@dataclass
class Fourier:
    N: int
    ud: float
    dactupix: int


def fourier_space(nactu_diam: int, dtel: float) -> Fourier:
    dactu = dtel / (nactu_diam - 1)
    N = max(8 * 2 ** int(np.log2(nactu_diam) + 0.5), 512)
    ud = 3 * dtel / float(N)
    km = int(dactu / ud + 1)
    return Fourier(N=N, ud=dactu / km, dactupix=km)


def influence(x, y, x0):
    return 1.e-6 * np.exp(-(x * x + y * y) / (2 * x0 * x0))


def make_abs2fi(N: int, ud: float, dtel: float, x0: float) -> np.ndarray:
    """N x N array, C-ordered as the reference reads it (flat index j*N + i)."""
    y = np.tile((np.arange(N) + 1 - (N // 2 + 1)) * ud / (dtel / 2.), (N, 1)).T
    x = y.T.copy()
    fi = influence(x, y, x0)
    return np.abs(np.fft.fft2(fi.T)) ** 2


def otf_telescope(N: int, ud: float, dtel: float, obs: float) -> np.ndarray:
    x = ud / (dtel / 2.) * (np.arange(N) + 1 - (N // 2 + 1))
    x2 = np.tile(x * x, (x.size, 1))
    r = np.sqrt(x2 + x2.T)
    pup = ((r <= 1.0) * 1 * (r > obs) * 1).astype(np.float64)
    surface_pix = dtel ** 2 * (1 - obs ** 2) * np.pi / 4. / ud ** 2
    b = np.abs(np.fft.fft2(pup))
    b = np.fft.ifft2(b * b).real
    return (b / surface_pix ** 2).T.copy()


def make_dx(nact: int, nmeasts: int, seed: int = 1234) -> np.ndarray:
    """Seeded N(0,1) actuator projection, nact x nmeasts, Fortran order."""
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((nact, nmeasts)))


@dataclass
class IntersampleInputs:
    dm: DM
    fourier: Fourier
    idx: np.ndarray
    abs2fi: np.ndarray
    otf: np.ndarray
    np_: int

    @property
    def nact(self) -> int:
        return self.dm.nactu


def intersample_inputs(nssp_ts: int, dtel: float, obs: float, couplage: float = 0.2) -> IntersampleInputs:
    dm = make_dm(nssp_ts, couplage, obs)
    fo = fourier_space(dm.ndiam, dtel)
    return IntersampleInputs(dm=dm, fourier=fo, idx=make_idx(dm),
                             abs2fi=make_abs2fi(fo.N, fo.ud, dtel, dm.x0),
                             otf=otf_telescope(fo.N, fo.ud, dtel, obs), np_=nssp_ts + 1)
