"""System and atmosphere parameter sets in the reference's positional text format.

The reference reads ``sys-params.txt`` and ``prof*-atmos-night*.txt`` positionally:
every value line is preceded by one comment line (``SysParams::getParams``,
common/tomo_struct/sysParams.cpp:166-204; ``AtmParams::getParams``,
common/tomo_struct/atmParams.cpp:93-102; ``readIO``, common/io/IO.cpp.in:64).
Vectors are whitespace-separated on a single line.  This module writes files in
that layout (so the same files feed the reference and this library) and builds
the synthetic systems used by the tests and the benchmark:

* ``config_small``   - 8 m telescope, 3 LGS + 1 NGS + truth sensor, 10x10
                        subapertures, 3 layers (nmeas 640, nmeasts 160).
* ``config_elt``     - 39 m telescope, 6 LGS + 2 NGS + truth sensor, 64x64
                        subapertures, 35 layers (nmeas 47,552, nmeasts 5,944).
* ``config_random``  - the uneven batched instances (20..50 subapertures across,
                        2..8 WFS, 1..20 layers, Dirichlet Cn2 fractions).

Values not fixed by those descriptions take the reference's own defaults from the
``SysParams(d, nNGS, nLGS, ...)`` constructor (common/tomo_struct/sysParams.cpp:53-104).
Layer strengths follow the reference's convention that ``cn2`` is used directly as
an r0^(-5/3) weight (common/kernels/matcov_kernels.cpp:296), so a profile with Cn2
fractions f_l and Fried parameter r0 is written as ``cn2_l = f_l * r0**(-5/3)``.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field, asdict
from typing import List

import numpy as np


@dataclass
class SysParams:
    """Field order and meaning of common/tomo_struct/sysParams.hpp:11-47."""
    diam: float = 8.0
    obs: float = 0.2
    tFrame: float = 0.004
    nW: int = 5
    nLgs: int = 3
    nTarget: int = 1
    nssp: int = 10
    gsAlt: List[float] = field(default_factory=list)
    gsType: List[int] = field(default_factory=list)
    alphaX_as: List[float] = field(default_factory=list)
    alphaY_as: List[float] = field(default_factory=list)
    XPup: List[float] = field(default_factory=list)
    YPup: List[float] = field(default_factory=list)
    thetaML: List[float] = field(default_factory=list)
    thetaCam: List[float] = field(default_factory=list)
    sensibilite: List[float] = field(default_factory=list)
    tracking: List[float] = field(default_factory=lambda: [1.0, 1.0, 1.0])
    pasDphi: float = 0.0001
    ncpu: int = 1
    mrNGS: List[float] = field(default_factory=list)
    lgsFlux: float = 1.0e7
    ngsPixSize: float = 0.3
    lgsPixSize: float = 1.0
    lambdaNGS: float = 6.5e-07
    lambdaLGS: float = 5.89e-07
    bdw_m: float = 3.3e-07
    throughNGS: float = 0.425
    throughLGS: float = 0.382
    throughAtm: float = 0.84
    RON: int = 3
    lgsCst: float = 0.1
    spotWidth: float = 1.0
    lgsAlt: float = 100000.0
    lgsDepth: float = 50000.0
    targetX_as: List[float] = field(default_factory=lambda: [0.0])
    targetY_as: List[float] = field(default_factory=lambda: [0.0])

    @property
    def nNgs(self) -> int:
        return self.nW - self.nLgs - 1


@dataclass
class AtmParams:
    """Field order of common/tomo_struct/atmParams.hpp:10-14."""
    nLayer: int = 1
    r0: float = 0.15
    cn2: List[float] = field(default_factory=list)
    h: List[float] = field(default_factory=list)
    L0: List[float] = field(default_factory=list)


_SYS_COMMENTS = [
    ("diam", "diam       : meter     : Telescope diameter"),
    ("obs", "obs        : percent   : Central obscuration"),
    ("tFrame", "tFrame     : second    : frame rate"),
    ("nW", "nW         :           : number of WFS"),
    ("nLgs", "nLgs       :           : number of LGS"),
    ("nTarget", "nTarget    :           : number of Target"),
    ("nssp", "Nssp       :           : number of subaperture per wfs along the diameter"),
    ("gsAlt", "gsAlt      : meter^-1  : inverse of lazer altitude"),
    ("gsType", "type       :           : guide star type (1:NGS, 2:LGS)"),
    ("alphaX_as", "alphaX_as  : arcsec    : pointing direction of the wfs on x axis"),
    ("alphaY_as", "alphaY_as  : arcsec    : pointing direction of the wfs on y axis"),
    ("XPup", "XPup       : meter     : pupil shift of the WFS"),
    ("YPup", "YPup       : meter     : pupil shift of the WFS"),
    ("thetaML", "thetaML    :           : rotation of the microlenses"),
    ("thetaCam", "thetaCam   :           : rotation of the camera"),
    ("sensibilite", "sensibility:           : sensitivity coeff of this WFS"),
    ("tracking", "tracking   : arcsec^2  : telescope tracking error parameters (x^2, y^2 and xy)"),
    ("pasDphi", "pasDPHI    :           : Precision of DPHI precomputation. //deprecated"),
    ("ncpu", "ncpu       :           : Number of CPU used (only with openMP)"),
    ("mrNGS", "mrNGS      :           : magnitude of NGS"),
    ("lgsFlux", "lgsFlux    : (ph/m2/s) : LGS photon return at M1"),
    ("ngsPixSize", "ngsPixSize : arcsec    : NGS pixel size"),
    ("lgsPixSize", "lgsPixSize : arcsec    : LGS pixel size"),
    ("lambdaNGS", "lambdaNGS  : meter     : wave length for NGS"),
    ("lambdaLGS", "lambdaLGS  : meter     : wave length for LGS"),
    ("bdw_m", "bdw_m      : meter     : bandwidth"),
    ("throughNGS", "throughNGS : percent   : transmission for NGS"),
    ("throughLGS", "throughLGS : percent   : transmission for LGS"),
    ("throughAtm", "throughAtm : percent   : atmosphere transmission"),
    ("RON", "RON        : nb of e-  : Read Out Noise"),
    ("lgsCst", "lgsCst     :           : constant on lgs (simulate that LGS cannot measure tip-tilt and focus)"),
    ("spotWidth", "spotWidth  : arcsec    : lazer width"),
    ("lgsAlt", "lgsAlt     : meter     : sodium layer altitude"),
    ("lgsDepth", "lgsDepth   : meter     : depth of the sodium layer"),
    ("targetX_as", "targetX_as : arcsec    :  taget direction on x axis"),
    ("targetY_as", "targetY_as : arcsec    :  taget direction on y axis"),
]

_ATM_COMMENTS = [
    ("nLayer", "nLayer :       : number of turbulent layers"),
    ("r0", "r0     :       : global fried parameter"),
    ("cn2", "cn2    :       : layer strength r0^(-5/3)"),
    ("h", "h      : meter : layer altitude"),
    ("L0", "L0     : meter : outer scale"),
]


def _fmt(v) -> str:
    if isinstance(v, (list, tuple, np.ndarray)):
        return " ".join(_fmt(x) for x in v)
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return repr(float(v))


def write_sys(p: SysParams, path: str) -> None:
    with open(path, "w") as f:
        for key, comment in _SYS_COMMENTS:
            f.write(comment + "\n" + _fmt(getattr(p, key)) + "\n")


def write_atm(a: AtmParams, path: str) -> None:
    with open(path, "w") as f:
        for key, comment in _ATM_COMMENTS:
            f.write(comment + "\n" + _fmt(getattr(a, key)) + "\n")


def write_system(directory: str, sysp: SysParams, atm: AtmParams,
                 profile_names=("prof-1-atmos-night0.txt", "prof0-atmos-night0.txt")) -> str:
    """Write sys-params.txt plus the atmosphere profile(s) the drivers read.

    The lapack driver opens ``prof{snap*snapPerNight+obs}-atmos-night{night}.txt``
    (lapack/moao_lapack.cpp:54,102,140); the first refine step reads ``prof-1``.
    """
    os.makedirs(directory, exist_ok=True)
    write_sys(sysp, os.path.join(directory, "sys-params.txt"))
    for n in profile_names:
        write_atm(atm, os.path.join(directory, n))
    return directory


LEGACY_FIELDS = ["diam", "obs", "nW", "Nssp", "gsAlt", "type", "nLgs", "alphaX_as", "alphaY_as",
                 "XPup", "YPup", "thetaML", "thetaCam", "sensibilite", "tracking", "pasDphi", "ncpu",
                 "lgs_cst", "noise_var", "spot_width", "lgs_alt", "lgs_depth"]


def write_legacy_sys(values, path: str) -> None:
    """A sys-params.txt in the legacy benchmark layout (the 22 fields of
    LEGACY_FIELDS in that order, one comment line before each value line), as
    in the reference's datafile/benchmark directory."""
    if len(values) != len(LEGACY_FIELDS):
        raise ValueError("legacy layout: 22 value lines")
    ints = {"nW", "Nssp", "type", "nLgs", "ncpu"}
    vectors = {"gsAlt", "type", "alphaX_as", "alphaY_as", "XPup", "YPup", "thetaML", "thetaCam",
               "sensibilite", "tracking"}
    with open(path, "w") as f:
        for name, v in zip(LEGACY_FIELDS, values):
            v = [int(x) if name in ints else float(x) for x in v]
            f.write(name + "\n" + _fmt(v if name in vectors else v[0]) + "\n")


def _ring(n: int, radius: float):
    a = 2.0 * math.pi / n
    return ([radius * math.cos(i * a) for i in range(n)],
            [radius * math.sin(i * a) for i in range(n)])


def make_sys(diam: float, obs: float, nssp: int, nlgs: int, nngs: int,
             lgs_radius_as: float, rng: np.random.Generator,
             ngs_min_as: float = None, ngs_max_as: float = None) -> SysParams:
    """A system with LGS on a ring, seeded NGS positions and an on-axis truth sensor.

    NGS positions are drawn uniformly in an annulus between ``ngs_min_as`` and
    ``ngs_max_as`` (defaults: half the LGS radius to the LGS radius, like the
    reference's ``fillVectorRand`` use in sysParams.cpp:101-103).
    """
    nW = nlgs + nngs + 1
    p = SysParams(diam=diam, obs=obs, nW=nW, nLgs=nlgs, nssp=nssp)
    p.gsAlt = [1.0 / p.lgsAlt] * nlgs + [0.0] * (nngs + 1)
    p.gsType = [2] * nlgs + [1] * (nngs + 1)
    ax, ay = _ring(nlgs, lgs_radius_as) if nlgs else ([], [])
    lo = lgs_radius_as / 2.0 if ngs_min_as is None else ngs_min_as
    hi = lgs_radius_as if ngs_max_as is None else ngs_max_as
    for _ in range(nngs):
        r = rng.uniform(lo, hi)
        t = rng.uniform(0.0, 2.0 * math.pi)
        ax.append(r * math.cos(t))
        ay.append(r * math.sin(t))
    ax.append(0.0)
    ay.append(0.0)
    p.alphaX_as, p.alphaY_as = ax, ay
    p.XPup = [0.0] * nW
    p.YPup = [0.0] * nW
    p.thetaML = [0.0] * nW
    p.thetaCam = [0.0] * nW
    p.sensibilite = [1.0] * nW
    p.mrNGS = [13.0] * (nngs + 1)
    return p


def make_atm(h, fractions, r0: float, L0) -> AtmParams:
    f = np.asarray(fractions, dtype=np.float64)
    cn2 = (f * r0 ** (-5.0 / 3.0)).tolist()
    L0 = [float(L0)] * len(h) if np.isscalar(L0) else [float(x) for x in L0]
    return AtmParams(nLayer=len(h), r0=float(r0), cn2=cn2, h=[float(x) for x in h], L0=L0)


def config_small(seed: int = 1234):
    """8 m, obs 0.14, 10x10, 3 LGS on a 10 arcsec ring + 1 NGS + on-axis truth
    sensor; layers at 0/4/10 km with fractions 0.6/0.3/0.1, r0 0.15 m, L0 25 m."""
    rng = np.random.default_rng(seed)
    s = make_sys(8.0, 0.14, 10, 3, 1, 10.0, rng)
    a = make_atm([0.0, 4000.0, 10000.0], [0.6, 0.3, 0.1], 0.15, 25.0)
    return s, a


def config_elt(seed: int = 1234, nlayer: int = 35):
    """39 m, obs 0.28, 64x64, 6 LGS on a 7.5 arcmin ring (radius 225 arcsec) +
    2 NGS + on-axis truth sensor; 35 layers on 0..20 km with fractions
    exp(-h/5 km) x LogNormal(0, 0.2), normalised; r0 0.129 m, L0 25 m."""
    rng = np.random.default_rng(seed)
    s = make_sys(39.0, 0.28, 64, 6, 2, 225.0, rng)
    h = np.linspace(0.0, 20000.0, nlayer)
    f = np.exp(-h / 5000.0) * rng.lognormal(0.0, 0.2, nlayer)
    f /= f.sum()
    a = make_atm(h, f, 0.129, 25.0)
    return s, a


def config_scaled(nssp: int, nlayer: int, seed: int = 1234, nlgs: int = 6, nngs: int = 2,
                  diam: float = 39.0, obs: float = 0.28):
    """The ELT system at a reduced subaperture count (same geometry rules)."""
    rng = np.random.default_rng(seed)
    s = make_sys(diam, obs, nssp, nlgs, nngs, 225.0 * diam / 39.0, rng)
    h = np.linspace(0.0, 20000.0, nlayer)
    f = np.exp(-h / 5000.0) * rng.lognormal(0.0, 0.2, nlayer)
    f /= f.sum()
    return s, make_atm(h, f, 0.129, 25.0)


def config_random(rng: np.random.Generator, nssp_range=(20, 50), nwfs_range=(2, 8),
                  nlayer_range=(1, 20)):
    """One uneven instance: Nssp, WFS count and layer count drawn uniformly, layer
    altitudes U(0, 20 km), Dirichlet(1) Cn2 fractions, r0 ~ U(0.08, 0.2) m,
    L0 ~ U(10, 50) m (one L0 per layer)."""
    nssp = int(rng.integers(nssp_range[0], nssp_range[1] + 1))
    nwfs = int(rng.integers(nwfs_range[0], nwfs_range[1] + 1))
    nlgs = int(rng.integers(0, nwfs + 1))
    nngs = nwfs - nlgs
    diam = float(nssp) * 0.5
    s = make_sys(diam, 0.2, nssp, nlgs, nngs, 60.0, rng)
    nl = int(rng.integers(nlayer_range[0], nlayer_range[1] + 1))
    h = np.sort(rng.uniform(0.0, 20000.0, nl))
    f = rng.dirichlet(np.ones(nl))
    r0 = float(rng.uniform(0.08, 0.2))
    L0 = rng.uniform(10.0, 50.0, nl)
    return s, make_atm(h, f, r0, L0)


def as_dict(p) -> dict:
    return asdict(p)
