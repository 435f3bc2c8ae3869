"""Systems used by the tests, written in the reference's parameter-file format."""
import os
import tempfile

import numpy as np

from moao_b200 import params as P

_CACHE = {}


def check_system(nlayer: int):
    """The reference's smallest check system (datafile/check/nx456_nLayers{2,10}_wfs6_Nssp10:
    39 m, obs 0.2, 3 LGS + 3 NGS + truth sensor, 10x10, lgs_cst 1), rebuilt from its
    published values; the 10-layer profile is the 2-layer one's strengths split evenly
    over 10 altitudes (the reference's own 10-layer file is not reproduced)."""
    s = P.SysParams(diam=39.0, obs=0.2, tFrame=0.004, nW=7, nLgs=3, nTarget=1, nssp=10)
    s.gsAlt = [1e-05] * 3 + [0.0] * 4
    s.gsType = [2, 2, 2, 1, 1, 1, 1]
    s.alphaX_as = [23.0, -11.5, -11.5, -16.0, -32.0, 52.0, 0.0]
    s.alphaY_as = [0.0, 19.9186, -19.9186, -36.0, 38.0, -5.0, 0.0]
    s.XPup = [0.0] * 7; s.YPup = [0.0] * 7; s.thetaML = [0.0] * 7; s.thetaCam = [0.0] * 7
    s.sensibilite = [1.0] * 7
    s.tracking = [0.0, 0.0, 0.0]
    s.ncpu = 12
    s.mrNGS = [13.0] * 4
    s.lgsFlux = 6e7
    s.lgsCst = 1.0
    s.lgsDepth = 5000.0
    if nlayer == 2:
        a = P.AtmParams(nLayer=2, r0=0.128916, cn2=[28.5115, 1.88506], h=[30.0, 12500.0], L0=[25.0, 25.0])
    else:
        h = np.linspace(30.0, 15000.0, nlayer)
        cn2 = np.full(nlayer, (28.5115 + 1.88506) / nlayer)
        a = P.AtmParams(nLayer=nlayer, r0=0.128916, cn2=cn2.tolist(), h=h.tolist(), L0=[25.0] * nlayer)
    return s, a


SYSTEMS = {
    "small": lambda: P.config_small(),
    "check2": lambda: check_system(2),
    "check10": lambda: check_system(10),
    "elt16": lambda: P.config_scaled(16, 10),
    "elt24": lambda: P.config_scaled(24, 35),
}


def system_dir(name: str) -> str:
    """Directory with sys-params.txt and prof-1-atmos-night0.txt for a system."""
    if name not in _CACHE:
        d = os.path.join(tempfile.gettempdir(), f"moao_b200_sys_{os.getpid()}_{name}")
        s, a = SYSTEMS[name]()
        P.write_system(d, s, a)
        _CACHE[name] = d
    return _CACHE[name]


def files(name: str):
    d = system_dir(name)
    return os.path.join(d, "sys-params.txt"), os.path.join(d, "prof-1-atmos-night0.txt")
