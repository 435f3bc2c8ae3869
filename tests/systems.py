"""Systems used by the tests, written in the reference's parameter-file format."""
import json
import os
import tempfile

import numpy as np

from moao_b200 import params as P

_CACHE = {}


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CHECK_SETS = ["nx456_nLayers2_wfs6_Nssp10", "nx456_nLayers10_wfs6_Nssp10",
              "nx5120_nLayers2_wfs8_Nssp29", "nx5120_nLayers10_wfs8_Nssp29",
              "nx10112_nLayers2_wfs8_Nssp41", "nx10112_nLayers10_wfs8_Nssp41"]


def check_set(name: str):
    """One of the six systems of the reference's datafile/check directory, as
    parsed from its own sys-params.txt and prof-1-atmos-night0.txt into
    tests/golden/check_sets.json (tests/golden/make_check_sets.py)."""
    with open(os.path.join(GOLDEN, "check_sets.json")) as f:
        d = json.load(f)[name]
    return P.SysParams(**d["sys"]), P.AtmParams(**d["atm"])


SYSTEMS = {
    "small": lambda: P.config_small(),
    # the reference's smallest check sets (39 m, 3 LGS + 3 NGS + truth sensor, 10x10)
    "check2": lambda: check_set("nx456_nLayers2_wfs6_Nssp10"),
    "check10": lambda: check_set("nx456_nLayers10_wfs6_Nssp10"),
    "elt16": lambda: P.config_scaled(16, 10),
    "elt24": lambda: P.config_scaled(24, 35),
    "elt": lambda: P.config_elt(),
}
SYSTEMS.update({n: (lambda n=n: check_set(n)) for n in CHECK_SETS})


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
