"""Host-side logic and the C-ABI boundary (CPU only, no compute calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle as O
import systems
import moao_b200 as M
from moao_b200 import params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
TABLES = ["u", "v", "X", "Y", "sspSizeL", "L0diff", "cn2", "Nsubap", "Nssp", "noiseNGS",
          "noiseLGSxx", "noiseLGSyy", "noiseLGSxy", "alphaX", "alphaY", "lgsExt", "lgsTheta", "mr"]


def _declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names |= set(re.findall(r"\b(moao_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol(built):
    lib = C.CDLL(M.LIB_PATH)
    missing = [n for n in sorted(_declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing
    assert len(_declared_symbols()) >= 27


@pytest.mark.parametrize("name", ["small", "check2", "check10"])
def test_geometry_matches_reference_golden(built, name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    t = M.Tomo(*systems.files(name))
    for k in TABLES:
        assert np.array_equal(t.table(k), z[k]), k
    nW, nLgs, nL, Nx, nm, nts = z["info"]
    assert (t.info.nW, t.info.nLgs, t.info.nLayer, t.info.Nx) == (nW, nLgs, nL, Nx)
    assert (t.getNMeas(), t.getNMeasTS()) == (nm, nts)


@pytest.mark.skipif(not O.RefTomo.available(), reason="reference library not built here")
@pytest.mark.parametrize("name", ["elt16", "check10"])
def test_geometry_bit_identical_to_reference_after_updates(built, name, tmp_path):
    sf, af = systems.files(name)
    ref, mine = O.RefTomo(sf, af), M.Tomo(sf, af)
    s, a = systems.SYSTEMS[name]()
    a.h = [x * 1.3 for x in a.h]
    a.L0 = [30.0 + i for i in range(a.nLayer)]
    af2 = str(tmp_path / "prof0-atmos-night0.txt")
    P.write_atm(a, af2)
    ref.updateAtm(af2)
    mine.updateAtm(af2)
    ref.setTarget(0)
    mine.setTarget(0)
    for k in TABLES:
        assert np.array_equal(ref.table(k), mine.table(k)), k


def test_sys_file_round_trip(tmp_path):
    s, a = P.config_elt()
    P.write_system(str(tmp_path), s, a)
    t = M.Tomo(str(tmp_path / "sys-params.txt"), str(tmp_path / "prof-1-atmos-night0.txt"))
    i = t.info
    assert (i.nW, i.nLgs, i.nLayer) == (9, 6, 35)
    assert (t.getNMeas(), t.getNMeasTS()) == (47552, 5944)
    assert np.allclose(t.table("cn2"), a.cn2, rtol=0, atol=0)


def test_bad_parameter_files_raise(tmp_path):
    with pytest.raises(M.MoaoError) as e:
        M.Tomo(str(tmp_path / "nope.txt"), str(tmp_path / "nope2.txt"))
    assert e.value.name == "MOAO_ERR_IO"
    s, a = P.config_small()
    s.alphaX_as = s.alphaX_as[:2]  # vector too short
    P.write_system(str(tmp_path), s, a)
    with pytest.raises(M.MoaoError):
        M.Tomo(str(tmp_path / "sys-params.txt"), str(tmp_path / "prof-1-atmos-night0.txt"))


def test_profile_validation(built):
    t = M.Tomo(*systems.files("small"))
    with pytest.raises(M.MoaoError):
        t.set_profile([1.0], [0.0], [0.0])  # L0 must be > 0
    with pytest.raises(M.MoaoError):
        t.setTarget(5)


def test_status_strings(built):
    lib = M.lib()
    assert lib.moao_status_string(2) == b"MOAO_ERR_NOT_SPD"
    assert lib.moao_status_string(99) == b"MOAO_ERR_UNKNOWN"


def test_configs_have_the_stated_sizes():
    for fn, nm, nts, nl in ((P.config_small, 640, 160, 3), (P.config_elt, 47552, 5944, 35)):
        s, a = fn()
        assert a.nLayer == nl
        assert abs(sum(np.array(a.cn2)) * a.r0 ** (5 / 3) - 1) < 1e-12
    rng = np.random.default_rng(0)
    for _ in range(20):
        s, a = P.config_random(rng)
        assert 20 <= s.nssp <= 50 and 3 <= s.nW <= 9 and 1 <= a.nLayer <= 20


@pytest.mark.parametrize("name", systems.CHECK_SETS + ["elt"])
def test_check_set_geometry_matches_reference_golden(built, name):
    """The six reference check systems (parsed from the reference's own
    parameter files) and the ELT-scale system: every geometry table equals the
    reference's Tomo_struct on the original files (small tables whole, large
    ones through seeded samples, sums and norms)."""
    z = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    t = M.Tomo(*systems.files(name))
    for k in ["sspSizeL", "L0diff", "cn2", "Nsubap", "Nssp", "noiseNGS", "alphaX", "alphaY",
              "lgsExt", "lgsTheta", "mr"]:
        assert np.array_equal(t.table(k), z[k]), k
    for k in ["u", "v", "X", "Y", "noiseLGSxx", "noiseLGSyy", "noiseLGSxy"]:
        v = t.table(k)
        assert v.size == int(z[f"{k}_n"]), k
        assert np.array_equal(v[z[f"{k}_idx"]], z[f"{k}_val"]), k
        assert v.sum() == float(z[f"{k}_sum"]) and np.linalg.norm(v) == float(z[f"{k}_fro"]), k
    nW, nLgs, nL, Nx, nm, nts = z["info"]
    assert (t.info.nW, t.info.nLgs, t.info.nLayer, t.info.Nx) == (nW, nLgs, nL, Nx)
    assert (t.getNMeas(), t.getNMeasTS()) == (nm, nts)
