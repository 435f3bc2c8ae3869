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


@pytest.mark.parametrize("name", ["nx5120_wfs8_Nssp29", "nx10112_wfs8_Nssp41"])
def test_legacy_benchmark_sys_file(built, name, tmp_path):
    """A system file in the reference's legacy benchmark layout
    (datafile/benchmark/*/sys-params.txt, tests/golden/legacy_sets.json) is
    detected and read: its geometry equals the same system written in the
    current layout, and its noise tables follow the legacy model (noise_var on
    every NGS slope; across / along each LGS spot noise_var and
    noise_var (ext^2 + w^2) / w^2)."""
    import json
    vals = json.load(open(os.path.join(GOLDEN, "legacy_sets.json")))[name]
    f = dict(zip(P.LEGACY_FIELDS, vals))
    sf = str(tmp_path / "legacy-sys-params.txt")
    P.write_legacy_sys(vals, sf)
    _, a = P.config_small()
    af = str(tmp_path / "prof-1-atmos-night0.txt")
    P.write_atm(a, af)
    t = M.Tomo(sf, af)
    nW, nLgs, nssp = int(f["nW"][0]), int(f["nLgs"][0]), int(f["Nssp"][0])
    assert (t.info.nW, t.info.nLgs, t.info.nLayer) == (nW, nLgs, a.nLayer)
    assert np.all(t.table("Nssp") == nssp)
    # the same system in the current layout (photometric fields at their defaults)
    s = P.SysParams(diam=f["diam"][0], obs=f["obs"][0], nW=nW, nLgs=nLgs, nTarget=1, nssp=nssp,
                    gsAlt=f["gsAlt"], gsType=[int(x) for x in f["type"]], alphaX_as=f["alphaX_as"],
                    alphaY_as=f["alphaY_as"], XPup=f["XPup"], YPup=f["YPup"], thetaML=f["thetaML"],
                    thetaCam=f["thetaCam"], sensibilite=f["sensibilite"], tracking=f["tracking"],
                    pasDphi=f["pasDphi"][0], ncpu=int(f["ncpu"][0]), mrNGS=[0.0] * (nW - nLgs),
                    lgsCst=f["lgs_cst"][0], spotWidth=f["spot_width"][0], lgsAlt=f["lgs_alt"][0],
                    lgsDepth=f["lgs_depth"][0])
    sf2 = str(tmp_path / "sys-params.txt")
    P.write_sys(s, sf2)
    t2 = M.Tomo(sf2, af)
    for k in ["u", "v", "X", "Y", "sspSizeL", "Nsubap", "lgsExt", "lgsTheta"]:
        assert np.array_equal(t.table(k), t2.table(k)), k
    assert t.getNMeas() == t2.getNMeas() and t.info.lgsCst == f["lgs_cst"][0]
    v, w2 = f["noise_var"][0], f["spot_width"][0] ** 2
    ext, th = t.table("lgsExt"), t.table("lgsTheta")
    nl = int(np.sum(t.table("Nsubap")[:nLgs]))
    L = v * (ext[:nl] ** 2 + w2) / w2
    c, sn = np.cos(th[:nl]), np.sin(th[:nl])
    assert np.allclose(t.table("noiseLGSxx")[:nl], L * c * c + v * sn * sn, rtol=1e-14, atol=0)
    assert np.allclose(t.table("noiseLGSyy")[:nl], L * sn * sn + v * c * c, rtol=1e-14, atol=0)
    assert np.allclose(t.table("noiseLGSxy")[:nl], (L - v) * sn * c, rtol=1e-13, atol=1e-18)
    assert np.all(t.table("noiseNGS") == v)
    # a current-layout file still takes the photometric model
    assert not np.all(t2.table("noiseNGS") == v)


def test_legacy_file_with_short_vectors_is_rejected(built, tmp_path):
    """The eight wfs9 legacy files declare 10 WFS but list 9 guide-star
    altitudes and types: rejected with MOAO_ERR_IO naming the short vector."""
    import json
    vals = json.load(open(os.path.join(GOLDEN, "legacy_sets.json")))["nx50184_wfs9_Nssp86"]
    sf = str(tmp_path / "sys-params.txt")
    P.write_legacy_sys(vals, sf)
    _, a = P.config_small()
    af = str(tmp_path / "prof-1-atmos-night0.txt")
    P.write_atm(a, af)
    with pytest.raises(M.MoaoError) as e:
        M.Tomo(sf, af)
    assert e.value.name == "MOAO_ERR_IO" and "gsAlt" in str(e.value)


@pytest.mark.parametrize("nssp,diam,obs", [(10, 8.0, 0.14), (29, 39.0, 0.2), (64, 39.0, 0.28)])
def test_dm_and_idx_synthesis_matches_tooling(built, nssp, diam, obs):
    """moao_intersample_inputs (C++, no Python tooling) gives the actuator count,
    FFT support and idx of the reference tooling's formulas (restated in
    moao_b200.inputs) exactly; host-only, no GPU."""
    from moao_b200 import inputs as I
    na, N, idx, _, _ = M.intersample_inputs(nssp, diam, obs, tables=False)
    x = I.intersample_inputs(nssp, diam, obs)
    assert na == x.nact and N == x.fourier.N
    assert np.array_equal(idx, x.idx)
