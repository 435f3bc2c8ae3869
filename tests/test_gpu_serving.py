"""Serving loop on the GPU: requests of different systems, sizes, profiles and
precisions run concurrently on several slots give the same results as each
request run alone (tolerance: relative max error 1e-12; the kernels are
deterministic, so the results are expected to be identical), and the FP64
result of a request equals the direct API's."""
import numpy as np
import pytest

import systems
import moao_b200 as M
from moao_b200 import inputs as I
from moao_b200 import params as P
from moao_b200.serve import Server

pytestmark = pytest.mark.gpu


def profile(rng, nl):
    f = rng.dirichlet(np.ones(nl))
    r0 = rng.uniform(0.08, 0.2)
    cn2 = f * r0 ** (-5.0 / 3.0)
    return cn2, np.sort(rng.uniform(0, 20000, nl)), rng.uniform(10, 50, nl)


def register(srv, plan):
    out = []
    for name, with_psf in plan:
        sf, af = systems.files(name)
        t = M.Tomo(sf, af)
        nts = t.getNMeasTS()
        if with_psf:
            s, _ = systems.SYSTEMS[name]()
            x = I.intersample_inputs(s.nssp, s.diam, s.obs)
            Dx = I.make_dx(x.nact, nts, seed=5)
            sid = srv.add_system(sf, af, Dx=Dx, idx=x.idx, abs2fi=x.abs2fi, otf=x.otf)
        else:
            sid = srv.add_system(sf, af)
        out.append(sid)
    return out


def requests(rng, sids):
    reqs = []
    for k in range(8):
        sid = sids[k % len(sids)]
        reqs.append(dict(system=sid, prof=profile(rng, int(rng.integers(1, 12))),
                         prec="mixed" if k % 3 == 2 else "fp64"))
    return reqs


def run(srv, reqs, sids_psf):
    outs, ids = [], []
    for q in reqs:
        info = srv.system_info(q["system"])
        R = np.zeros(info["nmeas"] * info["nmeasts"])
        Cvv = np.zeros(info["nact"] ** 2) if info["nact"] else None
        psf = np.zeros(info["psf_n"] ** 2) if info["psf_n"] else None
        ids.append(srv.submit(q["system"], *q["prof"], prec=q["prec"], R=R, Cvv=Cvv, psf=psf))
        outs.append((R, Cvv, psf))
    res = [srv.wait(i) for i in ids]
    for r in res:
        assert r["status"] == 0, r
    return outs, res


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def test_same_alone_and_in_the_mix(built, cuda):
    plan = [("small", True), ("check2", False), ("elt16", False)]
    rng = np.random.default_rng(11)
    with Server(slots=3) as srv:
        sids = register(srv, plan)
        reqs = requests(rng, sids)
        mix, res = run(srv, reqs, sids[:1])
        assert srv.stats()["max_in_flight"] >= 2
    with Server(slots=1) as srv:
        register(srv, plan)
        alone = []
        for q in reqs:
            o, _ = run(srv, [q], sids[:1])
            alone.append(o[0])
    for q, m, a in zip(reqs, mix, alone):
        for x, y in zip(m, a):
            if y is not None:
                assert rel(x, y) <= 1e-12, (q["prec"], rel(x, y))


def test_fp64_request_equals_direct_api(built, ctx):
    sf, af = systems.files("check2")
    rng = np.random.default_rng(3)
    cn2, h, L0 = profile(rng, 4)
    with Server(slots=2) as srv:
        sid = srv.add_system(sf, af)
        info = srv.system_info(sid)
        R = np.zeros(info["nmeas"] * info["nmeasts"])
        assert srv.wait(srv.submit(sid, cn2, h, L0, R=R))["status"] == 0
    t = M.Tomo(sf, af)
    t.set_profile(cn2, h, L0)
    t.setTarget(0)
    nm, nts = t.getNMeas(), t.getNMeasTS()
    C = np.zeros((nm, nm), order="F")
    T = np.zeros((nts, nm), order="F")
    M.matcov_tile(C, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
    M.matcov_tile(T, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
    M.reconstructor(nm, nts, C, nm, T, nts, 1, ctx=ctx)
    assert rel(R.reshape(nm, nts).T, T) <= 1e-12


def test_mixed_request_cvv_and_psf_against_fp64_oracle(built, cuda, ctx, tmp_path):
    """A mixed request's Cvv comes from the refinement's last (R_k, E_k) pair
    (Cee is stationary in R, so the shortcut moves it only to second order); its
    R, Cvv and PSF against the FP64 oracle (oracle.reconstructor / cee_cvv /
    intersample, the reference's steps) for a system registered with
    synthesised PSF tables: R <= 1e-5, Cvv <= 1e-6 relative Frobenius, PSF
    within 1e-6 of its peak."""
    import oracle as O
    sp, ap = P.config_scaled(16, 10)
    d = str(tmp_path / "sys")
    P.write_system(d, sp, ap)
    sf, af = d + "/sys-params.txt", d + "/prof-1-atmos-night0.txt"
    t = M.Tomo(sf, af)
    nm, nts = t.getNMeas(), t.getNMeasTS()
    nact, N, idx, a2, otf = M.intersample_inputs(t.info.nssp_ts, t.info.diam, t.info.obs, ctx=ctx)
    Dx = I.make_dx(nact, nts, seed=7) * 0.2   # Strehl ~0.5 here, not the all-halo regime
    with Server(slots=1, hbm_budget_gb=40.0) as srv:
        sid = srv.add_system_synth(sf, af, Dx)
        R = np.zeros(nm * nts)
        Cvv = np.zeros(nact * nact)
        psf = np.zeros(N * N)
        prof = (np.array(ap.cn2), np.array(ap.h), np.array(ap.L0))
        r = srv.wait(srv.submit(sid, *prof, prec="mixed", R=R, Cvv=Cvv, psf=psf))
        assert r["status"] == 0, r
    g = O.Geometry.from_tomo(t)
    t.setTarget(0)
    Cmm = O.matcov(g, nm, nm, 0, 0, 1, nthreads=8)
    Ctm = O.matcov(g, nts, nm, 0, 0, 3, nthreads=8)
    Ctt = O.matcov(g, nts, nts, 0, 0, 4, nthreads=8)
    _, R_ref, _ = O.reconstructor(Cmm, Ctm)
    _, Cvv_ref, *_ = O.cee_cvv(Cmm, Ctt, Ctm, R_ref, Dx)
    psf_ref = O.intersample(Cvv_ref, idx, a2, otf, t.info.nssp_ts + 1)
    assert O.rel_fro(R.reshape(nts, nm, order="F"), R_ref) <= 1e-5
    assert O.rel_fro(Cvv.reshape(nact, nact, order="F"), Cvv_ref) <= 1e-6
    assert np.max(np.abs(psf.reshape(N, N) - psf_ref)) <= 1e-6 * np.max(np.abs(psf_ref))
