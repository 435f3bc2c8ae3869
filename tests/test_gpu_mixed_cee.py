"""Mixed-precision error covariances and PSF against the FP64 oracle (GPU).

The mixed path (moao_cee_cvv_prec with MOAO_PREC_MIXED) evaluates
Cee = Ctt - R Ctm^T - E R^T with the residual E = Ctm - R Cmm, the three
products on the int8 tensor cores (Ozaki splitting), and Cvv = Dx Cee Dx^T in
FP64. The oracle is the reference's nine-step FP64 chain (oracle.cee_cvv,
lapack/compute/cee_cvv.cpp:50-125) and the intersample PSF restatement
(oracle.intersample, common/tomo_struct/intersample.cpp:74-170).

Stated tolerances (relative Frobenius against the oracle; Strehl ratio = PSF
peak over the peak of the telescope-only PSF, Cvv = 0; Cvv scaled by the one
factor that puts the FP64 Strehl at 0.5, because a seeded N(0, 1) Dx, the
configurations' synthetic command matrix, gives phase variances whose PSF is all
halo, Strehl ~1e-5, where a Strehl difference says nothing):
* chain arithmetic alone (oracle R in both):   Cee, Cvv <= 2e-8 ||Ctt|| / ||Cee||
* end to end from the mixed reconstructor:     R <= 1e-5, Cee, Cvv <= 1e-6,
                                               |delta Strehl| <= 1e-6
Cee does not move to first order with an error in R (d Cee / d R = 0 at the
exact R), so the mixed R's 1e-6..1e-5 error enters Cee only squared. The
chain's own error comes from R Cmm: five int8 slices keep ~2^-28 of the
product's scale (~2^-35 per slice set, less the bits lost to each row's
dynamic range), which reaches Cee through E R^T; measured 3e-8 of Cee on the
ELT-geometry systems and 2e-7 on the 8 m one (whose Cee is 50x smaller than Ctt).
When MOAO_PARITY_REPORT names a file, the measured errors are appended to it.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
import systems
import moao_b200 as M
from moao_b200 import inputs as I

pytestmark = pytest.mark.gpu


def report(**kw):
    path = os.environ.get("MOAO_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(kw) + "\n")


def dev(A):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(A, dtype=np.float64).T)).cuda()


def host(t):
    return t.cpu().numpy().T.copy(order="F")


def strehl(psf, psf0):
    return float(np.max(psf) / np.max(psf0))


def strehl_scale(Cvv, x, target=0.5):
    """The factor c for which the PSF of c Cvv has the given Strehl ratio
    (bisection in log c; the Strehl ratio falls as the phase variance grows)."""
    psf0 = O.intersample(np.zeros_like(Cvv), x.idx, x.abs2fi, x.otf, x.np_)
    lo, hi = -40.0, 10.0
    for _ in range(48):
        mid = 0.5 * (lo + hi)
        s = strehl(O.intersample(10.0 ** mid * Cvv, x.idx, x.abs2fi, x.otf, x.np_), psf0)
        lo, hi = (mid, hi) if s > target else (lo, mid)
    return 10.0 ** (0.5 * (lo + hi)), psf0


def inputs(name):
    sf, af = systems.files(name)
    t = M.Tomo(sf, af)
    g = O.Geometry.from_tomo(t)
    nm, nts = g.nmeas, g.nmeasts
    t.setTarget(0)
    Cmm = O.matcov(g, nm, nm, 0, 0, 1, nthreads=8)
    Ctm = O.matcov(g, nts, nm, 0, 0, 3, nthreads=8)
    Ctt = O.matcov(g, nts, nts, 0, 0, 4, nthreads=8)
    x = I.intersample_inputs(t.info.nssp_ts, t.info.diam, t.info.obs)
    return t, nm, nts, Cmm, Ctm, Ctt, x


def run_chain(ctx, nm, nts, nact, Cmm, Ctt, Ctm, R, Dx, prec):
    import torch
    d = {k: dev(v) for k, v in dict(Cmm=Cmm, Cpp=Ctt, Cpm=Ctm, R=R, Dx=Dx).items()}
    Cee = torch.zeros((nts, nts), dtype=torch.float64, device="cuda")
    Cvv = torch.zeros((nact, nact), dtype=torch.float64, device="cuda")
    Tmp = torch.zeros((nts, nact), dtype=torch.float64, device="cuda")
    M.Cee_Cvv(nm, nts, nact, d["Cmm"], nm, d["Cpp"], nts, d["Cpm"], nts, d["R"], nts, d["Dx"],
              nact, Cee, nts, Cvv, nact, Tmp, nact, prec=prec, ctx=ctx)
    ctx.synchronize()
    return host(Cee), host(Cvv), host(Tmp), host(d["Cpm"]), host(d["Cpp"])


@pytest.mark.parametrize("name", ["small", "elt16", "elt24"])
def test_mixed_cee_cvv_psf_against_fp64_oracle(ctx, name):
    t, nm, nts, Cmm, Ctm, Ctt, x = inputs(name)
    nact = x.nact
    Dx = I.make_dx(nact, nts, seed=5)
    _, R_ref, info = O.reconstructor(Cmm, Ctm)
    assert info == 0
    Cee_ref, Cvv_ref, _, Cpm_ref, _ = O.cee_cvv(Cmm, Ctt, Ctm, R_ref, Dx)
    scale = np.linalg.norm(Ctt) / np.linalg.norm(Cee_ref)
    ctx.set_offsets_from_tomo(t)
    ctx.set_mixed()
    try:
        # (1) the mixed chain on the oracle's R: its own arithmetic error
        Cee, Cvv, Tmp, Cpm, Cpp = run_chain(ctx, nm, nts, nact, Cmm, Ctt, Ctm, R_ref, Dx, "mixed")
        e_cee1, e_cvv1 = O.rel_fro(Cee, Cee_ref), O.rel_fro(Cvv, Cvv_ref)
        assert e_cee1 <= 2e-8 * scale and e_cvv1 <= 2e-8 * scale, (e_cee1, e_cvv1, scale)
        # Cpm = Ctm - E carries E's error: ~2^-28 of the product's scale
        assert O.rel_fro(Cpm, Cpm_ref) <= 1e-7, "Cpm must end as R Cmm"
        assert np.array_equal(Cpp, Ctt), "the mixed path leaves Cpp as given"
        assert O.rel_fro(Tmp, Dx @ (np.tril(Cee) + np.tril(Cee, -1).T)) <= 1e-12
        # (2) end to end: mixed reconstructor, then the mixed chain
        dC, dT = dev(Cmm), dev(Ctm)
        M.reconstructor(nm, nts, dC, nm, dT, nts, 1, prec="mixed", ctx=ctx)
        R_mx = host(dT)
        e_r = O.rel_fro(R_mx, R_ref)
        Cee2, Cvv2, *_ = run_chain(ctx, nm, nts, nact, Cmm, Ctt, Ctm, R_mx, Dx, "mixed")
    finally:
        ctx.set_offsets([], [], [])
    e_cee, e_cvv = O.rel_fro(Cee2, Cee_ref), O.rel_fro(Cvv2, Cvv_ref)
    # (3) PSF and Strehl ratio on the truth direction
    c, psf0 = strehl_scale(Cvv_ref, x)
    isx = M.Intersample(nact * nact, x.np_, t.info.diam, x.idx, x.abs2fi, x.otf, ctx=ctx)
    psf_mx = isx.process((c * Cvv2).copy(order="F"))
    isx.close()
    psf_ref = O.intersample(c * Cvv_ref, x.idx, x.abs2fi, x.otf, x.np_)
    s_ref, s_mx = strehl(psf_ref, psf0), strehl(psf_mx, psf0)
    report(test="mixed_cee_cvv", system=name, nmeas=nm, nmeasts=nts, nact=nact,
           chain_only_Cee=e_cee1, chain_only_Cvv=e_cvv1, chain_bound=2e-8 * scale,
           R=e_r, Cee=e_cee, Cvv=e_cvv, strehl_fp64=s_ref, strehl_mixed=s_mx,
           strehl_delta=abs(s_mx - s_ref), cvv_scale_for_strehl_half=c)
    assert e_r <= 1e-5, e_r
    assert e_cee <= 1e-6 and e_cvv <= 1e-6, (e_cee, e_cvv)
    assert abs(s_ref - 0.5) < 1e-3
    assert abs(s_mx - s_ref) <= 1e-6, (s_mx, s_ref)


def test_mixed_cee_cvv_padded_and_empty(ctx):
    """Leading dimensions above the sizes, and nact = 0 (Cee only)."""
    import torch
    t, nm, nts, Cmm, Ctm, Ctt, x = inputs("small")
    _, R_ref, _ = O.reconstructor(Cmm, Ctm)
    nact = 37
    Dx = I.make_dx(nact, nts, seed=9)
    Cee_ref, Cvv_ref, *_ = O.cee_cvv(Cmm, Ctt, Ctm, R_ref, Dx)
    scale = np.linalg.norm(Ctt) / np.linalg.norm(Cee_ref)

    def pad(A, extra):
        P = np.full((A.shape[0] + extra, A.shape[1]), 3.0)
        P[:A.shape[0]] = A
        return dev(P)
    p = 5
    ctx.set_offsets_from_tomo(t)
    d = dict(Cmm=pad(Cmm, p), Cpp=pad(Ctt, p), Cpm=pad(Ctm, p), R=pad(R_ref, p), Dx=pad(Dx, p))
    Cee = torch.zeros((nts, nts + p), dtype=torch.float64, device="cuda")
    Cvv = torch.zeros((nact, nact + p), dtype=torch.float64, device="cuda")
    Tmp = torch.zeros((nts, nact + p), dtype=torch.float64, device="cuda")
    try:
        M.Cee_Cvv(nm, nts, nact, d["Cmm"], nm + p, d["Cpp"], nts + p, d["Cpm"], nts + p, d["R"],
                  nts + p, d["Dx"], nact + p, Cee, nts + p, Cvv, nact + p, Tmp, nact + p,
                  prec="mixed", ctx=ctx)
        ctx.synchronize()
        Cee0 = torch.zeros((nts, nts), dtype=torch.float64, device="cuda")
        one = torch.zeros(1, dtype=torch.float64, device="cuda")
        M.Cee_Cvv(nm, nts, 0, dev(Cmm), nm, dev(Ctt), nts, dev(Ctm), nts, dev(R_ref), nts, one, 1,
                  Cee0, nts, one, 1, one, 1, prec="mixed", ctx=ctx)
        ctx.synchronize()
    finally:
        ctx.set_offsets([], [], [])
    assert O.rel_fro(host(Cee)[:nts], Cee_ref) <= 2e-8 * scale
    assert O.rel_fro(host(Cvv)[:nact], Cvv_ref) <= 2e-8 * scale
    assert np.all(host(d["Cpm"])[nts:] == 3.0), "wrote into Cpm's padding"
    # nact = 0: Cee only
    assert O.rel_fro(host(Cee0), Cee_ref) <= 2e-8 * scale
