"""FP64 parity on the reference's own check systems and at ELT size (GPU).

* Covariance tiles of the six datafile/check systems of the reference and of the
  ELT-scale system (nmeas 47,552): the full matrices are generated on the GPU as
  the benchmark generates them (types 1, 3 and 4 through the shared-point,
  offset-table and per-pair kernels) and 48x48 tiles are compared with the
  reference's own tiles (tests/golden/ref_*.npz): per tile, max |gpu - ref| <=
  1e-11 max |C| (C the whole matrix) and relative Frobenius <= 1e-8. The
  per-tile relative bound is loose on purpose: far-apart subaperture pairs give
  tiles ~1e-3 of the matrix maximum whose 4-point stencils cancel, so ulp-level
  differences of the structure function (evaluated in a different order here)
  reach ~1e-10 of such a tile; relative to the matrix they stay near 1e-12.
* FP64 reconstructor, Cee and Cvv on every check system against the oracle
  (LAPACK in the reference's call order, lapack/compute/reconstructor.cpp:32-58
  and cee_cvv.cpp:50-125) on the same GPU-generated Cmm, Ctm and Ctt: R and L
  within max(1e-10, 50 kappa eps), kappa = cond2(Cmm) estimated by power and
  inverse iteration; Cee and Cvv (from the oracle's R, so that the chain alone
  is tested) within 200 sqrt(nmeas) eps ||Ctt|| / ||Cee||: the chain's dot
  products of length nmeas carry ~sqrt(nmeas) eps of the terms' scale ||Ctt||,
  and Cee is their difference, smaller by ||Ctt|| / ||Cee||.
When MOAO_PARITY_REPORT names a file, every measured error is appended to it as
one JSON line.
"""
import json
import os

import numpy as np
import pytest
import scipy.linalg as sla

import oracle as O
import systems
import moao_b200 as M
from moao_b200 import inputs as I

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def report(**kw):
    path = os.environ.get("MOAO_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(kw) + "\n")


def host(t):
    return t.cpu().numpy().T.copy(order="F")


def errors(got, want):
    scale = np.max(np.abs(want))
    return float(np.max(np.abs(got - want)) / scale), float(O.rel_fro(got, want))


def generate(ctx, t, typ, nr, nc):
    """Full nr x nc matrix of one type on the GPU (column-major, zero-initialised)."""
    import torch
    d = torch.zeros((nc, nr), dtype=torch.float64, device="cuda")
    M.matcov_tile(d, nr, nc, 0, 0, nr, t, typ, ctx=ctx)
    ctx.synchronize()
    return d


@pytest.mark.parametrize("name", systems.CHECK_SETS + ["elt"])
def test_covariance_tiles_match_reference(ctx, name):
    import torch
    z = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    t = M.Tomo(*systems.files(name))
    nm, nts = t.getNMeas(), t.getNMeasTS()
    t.setTarget(0)
    spec, vals = z["tile_spec"], z["tile_vals"]
    nt = vals.shape[1]
    worst = [0.0, 0.0, 0.0]
    for typ, nr, nc in ((1, nm, nm), (3, nts, nm), (4, nts, nts)):
        d = generate(ctx, t, typ, nr, nc)
        dmax = float(d.abs().max())
        for (ty, r0, c0), want in zip(spec, vals):
            if ty != typ:
                continue
            got = d[c0:c0 + nt, r0:r0 + nt].cpu().numpy().T
            mx, rf = errors(got, want)
            mm = float(np.max(np.abs(got - want))) / dmax
            assert mm <= 1e-11 and rf <= 1e-8, (name, typ, r0, c0, mm, mx, rf)
            worst = [max(worst[0], mx), max(worst[1], rf), max(worst[2], mm)]
        del d
        torch.cuda.empty_cache()
    report(test="covariance_tiles", system=name, nmeas=nm, nmeasts=nts, tiles=int(len(spec)),
           max_rel=worst[0], rel_fro=worst[1], max_rel_to_matrix_max=worst[2], bound_matrix=1e-11, bound_tile_fro=1e-8)


def kappa2(S, L, iters=60):
    """cond2 of the SPD matrix S (lower Cholesky factor L): power iteration for
    the largest eigenvalue, inverse iteration through L for the smallest."""
    rng = np.random.default_rng(0)
    x = rng.standard_normal(S.shape[0])
    for _ in range(iters):
        x = S @ x
        x /= np.linalg.norm(x)
    lmax = float(x @ (S @ x))
    y = rng.standard_normal(S.shape[0])
    for _ in range(iters):
        y = sla.solve_triangular(L, sla.solve_triangular(L, y, lower=True), lower=True, trans=1)
        y /= np.linalg.norm(y)
    lmin = float(y @ (S @ y))
    return lmax / lmin


@pytest.mark.parametrize("name", systems.CHECK_SETS)
def test_fp64_chain_on_check_sets(ctx, name):
    import torch
    t = M.Tomo(*systems.files(name))
    nm, nts = t.getNMeas(), t.getNMeasTS()
    Cmm_d = generate(ctx, t, 1, nm, nm)
    t.setTarget(0)
    Ctm_d = generate(ctx, t, 3, nts, nm)
    Ctt_d = generate(ctx, t, 4, nts, nts)
    Cmm, Ctm, Ctt = host(Cmm_d), host(Ctm_d), host(Ctt_d)
    # oracle: LAPACK in the reference's call order
    L_ref, R_ref, info = O.reconstructor(Cmm, Ctm)
    assert info == 0
    S = np.tril(Cmm) + np.tril(Cmm, -1).T
    kappa = kappa2(S, np.tril(L_ref))
    del S
    tol = max(1e-10, 50 * kappa * EPS)
    # GPU FP64 path (panel 1024, the default)
    C2, T2 = Cmm_d.clone(), Ctm_d.clone()
    rep = M.reconstructor(nm, nts, C2, nm, T2, nts, 1, ctx=ctx)
    assert rep["info"] == 0
    R_mx, R_rf = errors(host(T2), R_ref)
    L_mx, L_rf = errors(np.tril(host(C2)), np.tril(L_ref))
    del C2, T2
    assert R_rf <= tol and R_mx <= tol, (name, R_mx, R_rf, tol)
    assert L_rf <= tol and L_mx <= tol, (name, L_mx, L_rf, tol)
    # Cee / Cvv from the oracle's R
    nact = I.make_dm(t.info.nssp_ts, 0.2, t.info.obs).nactu
    Dx = I.make_dx(nact, nts, seed=11)
    Cee_ref, Cvv_ref, *_ = O.cee_cvv(Cmm, Ctt, Ctm, R_ref, Dx)
    dev = lambda A: torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    R_d, Dx_d = dev(R_ref), dev(Dx)
    Cee = torch.zeros((nts, nts), dtype=torch.float64, device="cuda")
    Cvv = torch.zeros((nact, nact), dtype=torch.float64, device="cuda")
    Tmp = torch.zeros((nts, nact), dtype=torch.float64, device="cuda")
    M.Cee_Cvv(nm, nts, nact, Cmm_d, nm, Ctt_d, nts, Ctm_d, nts, R_d, nts, Dx_d, nact, Cee, nts,
              Cvv, nact, Tmp, nact, ctx=ctx)
    ctx.synchronize()
    ctol = 200 * np.sqrt(nm) * EPS * np.linalg.norm(Ctt) / np.linalg.norm(Cee_ref)
    Cee_mx, Cee_rf = errors(host(Cee), Cee_ref)
    Cvv_mx, Cvv_rf = errors(host(Cvv), Cvv_ref)
    report(test="fp64_chain", system=name, nmeas=nm, nmeasts=nts, nact=nact, kappa=kappa,
           R_max_rel=R_mx, R_rel_fro=R_rf, L_max_rel=L_mx, L_rel_fro=L_rf, R_bound=tol,
           Cee_max_rel=Cee_mx, Cee_rel_fro=Cee_rf, Cvv_max_rel=Cvv_mx, Cvv_rel_fro=Cvv_rf,
           CeeCvv_bound=ctol)
    assert Cee_rf <= ctol and Cee_mx <= ctol, (name, Cee_mx, Cee_rf, ctol)
    assert Cvv_rf <= ctol and Cvv_mx <= ctol, (name, Cvv_mx, Cvv_rf, ctol)
