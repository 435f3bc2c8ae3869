"""Parity of the CUDA path with the oracle (FP64 path), through the C ABI.

Tolerances (stated per check):
* covariance tiles: max |gpu - oracle| <= 1e-11 * max |oracle| and relative
  Frobenius <= 1e-11. The kernel evaluates x^(5/3) as x cbrt(x)^2, sums the
  11-term series in Horner form and factors the per-layer amplitude out of the
  4-point stencils, so it differs from the reference by rounding only; the
  stencils' cancellation amplifies ulp differences to ~1e-13.
* reconstructor, Cee, Cvv: relative Frobenius <= max(1e-10, 50 kappa eps),
  with kappa the measured condition number of Cmm: two correct FP64 Cholesky
  solves with different blockings agree to O(kappa eps), not better.
* PSF: max |gpu - oracle| <= 1e-10 * max |oracle|.
"""
import numpy as np
import pytest

import oracle as O
import systems
import moao_b200 as M
from moao_b200 import inputs as I

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


def dev(A):
    """Column-major numpy matrix -> CUDA tensor holding the same column-major data."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(A, dtype=np.float64).T)).cuda()


def host(t):
    return t.cpu().numpy().T.copy(order="F")


def assert_close(got, want, rel, what):
    scale = np.max(np.abs(want))
    err = np.max(np.abs(got - want))
    assert err <= rel * scale, f"{what}: max err {err / scale:.3e} (relative to max) > {rel}"
    rf = O.rel_fro(got, want)
    assert rf <= rel, f"{what}: relative Frobenius {rf:.3e} > {rel}"


def tomo_and_geom(name):
    sf, af = systems.files(name)
    t = M.Tomo(sf, af)
    return t, O.Geometry.from_tomo(t)


@pytest.mark.parametrize("name", ["small", "check2", "check10", "elt16"])
def test_matcov_full_matrices(ctx, name):
    import torch
    t, g = tomo_and_geom(name)
    nm, nts = g.nmeas, g.nmeasts
    for typ, nr, nc in ((1, nm, nm), (3, nts, nm), (4, nts, nts)):
        want = O.matcov(g, nr, nc, 0, 0, typ, nthreads=8)
        d = torch.zeros((nc, nr), dtype=torch.float64, device="cuda")  # column-major nr x nc
        M.matcov_tile(d, nr, nc, 0, 0, nr, t, typ, ctx=ctx)
        ctx.synchronize()
        got = host(d)
        if typ == 1:
            assert np.all(np.triu(got, 1) == 0), "type 1 wrote above the diagonal"
        assert_close(got, want, 1e-11, f"{name} type {typ}")


def test_matcov_symmetric_fill_and_tiles(ctx):
    import torch
    t, g = tomo_and_geom("check2")
    nm = g.nmeas
    want = O.matcov(g, nm, nm, 0, 0, 1, nthreads=8)
    full = np.tril(want) + np.tril(want, -1).T
    d = torch.zeros((nm, nm), dtype=torch.float64, device="cuda")
    M.matcov_tile(d, nm, nm, 0, 0, nm, t, 5, ctx=ctx)
    ctx.synchronize()
    assert_close(host(d), full, 1e-11, "type 5")
    # tiles at odd offsets through the host-buffer entry point, with untouched
    # elements preserved (the reference only writes the lower triangle)
    for typ, (x0, y0, nr, nc) in [(1, (37, 11, 100, 90)), (1, (200, 250, 64, 96)),
                                  (3, (5, 61, 40, 77)), (4, (3, 9, 50, 31)), (2, (10, 3, 60, 50))]:
        if typ == 2:  # Cmt: rows = WFS, columns = truth sensor == transpose of Ctm
            ctm = O.matcov(g, g.nmeasts, nm, 0, 0, 3, nthreads=8)
            ref = ctm.T[x0:x0 + nr, y0:y0 + nc]
        else:
            ref = O.matcov(g, nr, nc, x0, y0, typ)
        buf = np.full((nr + 3, nc), 7.0, order="F")
        M.matcov_tile(buf, nr, nc, x0, y0, nr + 3, t, typ, ctx=ctx)
        got = buf[:nr]
        if typ == 1:
            gx = np.arange(nr)[:, None] + x0
            gy = np.arange(nc)[None, :] + y0
            assert np.all(got[gy > gx] == 7.0), "untouched upper elements were modified"
            ref = np.where(gy > gx, 7.0, ref)
        assert np.all(buf[nr:] == 7.0), "wrote outside the tile (ld padding)"
        assert_close(got, ref, 1e-11, f"tile type {typ} at {x0},{y0}")


def test_matcov_tiles_through_shared_point_blocks(ctx):
    """Tiles of the ELT-like system that cut through LGS x NGS and truth-sensor x
    LGS blocks, which the shared-point kernel evaluates (edge-aligned WFS pairs
    without an offset table): partial 4x4 / 8x8 cell tiles, the lower-triangle
    mask, ld padding and untouched elements."""
    t, g = tomo_and_geom("elt16")
    nm, nts = g.nmeas, g.nmeasts
    nlgs_rows = 2 * int(sum(g.t["Nsubap"][:g.nLgs]))  # slopes of the LGS
    assert 0 < nlgs_rows < nm
    cases = [(1, (nlgs_rows + 7, 13, 151, 173)),       # NGS rows x LGS columns
             (1, (nlgs_rows - 40, nlgs_rows - 90, 97, 120)),  # across the LGS/NGS boundary
             (3, (3, 29, nts - 10, 211)),               # truth sensor x LGS
             (3, (11, nlgs_rows - 31, 60, 90))]         # truth sensor across LGS/NGS
    for typ, (x0, y0, nr, nc) in cases:
        ref = O.matcov(g, nr, nc, x0, y0, typ, nthreads=8)
        buf = np.full((nr + 3, nc), 7.0, order="F")
        M.matcov_tile(buf, nr, nc, x0, y0, nr + 3, t, typ, ctx=ctx)
        got = buf[:nr]
        if typ == 1:
            gx = np.arange(nr)[:, None] + x0
            gy = np.arange(nc)[None, :] + y0
            assert np.all(got[gy > gx] == 7.0), "untouched upper elements were modified"
            ref = np.where(gy > gx, 7.0, ref)
        assert np.all(buf[nr:] == 7.0), "wrote outside the tile (ld padding)"
        assert_close(got, ref, 1e-11, f"elt16 tile type {typ} at {x0},{y0}")


def test_matcov_bad_type_raises(ctx):
    t, g = tomo_and_geom("small")
    buf = np.zeros((4, 4), order="F")
    with pytest.raises(M.MoaoError) as e:
        M.matcov_tile(buf, 4, 4, 0, 0, 4, t, 7, ctx=ctx)
    assert e.value.name == "MOAO_ERR_BAD_ARG"
    with pytest.raises(M.MoaoError):
        M.matcov_tile(buf, 4, 4, g.nmeas, 0, 4, t, 1, ctx=ctx)  # outside the matrix


def _kappa(S):
    w = np.linalg.eigvalsh(S)
    return w.max() / w.min()


def _pipeline_case(name):
    t, g = tomo_and_geom(name)
    nm, nts = g.nmeas, g.nmeasts
    Cmm = O.matcov(g, nm, nm, 0, 0, 1, nthreads=8)
    t.setTarget(0)
    Ctm = O.matcov(g, nts, nm, 0, 0, 3, nthreads=8)
    Ctt = O.matcov(g, nts, nts, 0, 0, 4, nthreads=8)
    S = np.tril(Cmm) + np.tril(Cmm, -1).T
    return t, g, Cmm, Ctm, Ctt, _kappa(S)


@pytest.mark.parametrize("name", ["small", "check2"])
@pytest.mark.parametrize("nb", [64, 256])
def test_reconstructor_fp64(ctx, name, nb):
    t, g, Cmm, Ctm, Ctt, kappa = _pipeline_case(name)
    tol = max(1e-10, 50 * kappa * EPS)
    L_ref, R_ref, info = O.reconstructor(Cmm, Ctm)
    assert info == 0
    ctx.set_block(nb)
    try:
        dC, dT = dev(Cmm), dev(Ctm)
        nm, nts = g.nmeas, g.nmeasts
        rep = M.reconstructor(nm, nts, dC, nm, dT, nts, 1, ctx=ctx)
        ctx.synchronize()
    finally:
        ctx.set_block(256)
    assert rep["info"] == 0
    R = host(dT)
    L = host(dC)
    assert_close(R, R_ref, tol, f"R ({name}, kappa {kappa:.2e})")
    assert_close(np.tril(L), np.tril(L_ref), tol, "L")
    assert np.array_equal(np.triu(L, 1), np.triu(Cmm, 1)), "upper triangle of Cmm modified"


def test_reconstructor_random_spd_odd_sizes(ctx):
    rng = np.random.default_rng(5)
    for n, m, nb in ((1000, 77, 256), (333, 5, 64), (700, 130, 128)):
        A = rng.standard_normal((n, n))
        C = A @ A.T / n + np.eye(n)
        T = rng.standard_normal((m, n))
        L_ref, R_ref, _ = O.reconstructor(np.tril(C), T)
        ctx.set_block(nb)
        try:
            dC, dT = dev(np.tril(C)), dev(T)
            M.reconstructor(n, m, dC, n, dT, m, 1, ctx=ctx)
        finally:
            ctx.set_block(256)
        assert_close(host(dT), R_ref, 1e-11, f"R {n}x{m}")
        assert_close(np.tril(host(dC)), np.tril(L_ref), 1e-11, f"L {n}")


def test_reconstructor_multiple_targets_and_host_path(ctx):
    t, g, Cmm, Ctm, Ctt, kappa = _pipeline_case("small")
    nm, nts = g.nmeas, g.nmeasts
    tol = max(1e-10, 50 * kappa * EPS)
    T2 = np.concatenate([Ctm.flatten("F"), 0.5 * Ctm.flatten("F")])
    C = Cmm.copy(order="F")
    M.reconstructor(nm, nts, C, nm, T2, nts, 2, ctx=ctx)   # host buffers
    _, R_ref, _ = O.reconstructor(Cmm, Ctm)
    R0 = T2[: nm * nts].reshape((nts, nm), order="F")
    R1 = T2[nm * nts:].reshape((nts, nm), order="F")
    assert_close(R0, R_ref, tol, "target 0")
    assert_close(R1, 0.5 * R_ref, tol, "target 1")


def test_reconstructor_not_spd(ctx):
    n = 200
    C = np.eye(n)
    C[150, 150] = -1.0
    T = np.ones((3, n))
    Th = T.copy(order="F")
    with pytest.raises(M.NotSPDError) as e:
        M.reconstructor(n, 3, C.copy(order="F"), n, Th, 3, 1, ctx=ctx)
    assert e.value.column == 151
    assert np.array_equal(Th, T), "Ctm must be left untouched on failure"
    # the context stays usable
    rng = np.random.default_rng(0)
    A = rng.standard_normal((64, 64))
    S = A @ A.T + 64 * np.eye(64)
    R = np.ones((2, 64), order="F")
    M.reconstructor(64, 2, S.copy(order="F"), 64, R, 2, 1, ctx=ctx)
    assert np.allclose(R @ S, np.ones((2, 64)), atol=1e-10)


@pytest.mark.parametrize("name", ["small", "check2"])
def test_cee_cvv_fp64(ctx, name):
    t, g, Cmm, Ctm, Ctt, kappa = _pipeline_case(name)
    nm, nts = g.nmeas, g.nmeasts
    _, R, _ = O.reconstructor(Cmm, Ctm)
    nact = 100
    Dx = I.make_dx(nact, nts, seed=3)
    Cee_ref, Cvv_ref, Cpp_ref, Cpm_ref, Tmp_ref = O.cee_cvv(Cmm, Ctt, Ctm, R, Dx)
    d = {k: dev(v) for k, v in dict(Cmm=Cmm, Cpp=Ctt, Cpm=Ctm, R=R, Dx=Dx).items()}
    import torch
    Cee = torch.zeros((nts, nts), dtype=torch.float64, device="cuda")
    Cvv = torch.zeros((nact, nact), dtype=torch.float64, device="cuda")
    Tmp = torch.zeros((nts, nact), dtype=torch.float64, device="cuda")
    M.Cee_Cvv(nm, nts, nact, d["Cmm"], nm, d["Cpp"], nts, d["Cpm"], nts, d["R"], nts, d["Dx"], nact,
              Cee, nts, Cvv, nact, Tmp, nact, ctx=ctx)
    ctx.synchronize()
    # Cee carries the cancellation Ctt - 2 Ctm R^T + R Cmm R^T; bound it by the
    # size of the terms, not of the (much smaller) result.
    scale = np.linalg.norm(Ctt) / np.linalg.norm(Cee_ref)
    tol = 1e-12 * scale
    assert_close(host(Cee), Cee_ref, tol, "Cee")
    assert_close(host(Cvv), Cvv_ref, tol, "Cvv")
    assert_close(np.tril(host(d["Cpp"])), np.tril(Cpp_ref), tol, "Cpp after")
    assert_close(host(d["Cpm"]), Cpm_ref, 1e-12, "Cpm after")
    assert_close(host(Tmp), Tmp_ref, tol, "Tmp")


def test_cee_cvv_host_buffers(ctx):
    t, g, Cmm, Ctm, Ctt, kappa = _pipeline_case("small")
    nm, nts, nact = g.nmeas, g.nmeasts, 100
    _, R, _ = O.reconstructor(Cmm, Ctm)
    Dx = I.make_dx(nact, nts)
    Cee_ref, Cvv_ref, *_ = O.cee_cvv(Cmm, Ctt, Ctm, R, Dx)
    Cpp, Cpm = Ctt.copy(order="F"), Ctm.copy(order="F")
    Cee = np.zeros((nts, nts), order="F")
    Cvv = np.zeros((nact, nact), order="F")
    Tmp = np.zeros((nact, nts), order="F")
    M.Cee_Cvv(nm, nts, nact, Cmm.copy(order="F"), nm, Cpp, nts, Cpm, nts, R.copy(order="F"), nts,
              Dx.copy(order="F"), nact, Cee, nts, Cvv, nact, Tmp, nact, ctx=ctx)
    scale = np.linalg.norm(Ctt) / np.linalg.norm(Cee_ref)
    assert_close(Cee, Cee_ref, 1e-12 * scale, "Cee host")
    assert_close(Cvv, Cvv_ref, 1e-12 * scale, "Cvv host")


@pytest.mark.parametrize("nssp,diam,obs", [(10, 8.0, 0.14), (64, 39.0, 0.28)])
def test_intersample(ctx, nssp, diam, obs):
    x = I.intersample_inputs(nssp, diam, obs)
    nact = x.nact
    rng = np.random.default_rng(2)
    B = rng.standard_normal((nact, nact)) * 1e-3 / np.sqrt(nact)
    Cvv = B @ B.T
    want = O.intersample(Cvv, x.idx, x.abs2fi, x.otf, x.np_)
    isx = M.Intersample(nact * nact, x.np_, diam, x.idx, x.abs2fi, x.otf, ctx=ctx)
    got = isx.process(Cvv.copy(order="F"))
    assert_close(got, want, 1e-10, "psf (host)")
    import torch
    got_d = isx.process(dev(Cvv))
    ctx.synchronize()
    assert_close(got_d.cpu().numpy(), want, 1e-10, "psf (device)")
    isx.close()


def test_intersample_rejects_bad_idx(ctx):
    x = I.intersample_inputs(10, 8.0, 0.14)
    idx = x.idx.copy()
    idx[5] = 10 ** 6
    with pytest.raises(M.MoaoError):
        M.Intersample(x.nact ** 2, x.np_, 8.0, idx, x.abs2fi, x.otf, ctx=ctx)


def test_full_pipeline_elt16_properties(ctx):
    """Size-independent properties on a larger system computed entirely on the GPU:
    R Cmm = Ctm and Cmm SPD, against a full oracle R."""
    import torch
    t, g = tomo_and_geom("elt16")
    nm, nts = g.nmeas, g.nmeasts
    C = torch.zeros((nm, nm), dtype=torch.float64, device="cuda")
    T = torch.zeros((nm, nts), dtype=torch.float64, device="cuda")
    M.matcov_tile(C, nm, nm, 0, 0, nm, t, 5, ctx=ctx)
    t.setTarget(0)
    M.matcov_tile(T, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
    ctx.synchronize()  # the library runs on the context stream, torch on its own
    Cfull = C.clone()
    Tctm = T.clone()
    M.reconstructor(nm, nts, C, nm, T, nts, 1, ctx=ctx)
    ctx.synchronize()
    R = host(T)
    S = host(Cfull)
    resid = np.linalg.norm(R @ S - host(Tctm)) / np.linalg.norm(host(Tctm))
    assert resid < 1e-10, resid
    Cmm_o = O.matcov(g, nm, nm, 0, 0, 1, nthreads=8)
    Ctm_o = O.matcov(g, nts, nm, 0, 0, 3, nthreads=8)
    _, R_ref, _ = O.reconstructor(Cmm_o, Ctm_o)
    kappa = _kappa(np.tril(Cmm_o) + np.tril(Cmm_o, -1).T)
    assert_close(R, R_ref, max(1e-10, 50 * kappa * EPS), "elt16 R")
