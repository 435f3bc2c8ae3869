"""The oracle is pinned before it is trusted (CPU only).

* Covariance generation: the C restatement against the reference's own code
  compiled from its sources (oracle/_ref) and against the committed golden
  fixtures generated from that code (tests/golden/make_golden.py).
* LAPACK/BLAS restatements: identities the reference's semantics imply.
* Intersample restatement: structural properties of the PSF.
"""
import os

import numpy as np
import pytest

import oracle as O
import systems
from moao_b200 import Tomo, inputs as I

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _geom(name):
    sf, af = systems.files(name)
    return O.Geometry.from_tomo(Tomo(sf, af))


@pytest.mark.parametrize("name", ["small", "check2", "check10"])
def test_oracle_matches_golden_samples(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    g = _geom(name)
    for tag, typ, nr, nc in (("Cmm", 1, g.nmeas, g.nmeas), ("Ctm", 3, g.nmeasts, g.nmeas),
                             ("Ctt", 4, g.nmeasts, g.nmeasts)):
        M = O.matcov(g, nr, nc, 0, 0, typ, nthreads=os.cpu_count() or 1)
        r, c, v = z[f"{tag}_rows"], z[f"{tag}_cols"], z[f"{tag}_vals"]
        assert np.array_equal(M[r, c], v), f"{name} {tag}: oracle differs from the reference"
        part = np.tril(M) if typ == 1 else M
        assert np.array_equal(part.sum(axis=0), z[f"{tag}_colsum"])


@pytest.mark.skipif(not O.RefTomo.available(), reason="reference library not built here")
@pytest.mark.parametrize("name", ["small", "check2"])
def test_oracle_bit_identical_to_reference_tiles(name):
    """Tiles at odd offsets (the reference's tile entry point) are bit-identical."""
    sf, af = systems.files(name)
    ref = O.RefTomo(sf, af)
    g = _geom(name)
    for typ, (x0, y0, nr, nc) in [(1, (37, 11, 100, 90)), (1, (0, 0, 64, 64)), (3, (5, 61, 40, 77)),
                                  (4, (3, 9, 50, 31))]:
        A = np.zeros((nr, nc), order="F")
        B = np.zeros((nr, nc), order="F")
        ref.matcov_tile(A, nr, nc, x0, y0, nr, typ)
        O.matcov(g, nr, nc, x0, y0, typ, out=B)
        assert np.array_equal(A, B)


def test_dphi_model_properties():
    assert O.dphi(0.0, 0.0, 25.0) == 0.0
    # near-continuity where the series hands over to the 3-term asymptotic form
    # (x = Xlim): the model itself jumps by 2.6e-4 relative there
    L0 = 25.0
    rlim = 0.75 * 2 * np.pi * L0 / (2 * np.pi)
    lo, hi = O.dphi(rlim * (1 - 1e-9), 0, L0), O.dphi(rlim * (1 + 1e-9), 0, L0)
    assert abs(lo - hi) / abs(lo) < 1e-3
    # Kolmogorov regime: DPHI ~ 6.88 (r/r0)^(5/3) with r0 = 1 for r << L0
    r = 1e-3
    assert abs(O.dphi(r, 0, 1e4) / (6.88 * r ** (5 / 3)) - 1) < 1e-2
    # monotone increasing, saturating
    v = [O.dphi(x, 0, L0) for x in (0.1, 1, 10, 100, 1000)]
    assert all(b > a for a, b in zip(v, v[1:]))


def test_cmm_is_spd_and_scales_with_cn2():
    sf, af = systems.files("small")
    t = Tomo(sf, af)
    g = O.Geometry.from_tomo(t)
    C = O.matcov(g, g.nmeas, g.nmeas, 0, 0, 1)
    S = np.tril(C) + np.tril(C, -1).T
    assert np.linalg.eigvalsh(S).min() > 0
    # turbulence part is linear in cn2: doubling every layer doubles (C - noise)
    t2 = Tomo(sf, af)
    cn2 = t2.table("cn2")
    t2.set_profile(2 * cn2, t2.table("h"), t2.table("L0diff"))
    g2 = O.Geometry.from_tomo(t2)
    Ctm1 = O.matcov(g, g.nmeasts, g.nmeas, 0, 0, 3)
    Ctm2 = O.matcov(g2, g.nmeasts, g.nmeas, 0, 0, 3)
    assert np.allclose(Ctm2, 2 * Ctm1, rtol=1e-12, atol=0)


def test_lapack_restatement_identities():
    rng = np.random.default_rng(0)
    n, m, na = 60, 12, 9
    A = rng.standard_normal((n, n))
    Cmm = A @ A.T + n * np.eye(n)
    Ctm = rng.standard_normal((m, n))
    L, R, info = O.reconstructor(np.tril(Cmm), Ctm)
    assert info == 0
    assert np.allclose(R @ Cmm, Ctm, atol=1e-10)
    assert np.allclose(np.tril(L) @ np.tril(L).T, Cmm, atol=1e-10)
    B = rng.standard_normal((m, m))
    Ctt = B @ B.T
    Dx = rng.standard_normal((na, m))
    Cee, Cvv, *_ = O.cee_cvv(np.tril(Cmm), Ctt, Ctm, R, Dx)
    want = Ctt - Ctm @ R.T - R @ Ctm.T + R @ Cmm @ R.T
    assert np.allclose(Cee, want, atol=1e-9)
    assert np.allclose(Cvv, Dx @ Cee @ Dx.T, atol=1e-8)
    # the vectorised geadd equals the reference's in-place loop
    Cee2, Cvv2, *_ = O.cee_cvv(np.tril(Cmm), Ctt, Ctm, R, Dx, literal_geadd=True)
    assert np.array_equal(Cee, Cee2) and np.array_equal(Cvv, Cvv2)


def test_reconstructor_reports_non_spd():
    C = np.diag([1.0, -1.0, 1.0])
    _, R, info = O.reconstructor(C, np.ones((1, 3)))
    assert info == 2 and R is None


def test_intersample_restatement_properties():
    x = I.intersample_inputs(10, 8.0, 0.14)
    nact = x.nact
    rng = np.random.default_rng(1)
    B = rng.standard_normal((nact, nact)) * 1e-3
    Cvv = B @ B.T
    psf = O.intersample(Cvv, x.idx, x.abs2fi, x.otf, x.np_)
    N = x.fourier.N
    assert psf.shape == (N, N)
    # Zero residual gives the diffraction-limited PSF, whose peak is the Strehl 1
    # normalisation of OTF_telescope (peak = sum(otf) * N^2 / N^2 ...).
    psf0 = O.intersample(np.zeros_like(Cvv), x.idx, x.abs2fi, x.otf, x.np_)
    strehl = psf.max() / psf0.max()
    assert 0 < strehl <= 1.0
    assert abs(psf0.max() - x.otf.sum()) / x.otf.sum() < 1e-9


def test_compare_matrices_semantics():
    A = np.array([[1.0, 0.0], [2.0, 4.0]])
    B = np.array([[1.1, 5.0], [2.0, 4.0]])
    maxerr, fro = O.compare_matrices(A, B)
    assert np.isclose(maxerr, 5.0) and np.isclose(fro, np.sqrt(0.01 + 25))


@pytest.mark.parametrize("name", systems.CHECK_SETS + ["elt"])
def test_oracle_matches_reference_tiles_of_check_sets(name):
    """The C restatement reproduces, bit for bit, the reference's tiles of Cmm,
    Ctm and Ctt for the six reference check systems and the ELT-scale system
    (tests/golden/ref_*.npz, from the reference's compiled code)."""
    z = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    g = _geom(name)
    nt = z["tile_vals"].shape[1]
    for (typ, r0, c0), want in zip(z["tile_spec"], z["tile_vals"]):
        got = np.zeros((nt, nt), order="F")
        O.matcov(g, nt, nt, int(r0), int(c0), int(typ), out=got)
        assert np.array_equal(got, want), (name, typ, r0, c0)


needs_ref_dense = pytest.mark.skipif(not O.RefDense.available(),
                                     reason="reference dense library not built here")


def _dense_case(name):
    g = _geom(name)
    nm, nts = g.nmeas, g.nmeasts
    Cmm = O.matcov(g, nm, nm, 0, 0, 1, nthreads=8)
    Ctm = O.matcov(g, nts, nm, 0, 0, 3, nthreads=8)
    Ctt = O.matcov(g, nts, nts, 0, 0, 4, nthreads=8)
    return Cmm, Ctm, Ctt


@needs_ref_dense
@pytest.mark.parametrize("name", ["small", "check2"])
def test_reconstructor_restatement_equals_reference_code(name):
    """oracle.reconstructor against the reference's MOAO_LAPACK::reconstructor
    (lapack/compute/reconstructor.cpp:32-58) run here on the same matrices."""
    Cmm, Ctm, _ = _dense_case(name)
    L, R, info = O.reconstructor(Cmm, Ctm)
    L_ref, R_ref = O.RefDense.reconstructor(Cmm, Ctm)
    assert info == 0
    # the same OpenBLAS routines in the same order: bit-identical
    assert np.array_equal(np.tril(L), np.tril(L_ref))
    assert np.array_equal(R, R_ref)
    assert np.array_equal(np.triu(L_ref, 1), np.triu(Cmm, 1)), "reference left the upper part"


@needs_ref_dense
@pytest.mark.parametrize("name", ["small", "check2"])
def test_cee_cvv_restatement_equals_reference_code(name):
    """oracle.cee_cvv (both geadd forms) against the reference's nine steps
    (lapack/compute/cee_cvv.cpp:50-125) run here, including the in-place
    results left in Cpp and Cpm."""
    Cmm, Ctm, Ctt = _dense_case(name)
    _, R, _ = O.reconstructor(Cmm, Ctm)
    Dx = I.make_dx(100, Ctt.shape[0], seed=3)
    ref = O.RefDense.cee_cvv(Cmm, Ctt, Ctm, R, Dx)
    for literal in (True, False):
        got = O.cee_cvv(Cmm, Ctt, Ctm, R, Dx, literal_geadd=literal)
        Cee, Cvv, Cpp, Cpm, Tmp = got
        # the literal geadd loop is bit-identical; the mirrored form equals it
        # too (x + y and y + x round alike)
        assert np.array_equal(Cee, ref[0])
        assert np.array_equal(Cvv, ref[1])
        assert np.array_equal(np.tril(Cpp), np.tril(ref[2]))
        assert np.array_equal(Cpm, ref[3])
        assert np.array_equal(Tmp, ref[4])


@needs_ref_dense
@pytest.mark.parametrize("nssp,diam,obs", [(10, 8.0, 0.14), (10, 39.0, 0.2), (29, 39.0, 0.2)])
def test_intersample_restatement_equals_reference_code(nssp, diam, obs):
    """oracle.intersample (numpy FFTs) against the reference's intersample
    pipeline (common/tomo_struct/intersample.cpp:74-333) run here with the
    FFTW transforms restated in oracle/ref_dense_shim.cpp."""
    x = I.intersample_inputs(nssp, diam, obs)
    rng = np.random.default_rng(4)
    B = rng.standard_normal((x.nact, x.nact)) * 1e-3 / np.sqrt(x.nact)
    Cvv = B @ B.T
    got = O.intersample(Cvv, x.idx, x.abs2fi, x.otf, x.np_)
    ref = O.RefDense.intersample(Cvv, x.idx, x.abs2fi, x.otf, x.np_, diam)
    # measured: 1 ulp of the peak (numpy's FFT against the restated FFTW transforms)
    assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref))
    # a zero Cvv gives the telescope-only PSF in both
    z = np.zeros_like(Cvv)
    assert np.allclose(O.intersample(z, x.idx, x.abs2fi, x.otf, x.np_),
                       O.RefDense.intersample(z, x.idx, x.abs2fi, x.otf, x.np_, diam),
                       rtol=0, atol=1e-11 * np.max(np.abs(ref)))
