"""The intersample tables synthesised on the device (moao_intersample_inputs,
moao_intersample_create_synth) against the reference tooling's formulas
(moao_b200.inputs, numpy): abs2fi and the telescope OTF within 1e-12 of their
maxima (cuFFT against numpy's FFT, rounding only), idx exact, and a PSF from a
synthesised intersample object within 1e-6 of one built from the numpy tables:
the PSF's exponent multiplies the structure function by 2 (2 pi / lambda)^2 /
(N dactupix)^2 (~1e8 at N = 512), which turns rounding-level differences of
the tables into ~1e-7 of the PSF (measured 1.5e-7 at 10x10)."""
import numpy as np
import pytest

import moao_b200 as M
from moao_b200 import inputs as I

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nssp,diam,obs", [(10, 8.0, 0.14), (64, 39.0, 0.28)])
def test_synthesised_tables_match_tooling(ctx, nssp, diam, obs):
    na, N, idx, a, o = M.intersample_inputs(nssp, diam, obs, ctx=ctx)
    x = I.intersample_inputs(nssp, diam, obs)
    assert na == x.nact and N == x.fourier.N and np.array_equal(idx, x.idx)
    for got, want, name in ((a, x.abs2fi, "abs2fi"), (o, x.otf, "otf")):
        err = np.max(np.abs(got - want)) / np.max(np.abs(want))
        assert err <= 1e-12, (name, err)


def test_psf_from_synthesised_object(ctx):
    import ctypes as C
    from moao_b200._lib import lib, check
    nssp, diam, obs = 10, 8.0, 0.14
    x = I.intersample_inputs(nssp, diam, obs)
    rng = np.random.default_rng(8)
    B = rng.standard_normal((x.nact, x.nact)) * 1e-3 / np.sqrt(x.nact)
    Cvv = B @ B.T
    want = M.Intersample(x.nact ** 2, x.np_, diam, x.idx, x.abs2fi, x.otf, ctx=ctx).process(
        Cvv.copy(order="F"))
    h = C.c_void_p()
    check(lib().moao_intersample_create_synth(ctx.handle, nssp, diam, obs, 0.2, C.byref(h)),
          "moao_intersample_create_synth")
    got = np.zeros_like(want)
    check(lib().moao_intersample_process_host(h, Cvv.copy(order="F").ctypes.data, got.ctypes.data),
          "moao_intersample_process_host")
    lib().moao_intersample_destroy(h)
    assert np.max(np.abs(got - want)) <= 1e-6 * np.max(np.abs(want))
