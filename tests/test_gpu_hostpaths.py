"""The host-buffer (drop-in) entry points move only what the reference writes.

moao_matcov_tile_host sends the column panels' diagonal blocks down and the
written lower part back for type-1 tiles (no copy down for full tiles), and
moao_reconstructor_host moves only the lower part of Cmm both ways. These
tests fill every element the reference leaves untouched with a sentinel and
check it survives, on tiles spanning several 512-column panels, at odd
offsets and with padded leading dimensions, and compare the values with the
device entry points (FP64 and mixed).
"""
import numpy as np
import pytest

import oracle as O
import systems
import moao_b200 as M

pytestmark = pytest.mark.gpu
SENT = 7.25


def tomo(name):
    sf, af = systems.files(name)
    t = M.Tomo(sf, af)
    t.setTarget(0)
    return t


def test_matcov_host_type1_keeps_untouched_elements(ctx):
    import torch
    t = tomo("elt16")
    nm, nts = t.getNMeas(), t.getNMeasTS()
    full = torch.zeros((nm, nm), dtype=torch.float64, device="cuda")
    M.matcov_tile(full, nm, nm, 0, 0, nm, t, 5, ctx=ctx)  # both triangles
    ctx.synchronize()
    ref = full.cpu().numpy().T
    for (x0, y0, nr, nc, pad) in [(0, 0, nm, nm, 0), (0, 0, nm, nm, 3), (700, 37, 900, 1200, 5),
                                  (37, 700, 1100, 600, 0), (1000, 1000, 1100, 1100, 2)]:
        nr, nc = min(nr, nm - x0), min(nc, nm - y0)
        buf = np.full((nr + pad, nc), SENT, order="F")
        M.matcov_tile(buf, nr, nc, x0, y0, nr + pad, t, 1, ctx=ctx)
        gx = np.arange(nr)[:, None] + x0
        gy = np.arange(nc)[None, :] + y0
        written = gy <= gx
        got = buf[:nr]
        assert np.all(got[~written] == SENT), (x0, y0, "an untouched element changed")
        assert np.all(buf[nr:] == SENT), "wrote into the padding"
        want = ref[x0:x0 + nr, y0:y0 + nc]
        # tiles at other offsets may take other kernel paths: rounding-level agreement
        assert np.max(np.abs(got[written] - want[written]), initial=0.0) <= 1e-12 * np.abs(ref).max()
    # full tiles (type 3) need no copy down and write everything
    buf = np.full((nts + 4, nm), SENT, order="F")
    M.matcov_tile(buf, nts, nm, 0, 0, nts + 4, t, 3, ctx=ctx)
    d = torch.zeros((nm, nts), dtype=torch.float64, device="cuda")
    M.matcov_tile(d, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
    ctx.synchronize()
    assert np.array_equal(buf[:nts], d.cpu().numpy().T)
    assert np.all(buf[nts:] == SENT)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_reconstructor_host_lower_only(ctx, prec):
    import torch
    t = tomo("elt16")
    nm, nts = t.getNMeas(), t.getNMeasTS()
    if prec == "mixed":
        ctx.set_offsets_from_tomo(t)
    try:
        dC = torch.zeros((nm, nm), dtype=torch.float64, device="cuda")
        dT = torch.zeros((nm, nts), dtype=torch.float64, device="cuda")
        M.matcov_tile(dC, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
        M.matcov_tile(dT, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
        ctx.synchronize()
        Cmm = dC.cpu().numpy().T.copy(order="F")
        Ctm = dT.cpu().numpy().T.copy(order="F")
        M.reconstructor(nm, nts, dC, nm, dT, nts, 1, prec=prec, ctx=ctx)
        ctx.synchronize()
        L_dev, R_dev = dC.cpu().numpy().T, dT.cpu().numpy().T
        pad = 3
        Ch = np.full((nm + pad, nm), SENT, order="F")
        Ch[:nm][np.tril_indices(nm)] = Cmm[np.tril_indices(nm)]
        Th = Ctm.copy(order="F")
        M.reconstructor(nm, nts, Ch, nm + pad, Th, nts, 1, prec=prec, ctx=ctx)
    finally:
        ctx.set_offsets([], [], [])
    up = np.triu_indices(nm, 1)
    assert np.all(Ch[:nm][up] == SENT), "the upper triangle of Cmm changed"
    assert np.all(Ch[nm:] == SENT), "wrote into Cmm's padding"
    lo = np.tril_indices(nm)
    assert np.array_equal(Ch[:nm][lo], L_dev[lo])
    assert np.array_equal(Th, R_dev)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_host_cache_skips_the_uploads(ctx, prec):
    """With moao_ctx_set_host_cache on, the Cmm and Ctm that matcov_tile left in
    host buffers are not uploaded again by reconstructor: the outputs equal the
    uncached host path's bit for bit, the caller's upper triangle and padding
    survive, and a change the caller makes to the host Cmm in between (breaking
    the promise on purpose) is not seen, which shows the device copy was used.
    Another tile generated in between, or a different host buffer, misses the
    cache."""
    t = tomo("elt16")
    nm, nts = t.getNMeas(), t.getNMeasTS()
    pad = 3
    if prec == "mixed":
        ctx.set_offsets_from_tomo(t)

    def build(cache, tamper=False, other_tile=False):
        ctx.set_host_cache(cache)
        Ch = np.full((nm + pad, nm), SENT, order="F")
        Th = np.zeros((nts, nm), order="F")
        M.matcov_tile(Ch, nm, nm, 0, 0, nm + pad, t, 1, ctx=ctx)
        M.matcov_tile(Th, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
        if other_tile:
            Ctt = np.zeros((nts, nts), order="F")
            M.matcov_tile(Ctt, nts, nts, 0, 0, nts, t, 4, ctx=ctx)
        if tamper:
            lo = np.tril_indices(nm, -1)
            Ch[:nm][lo] *= 0.5
        M.reconstructor(nm, nts, Ch, nm + pad, Th, nts, 1, prec=prec, ctx=ctx)
        return Ch, Th

    try:
        C0, T0 = build(False)
        C1, T1 = build(True)
        if prec == "fp64":  # halving the off-diagonal part keeps Cmm SPD
            C2, T2 = build(True, tamper=True)
            C3, T3 = build(True, tamper=True, other_tile=True)
            C4, T4 = build(False, tamper=True)
    finally:
        ctx.set_host_cache(False)
        ctx.set_offsets([], [], [])
    up = np.triu_indices(nm, 1)
    for C in (C0, C1):
        assert np.all(C[:nm][up] == SENT) and np.all(C[nm:] == SENT)
    assert np.array_equal(C1, C0) and np.array_equal(T1, T0)
    if prec == "fp64":
        assert np.array_equal(C2, C0) and np.array_equal(T2, T0), "the device copy was not used"
        # Cmm's cache was dropped by the Ctt tile: the tampered matrix was uploaded
        assert np.all(C3[:nm][up] == SENT) and np.all(C3[nm:] == SENT)
        assert np.array_equal(C3, C4) and np.array_equal(T3, T4)
        assert not np.array_equal(T3, T0)
