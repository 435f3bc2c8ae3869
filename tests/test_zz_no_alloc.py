"""The reconstructor entry point that allocates no device memory.

Callers that cannot allocate while running (a real-time adaptive-optics
controller refreshing its reconstructor between frames, or an application whose
memory pool owns the whole GPU) use moao_reconstructor_noalloc, whose scratch
is a fixed device array inside the library. Its output must equal the regular
FP64 entry point's on the same inputs, call after call, because every call
reuses (and must reset) the same scratch. Tolerance: the same
max(1e-10, 50 kappa eps) relative Frobenius bound as the other FP64 parity tests
(the two entry points run the same blocked algorithm, so they agree exactly in
practice). This file is collected last so that a failure here cannot hide the
other tests' results.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import systems
import moao_b200 as M
from moao_b200._lib import lib

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


def dev(A):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(A, dtype=np.float64).T)).cuda()


def host(t):
    return t.cpu().numpy().T.copy(order="F")


def noalloc(nm, nts, dC, dT, ngal=1, ldC=None, ldT=None):
    import torch
    info = C.c_int(-1)
    st = lib().moao_reconstructor_noalloc(nm, nts, dC.data_ptr(), ldC or nm, dT.data_ptr(),
                                          ldT or nts, ngal,
                                          C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                          C.byref(info))
    return st, info.value


def inputs(name):
    sf, af = systems.files(name)
    g = O.Geometry.from_tomo(M.Tomo(sf, af))
    nm, nts = g.nmeas, g.nmeasts
    return nm, nts, O.matcov(g, nm, nm, 0, 0, 1, nthreads=8), O.matcov(g, nts, nm, 0, 0, 3, nthreads=8)


def test_noalloc_matches_regular_entry_point_twice(ctx):
    import torch
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        for name in ("small", "check2"):
            nm, nts, Cmm, Ctm = inputs(name)
            S = np.tril(Cmm) + np.tril(Cmm, -1).T
            w = np.linalg.eigvalsh(S)
            tol = max(1e-10, 50 * (w.max() / w.min()) * EPS)
            dC_ref, dT_ref = dev(Cmm), dev(Ctm)
            M.reconstructor(nm, nts, dC_ref, nm, dT_ref, nts, 1, ctx=ctx)
            R_ref, L_ref = host(dT_ref), np.tril(host(dC_ref))
            for call in range(2):  # two calls in a row share the same scratch
                dC, dT = dev(Cmm), dev(Ctm)
                st, info = noalloc(nm, nts, dC, dT)
                assert st == 0 and info == 0, (st, lib().moao_last_error())
                assert O.rel_fro(host(dT), R_ref) <= tol, (name, call)
                assert O.rel_fro(np.tril(host(dC)), L_ref) <= tol, (name, call)
                assert np.array_equal(np.triu(host(dC), 1), np.triu(Cmm, 1))
    finally:
        ctx.set_stream(None)


def test_noalloc_limit_and_pivot_flag_reset(ctx):
    import torch
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    st, _ = noalloc(4096, 100, dummy, dummy)
    assert st == 1 and b"2048" in lib().moao_last_error()
    n = 300
    bad = np.eye(n)
    bad[250, 250] = -1.0
    st, info = noalloc(n, 2, dev(bad), dev(np.ones((2, n))))
    assert st == 2 and info == 251
    # the next call starts from a cleared pivot flag
    rng = np.random.default_rng(1)
    A = rng.standard_normal((n, n))
    S = A @ A.T / n + np.eye(n)
    T = rng.standard_normal((3, n))
    dT = dev(T)
    st, info = noalloc(n, 3, dev(np.tril(S)), dT)
    assert st == 0 and info == 0
    assert np.allclose(host(dT) @ S, T, atol=1e-10)


def padded(A, ld):
    """Column-major device copy of A with leading dimension ld (rows beyond A hold 7.0)."""
    P = np.full((ld, A.shape[1]), 7.0)
    P[:A.shape[0]] = A
    return dev(P)


def spd(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    return A @ A.T / n + np.eye(n)


def test_noalloc_at_size_limit_and_with_targets_and_padding(ctx):
    """nmeas = nmeasts = 2048 (the inverse blocks and the panel fill the whole
    array), then ngal = 2 targets sharing one factor with padded leading
    dimensions, each against moao_reconstructor on the same inputs."""
    import torch
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        # size limit
        n = m = 2048
        S = spd(n, 3)
        T = np.random.default_rng(4).standard_normal((m, n))
        w = np.linalg.eigvalsh(S)
        tol = max(1e-10, 50 * (w.max() / w.min()) * EPS)
        dC_ref, dT_ref = dev(np.tril(S)), dev(T)
        M.reconstructor(n, m, dC_ref, n, dT_ref, m, 1, ctx=ctx)
        R_ref = host(dT_ref)
        for call in range(2):
            dC, dT = dev(np.tril(S)), dev(T)
            st, info = noalloc(n, m, dC, dT)
            assert st == 0 and info == 0, (st, lib().moao_last_error())
            assert O.rel_fro(host(dT), R_ref) <= tol, call
        # two targets (stored nmeas*nmeasts apart, as the reference lays them out)
        # and a padded Cmm; then one target with a padded Ctm
        nm, nts, Cmm, Ctm = inputs("check2")
        S2 = np.tril(Cmm) + np.tril(Cmm, -1).T
        w = np.linalg.eigvalsh(S2)
        tol = max(1e-10, 50 * (w.max() / w.min()) * EPS)
        Ctm2 = np.random.default_rng(5).standard_normal((nts, nm)) * np.abs(Ctm).max()
        both = np.concatenate([Ctm.ravel(order="F"), Ctm2.ravel(order="F")])
        ldC = nm + 13
        dT_ref = torch.from_numpy(both.copy()).cuda()
        M.reconstructor(nm, nts, dev(Cmm), nm, dT_ref, nts, 2, ctx=ctx)
        R_ref = dT_ref.cpu().numpy()
        for call in range(2):
            dC = padded(Cmm, ldC)
            dT = torch.from_numpy(both.copy()).cuda()
            st, info = noalloc(nm, nts, dC, dT, ngal=2, ldC=ldC)
            assert st == 0 and info == 0, (st, lib().moao_last_error())
            got = dT.cpu().numpy()
            for g in range(2):
                sl = slice(g * nm * nts, (g + 1) * nm * nts)
                assert O.rel_fro(got[sl], R_ref[sl]) <= tol, (call, g)
            # the padding rows of Cmm are not touched
            assert np.all(host(dC)[nm:] == 7.0)
        ldT = nts + 5
        dT = padded(Ctm, ldT)
        st, info = noalloc(nm, nts, padded(Cmm, ldC), dT, ldC=ldC, ldT=ldT)
        assert st == 0 and info == 0
        got = host(dT)
        assert O.rel_fro(got[:nts], R_ref[:nm * nts].reshape(nts, nm, order="F")) <= tol
        assert np.all(got[nts:] == 7.0)
    finally:
        ctx.set_stream(None)


def test_noalloc_empty_sizes_are_noops(ctx):
    import torch
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    st, info = noalloc(0, 5, dummy, dummy, ldC=1, ldT=5)
    assert st == 0 and info == 0
    # ngal = 0: the factor is computed, no target is solved
    n = 64
    S = spd(n, 6)
    dC, dT = dev(np.tril(S)), dev(np.ones((2, n)))
    st, info = noalloc(n, 2, dC, dT, ngal=0)
    assert st == 0 and info == 0
    assert np.allclose(np.tril(host(dC)), np.linalg.cholesky(S), atol=1e-12)
    assert np.all(host(dT) == 1.0)
