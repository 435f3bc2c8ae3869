"""The mixed path's refinement residual E = Ctm - R sym(Cmm) on its own
(moao_debug_residual) and inside the reconstructor.

* scheme 1 (CRT products, the default) against the exact product of the same
  35-bit rounded operands, computed in Python integers: equal up to the
  rounding of the 128-bit result to FP64 (1 ulp of the product) and of the
  final subtraction (1 ulp of E);
* both schemes against the FP64 product within the operand rounding,
  2^-35 (max|R_r.| sum_k |S_kc| + max|S_.c| sum_k |R_rk|) per element;
* the reconstructor's R with either scheme within 1e-5 of the FP64 path, and
  the CRT residual at least as small as the slice products'.
"""
import numpy as np
import pytest

import moao_b200 as M
from moao_b200._lib import check, lib

from test_gpu_mixed import case, dev, host

pytestmark = pytest.mark.gpu


def residual(ctx, scheme, R, Cmm, Ctm):
    m, n = R.shape
    dR, dC, dT = dev(R), dev(Cmm), dev(Ctm)
    dE = dev(np.zeros((m, n)))
    check(lib().moao_debug_residual(ctx.handle, scheme, m, n, dR.data_ptr(), m, dC.data_ptr(), n,
                                    dT.data_ptr(), m, dE.data_ptr(), m), "moao_debug_residual")
    return host(dE)


def problem(m, n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, n + 3))
    D = np.exp2(rng.integers(-6, 6, n))  # column (and row) scales of S: D S0 D
    S = (X @ X.T / n + np.eye(n)) * D[:, None] * D[None, :]
    R = rng.standard_normal((m, n)) * np.exp2(rng.integers(-12, 12, m))[:, None]
    Ctm = R @ S + 1e-6 * rng.standard_normal((m, n)) * np.abs(R @ S).max()
    Cmm = np.tril(S) + np.triu(rng.standard_normal((n, n)), 1) * 1e3  # upper part is never read
    return R, S, Cmm, Ctm


def exps(mx):
    return np.where(mx > 0, np.frexp(mx)[1], 0)


def test_crt_residual_is_the_exact_product_of_the_rounded_operands(ctx):
    m, n = 48, 300
    R, S, Cmm, Ctm = problem(m, n, 1)
    e = exps(np.abs(R).max(1))
    f = exps(np.abs(S).max(0))
    Rq = np.rint(R * np.exp2(34 - e)[:, None]).astype(np.int64)
    Sq = np.rint(S * np.exp2(34 - f)[None, :]).astype(np.int64)
    P = Rq.astype(object) @ Sq.astype(object)
    val = np.array([[np.ldexp(float(P[i, j]), int(e[i] + f[j] - 68)) for j in range(n)]
                    for i in range(m)])
    want = Ctm - val
    got = residual(ctx, 1, R, Cmm, Ctm)
    # one rounding of the 128-bit product to FP64 (within 1 ulp of val) and one
    # of the subtraction (ulp of E)
    tol = 2 * np.spacing(np.abs(val)) + 2 * np.spacing(np.abs(want)) + 1e-300
    ratio = np.abs(got - want) / tol
    i, j = np.unravel_index(np.argmax(ratio), ratio.shape)
    assert ratio.max() <= 1.0, (i, j, got[i, j], want[i, j], val[i, j])


@pytest.mark.parametrize("m,n", [(300, 2000), (130, 4100)])
def test_both_schemes_within_the_operand_rounding(ctx, m, n):
    R, S, Cmm, Ctm = problem(m, n, 2 + m)
    exact = Ctm - R @ S
    aR, aS = np.abs(R), np.abs(S)
    bound = 2.0 ** -35 * (aR.max(1)[:, None] * aS.sum(0)[None, :] +
                          aS.max(0)[None, :] * aR.sum(1)[:, None])
    e1 = residual(ctx, 1, R, Cmm, Ctm)
    e0 = residual(ctx, 0, R, Cmm, Ctm)
    assert np.all(np.abs(e1 - exact) <= 1.01 * bound + 1e-12 * np.abs(exact))
    # the slice products also drop the pairs whose slice indices sum past 6
    assert np.all(np.abs(e0 - exact) <= 4 * bound + 1e-12 * np.abs(exact))


@pytest.mark.parametrize("scheme", ["crt", "slices"])
def test_reconstructor_with_either_residual(ctx, scheme):
    import torch
    nm, nts, Cmm, Ctm = case("elt16")
    want = np.linalg.solve(np.tril(Cmm) + np.tril(Cmm, -1).T, Ctm.T).T
    ctx.set_residual_scheme(scheme)
    try:
        dC, dT = dev(Cmm), dev(Ctm)
        rep = M.reconstructor(nm, nts, dC, nm, dT, nts, 1, prec="mixed", ctx=ctx)
    finally:
        ctx.set_residual_scheme("crt")
    got = host(dT)
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err <= 1e-5, (scheme, err)
    assert rep["refine_steps"] >= 1 and rep["refine_resid"] < 1e-3


@pytest.mark.parametrize("name", ["elt16", "elt24"])
def test_crt_residual_with_declared_offsets(cuda, name):
    """The model's LGS offsets declared (the residual's operands are then
    sym(Cmm) minus the offsets, whose part of R Cmm comes from FP64 range sums):
    R within 1e-5 of the oracle with either residual, and the CRT residual's R
    at least as accurate as the slice products' (it drops no terms)."""
    import oracle as O
    import systems
    sf, af = systems.files(name)
    t = M.Tomo(sf, af)
    g = O.Geometry.from_tomo(t)
    nm, nts = g.nmeas, g.nmeasts
    Cmm = O.matcov(g, nm, nm, 0, 0, 1, nthreads=16)
    Ctm = O.matcov(g, nts, nm, 0, 0, 3, nthreads=16)
    _, R_ref, _ = O.reconstructor(Cmm, Ctm)
    errs = {}
    for scheme in ("crt", "slices"):
        c2 = M.Context(0)
        c2.set_offsets_from_tomo(t)
        c2.set_residual_scheme(scheme)
        dC, dT = dev(Cmm), dev(Ctm)
        M.reconstructor(nm, nts, dC, nm, dT, nts, 1, prec="mixed", ctx=c2)
        c2.synchronize()
        errs[scheme] = O.rel_fro(host(dT), R_ref)
        c2.close()
    assert errs["crt"] <= 1e-5 and errs["slices"] <= 1e-5, errs
    assert errs["crt"] <= 1.05 * errs["slices"], errs
