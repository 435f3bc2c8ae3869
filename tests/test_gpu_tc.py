"""The tcgen05 tensor-core GEMM (TMA + TMEM) in isolation, through the C ABI.

* bf16 -> fp32: compared with torch's fp32 product of the same bf16 values;
  tolerance 1e-5 relative (both accumulate exactly-representable products in
  fp32, in different orders).
* int8 -> int32 -> scaled fp64 (Ozaki slices): compared with an exact int64
  product; tolerance 1e-15 relative (one fp64 rounding per added term).
"""
import ctypes as C

import numpy as np
import pytest

import moao_b200 as M
from moao_b200._lib import check, lib

pytestmark = pytest.mark.gpu


def _ints(xs):
    return (C.c_int * len(xs))(*xs)


def tc_bf16(ctx, A, B, Cm, pairs, alpha=1.0, beta=0.0, lower=0):
    """A: [na, M, Kp] bf16, B: [nb, N, Kp] bf16 (row-major, Kp padded), Cm: [N, M] f32 (col-major C)."""
    na, Mr, Kp = A.shape
    nb, Nr, _ = B.shape
    pa, pb = _ints([p[0] for p in pairs]), _ints([p[1] for p in pairs])
    check(lib().moao_debug_tc_gemm(ctx.handle, 0, Mr, Nr, Kp, A.data_ptr(), Kp, na, B.data_ptr(), Kp,
                                   nb, len(pairs), pa, pb, Cm.data_ptr(), Mr, alpha, beta, None,
                                   None, 0, lower), "tc_gemm")


@pytest.mark.parametrize("Mr,Nr,K", [(128, 128, 64), (256, 384, 512), (300, 200, 136), (1000, 77, 1000)])
def test_bf16_single_product(ctx, Mr, Nr, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(1)
    A = torch.randn(1, Mr, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(1, Nr, K, device="cuda", generator=g).to(torch.bfloat16)
    Cm = torch.randn(Nr, Mr, device="cuda", generator=g)
    want = (0.5 * (A[0].float() @ B[0].float().T) + 2.0 * Cm.T).T.contiguous()
    tc_bf16(ctx, A, B, Cm, [(0, 0)], alpha=0.5, beta=2.0)
    err = (Cm - want).abs().max() / want.abs().max()
    assert err < 1e-5, float(err)


def test_bf16_split_products_and_lower(ctx):
    import torch
    g = torch.Generator(device="cuda").manual_seed(2)
    Mr = Nr = 384
    K = 256
    X = torch.randn(Mr, K, device="cuda", generator=g, dtype=torch.float64)
    hi = X.to(torch.bfloat16)
    lo = (X - hi.double()).to(torch.bfloat16)
    A = torch.stack([hi, lo])
    Cm = torch.zeros(Nr, Mr, device="cuda")
    tc_bf16(ctx, A, A, Cm, [(0, 0), (0, 1), (1, 0)], alpha=1.0, beta=0.0, lower=1)
    h, l = hi.double(), lo.double()
    want = (h @ h.T + h @ l.T + l @ h.T)
    got = Cm.T.double()
    low = torch.tril(torch.ones(Mr, Nr, device="cuda", dtype=torch.bool))
    err = ((got - want).abs() * low).max() / want.abs().max()
    assert err < 1e-5, float(err)  # fp32 accumulation over K = 768
    assert float(got[~low].abs().max()) == 0.0, "wrote above the diagonal"
    # the split product is far more accurate than a single bf16 product
    exact = X @ X.T
    assert float(((got - exact) * low).abs().max() / exact.abs().max()) < 1e-4


@pytest.mark.parametrize("Mr,Nr,K,pairs", [(128, 128, 128, [(0, 0)]), (200, 330, 384, [(0, 1), (1, 0)]),
                                           (640, 256, 4096, [(0, 2), (1, 1), (2, 0)])])
def test_int8_scaled_fp64(ctx, Mr, Nr, K, pairs):
    import torch
    rng = np.random.default_rng(3)
    na = max(p[0] for p in pairs) + 1
    nb = max(p[1] for p in pairs) + 1
    A = rng.integers(-64, 65, size=(na, Mr, K), dtype=np.int8)
    B = rng.integers(-64, 65, size=(nb, Nr, K), dtype=np.int8)
    er = rng.integers(-20, 20, size=Mr).astype(np.int32)
    ec = rng.integers(-20, 20, size=Nr).astype(np.int32)
    shift = -13
    C0 = rng.standard_normal((Mr, Nr))
    acc = sum(A[p].astype(np.int64) @ B[q].astype(np.int64).T for p, q in pairs)
    want = C0 + acc.astype(np.float64) * np.ldexp(1.0, er[:, None] + ec[None, :] + shift)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    dC = torch.from_numpy(np.ascontiguousarray(C0.T)).cuda()
    der, dec = torch.from_numpy(er).cuda(), torch.from_numpy(ec).cuda()
    pa, pb = _ints([p[0] for p in pairs]), _ints([p[1] for p in pairs])
    check(lib().moao_debug_tc_gemm(ctx.handle, 1, Mr, Nr, K, dA.data_ptr(), K, na, dB.data_ptr(), K, nb,
                                   len(pairs), pa, pb, dC.data_ptr(), Mr, 1.0, 0.0, der.data_ptr(),
                                   dec.data_ptr(), shift, 0), "tc_gemm int8")
    got = dC.cpu().numpy().T
    assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300)) < 1e-15
