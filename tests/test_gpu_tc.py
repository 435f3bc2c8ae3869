"""The tcgen05 tensor-core GEMM (TMA + TMEM) in isolation, through the C ABI.

* bf16 -> fp32: compared with torch's fp32 product of the same bf16 values;
  tolerance 1e-5 relative (both accumulate exactly-representable products in
  fp32, in different orders).
* int8 -> int32 -> scaled fp64 (Ozaki slices): compared with an exact int64
  product; tolerance 1e-15 relative (one fp64 rounding per added term).

Every case runs on single CTAs (128 x 256 tiles) and on CTA pairs (256 x 256
tiles, M = 256 MMAs; used where M > 128): sizes include a second B box wholly
past N (N = 77) and A rows of the second CTA partly past M.
"""
import ctypes as C

import numpy as np
import pytest

import moao_b200 as M
from moao_b200._lib import check, lib

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[0, 1], ids=["cta", "pair"])
def tcx(ctx, request):
    ctx.set_tc_pair(request.param)
    yield ctx
    ctx.set_tc_pair(False)


def _ints(xs):
    return (C.c_int * len(xs))(*xs)


def tc_bf16(tcx, A, B, Cm, pairs, alpha=1.0, beta=0.0, lower=0):
    """A: [na, M, Kp] bf16, B: [nb, N, Kp] bf16 (row-major, Kp padded), Cm: [N, M] f32 (col-major C)."""
    na, Mr, Kp = A.shape
    nb, Nr, _ = B.shape
    pa, pb = _ints([p[0] for p in pairs]), _ints([p[1] for p in pairs])
    check(lib().moao_debug_tc_gemm(tcx.handle, 0, Mr, Nr, Kp, A.data_ptr(), Kp, na, B.data_ptr(), Kp,
                                   nb, len(pairs), pa, pb, Cm.data_ptr(), Mr, alpha, beta, None,
                                   None, 0, lower), "tc_gemm")


@pytest.mark.parametrize("Mr,Nr,K", [(128, 128, 64), (256, 384, 512), (300, 200, 136), (1000, 77, 1000)])
def test_bf16_single_product(tcx, Mr, Nr, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(1)
    A = torch.randn(1, Mr, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(1, Nr, K, device="cuda", generator=g).to(torch.bfloat16)
    Cm = torch.randn(Nr, Mr, device="cuda", generator=g)
    want = (0.5 * (A[0].float() @ B[0].float().T) + 2.0 * Cm.T).T.contiguous()
    tc_bf16(tcx, A, B, Cm, [(0, 0)], alpha=0.5, beta=2.0)
    err = (Cm - want).abs().max() / want.abs().max()
    assert err < 1e-5, float(err)


def test_bf16_split_products_and_lower(tcx):
    import torch
    g = torch.Generator(device="cuda").manual_seed(2)
    Mr = Nr = 384
    K = 256
    X = torch.randn(Mr, K, device="cuda", generator=g, dtype=torch.float64)
    hi = X.to(torch.bfloat16)
    lo = (X - hi.double()).to(torch.bfloat16)
    A = torch.stack([hi, lo])
    Cm = torch.zeros(Nr, Mr, device="cuda")
    tc_bf16(tcx, A, A, Cm, [(0, 0), (0, 1), (1, 0)], alpha=1.0, beta=0.0, lower=1)
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
def test_int8_scaled_fp64(tcx, Mr, Nr, K, pairs):
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
    check(lib().moao_debug_tc_gemm(tcx.handle, 1, Mr, Nr, K, dA.data_ptr(), K, na, dB.data_ptr(), K, nb,
                                   len(pairs), pa, pb, dC.data_ptr(), Mr, 1.0, 0.0, der.data_ptr(),
                                   dec.data_ptr(), shift, 0), "tc_gemm int8")
    got = dC.cpu().numpy().T
    assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300)) < 1e-15


def test_f16_scaled_products(tcx):
    """fp16 operands stored scaled by 2^-e per row (two slices, 3 products): the
    epilogue's 2^(erow[r] + ecol[c]) restores the product of the unscaled values
    to ~2^-22 relative; rows span 2^-30..2^20 in magnitude."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(5)
    Mr, Nr, K = 320, 260, 192
    X = torch.randn(Mr, K, device="cuda", generator=g, dtype=torch.float64)
    Y = torch.randn(Nr, K, device="cuda", generator=g, dtype=torch.float64)
    X *= torch.pow(2.0, torch.randint(-30, 20, (Mr, 1), device="cuda", generator=g).double())
    Y *= torch.pow(2.0, torch.randint(-30, 20, (Nr, 1), device="cuda", generator=g).double())

    def slices(Z):
        e = torch.frexp(Z.abs().amax(dim=1)).exponent.to(torch.int32) - 14
        s = Z * torch.pow(2.0, -e.double())[:, None]
        hi = s.to(torch.float16)
        lo = (s - hi.double()).to(torch.float16)
        return torch.stack([hi, lo]).contiguous(), e.contiguous()
    A, ea = slices(X)
    B, eb = slices(Y)
    Cm = torch.zeros(Nr, Mr, device="cuda")
    pairs = [(1, 0), (0, 1), (0, 0)]
    check(lib().moao_debug_tc_gemm(tcx.handle, 2, Mr, Nr, K, A.data_ptr(), K, 2, B.data_ptr(), K, 2,
                                   3, _ints([p[0] for p in pairs]), _ints([p[1] for p in pairs]),
                                   Cm.data_ptr(), Mr, -1.0, 0.0, ea.data_ptr(), eb.data_ptr(), 0, 0),
          "tc_gemm f16")
    want = -(X @ Y.T)
    got = Cm.T.double()
    # error relative to each entry's natural scale |x_r| |y_c| sqrt(K)
    scale = X.abs().amax(1)[:, None] * Y.abs().amax(1)[None, :] * K ** 0.5
    err = ((got - want).abs() / scale).max().item()
    assert err < 1e-5, err


@pytest.mark.parametrize("kind,lower", [(0, 1), (2, 0), (2, 1)])
def test_accumulate_epilogue_through_tma_reduce(tcx, kind, lower):
    """beta = 1 with a 16-byte aligned C and ldc % 4 == 0 takes the TMA reduce-add
    epilogue: C += alpha * products, entries above the diagonal (lower = 1) and
    outside M x N (M, N not multiples of 32) left untouched."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(7 + kind + lower)
    Mr, Nr, K = 300, 220 if not lower else 300, 128
    ldc = 304
    dt = torch.bfloat16 if kind == 0 else torch.float16
    A = torch.randn(1, Mr, K, device="cuda", generator=g).to(dt)
    B = torch.randn(1, Nr, K, device="cuda", generator=g).to(dt)
    Cfull = torch.randn(Nr + 1, ldc, device="cuda", generator=g)   # column-major, ld 304, spare column
    C0 = Cfull.clone()
    ea = torch.full((Mr,), 1, dtype=torch.int32, device="cuda")
    eb = torch.full((Nr,), -2, dtype=torch.int32, device="cuda")
    exps = kind == 2
    check(lib().moao_debug_tc_gemm(tcx.handle, kind, Mr, Nr, K, A.data_ptr(), K, 1, B.data_ptr(), K, 1,
                                   1, _ints([0]), _ints([0]), Cfull.data_ptr(), ldc, -0.5, 1.0,
                                   ea.data_ptr() if exps else None, eb.data_ptr() if exps else None,
                                   0, lower), "tc_gemm reduce")
    prod = (A[0].float() @ B[0].float().T) * (0.5 if exps else 1.0)   # 2^(1-2) with exponents
    want = C0.clone()
    upd = -0.5 * prod.T                                                # [Nr, Mr] in C's layout
    if lower:
        r = torch.arange(Mr, device="cuda")[None, :]
        c = torch.arange(Nr, device="cuda")[:, None]
        upd = torch.where(r >= c, upd, torch.zeros_like(upd))
    want[:Nr, :Mr] += upd
    err = (Cfull - want).abs().max() / upd.abs().max()
    assert err < 1e-5, float(err)
    assert torch.equal(Cfull[:, Mr:], C0[:, Mr:]) and torch.equal(Cfull[Nr:], C0[Nr:])


@pytest.mark.parametrize("Mr,Nr,lower", [(2600, 2600, 0), (5000, 900, 0), (4700, 4700, 1)])
def test_more_tiles_than_resident_ctas(tcx, Mr, Nr, lower):
    """More tiles than resident CTAs (pairs): every CTA walks several tiles, so
    both accumulator buffers are reused and the epilogues hand them back across
    the pair; M spans several bands of the tile walk (2,048 rows each), the
    lower case with bands that end inside the triangle. Entries above the
    diagonal stay untouched."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(11 + Mr + lower)
    K = 128
    A = torch.randn(1, Mr, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(1, Nr, K, device="cuda", generator=g).to(torch.bfloat16)
    Cm = torch.full((Nr, Mr), 7.0, device="cuda")
    tc_bf16(tcx, A, B, Cm, [(0, 0)], alpha=1.0, beta=0.0, lower=lower)
    want = (A[0].float() @ B[0].float().T).T
    if lower:
        r = torch.arange(Mr, device="cuda")[None, :]
        c = torch.arange(Nr, device="cuda")[:, None]
        low = r >= c
        assert bool((Cm[~low] == 7.0).all()), "wrote above the diagonal"
        want = torch.where(low, want, Cm)
    err = (Cm - want).abs().max() / want.abs().max()
    assert err < 1e-5, float(err)
