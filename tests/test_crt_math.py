"""The arithmetic of the CRT refinement residual (mixed_kernels.cu), restated
in Python integers: centred residues, centred mixed-radix digits by Garner's
method with the kernel's inverse table, and reconstruction; the moduli are
pairwise coprime and cover the products the residual forms (nmeas up to
131,071 at 5 slices). The kernels reduce in floating point, x - M rint(x / M)
in FP64 for the operands and the Garner steps in FP32; both give exactly the
centred integer residues, checked here with numpy's FP64 and FP32 on the
boundary cases."""
import math
import random

import numpy as np

MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211]


def cmod(a, m):
    """C's a % m (the result keeps the sign of a)."""
    return -((-a) % m) if a < 0 else a % m


def residues(x, nmod):
    """The kernel's residues: low byte for 256, x = h 2^18 + l for the odd moduli."""
    r = [((x & 0xFF) ^ 0x80) - 0x80]
    h, l = x >> 18, x & 0x3FFFF
    for m in MODULI[1:nmod]:
        t = cmod(cmod(h, m) * (2 ** 18 % m) + l, m)
        if t > m // 2:
            t -= m
        elif t < -(m // 2):
            t += m
        r.append(t)
    return r


def garner(z, nmod):
    """z: residues in [0, m_i); returns the centred value."""
    v = [z[0] - 256 if z[0] >= 128 else z[0]]
    for i in range(1, nmod):
        m = MODULI[i]
        t = z[i]
        for j in range(i):
            inv = pow(MODULI[j] % m, -1, m)
            t = cmod((t - v[j]) * inv, m)
        if t > m // 2:
            t -= m
        elif t < -(m // 2):
            t += m
        v.append(t)
    p = 0
    for i in reversed(range(nmod)):
        p = p * MODULI[i] + v[i]
    return p


def moduli_for(ns, K):
    if K < 1 or K >= 1 << 17:
        return 0
    need = math.log2(K) + 2 * (7 * ns - 1) + 1
    have = 0.0
    for i, m in enumerate(MODULI):
        have += math.log2(m)
        if have > need + 1e-9:
            return i + 1
    return 0


def test_moduli_pairwise_coprime():
    for i in range(len(MODULI)):
        for j in range(i):
            assert math.gcd(MODULI[i], MODULI[j]) == 1, (MODULI[i], MODULI[j])


def test_residues_match_python_modulo():
    rng = random.Random(1)
    for _ in range(2000):
        x = rng.randint(-(2 ** 41), 2 ** 41)
        r = residues(x, 13)
        for m, ri in zip(MODULI, r):
            assert (ri - x) % m == 0 and -128 <= ri <= 127


def test_exact_products_reconstructed():
    """Sums of K products of 35-bit integers come back exactly from their
    residues modulo the moduli the residual uses."""
    rng = random.Random(2)
    for K in (1, 7, 1000, 47552, 131071):
        nmod = moduli_for(5, K)
        assert nmod > 0
        M = math.prod(MODULI[:nmod])
        for _ in range(30):
            # the extreme sums: K equal products of +-2^34 and random ones
            s = rng.choice([K * 2 ** 68, -K * 2 ** 68,
                            sum(rng.randint(-2 ** 34, 2 ** 34) * rng.randint(-2 ** 34, 2 ** 34)
                                for _ in range(min(K, 50))) * (K // min(K, 50))])
            assert abs(s) < M // 2
            z = [s % m for m in MODULI[:nmod]]
            assert garner(z, nmod) == s


def test_moduli_needed_at_elt_size():
    assert moduli_for(5, 47552) == 11       # 11 GEMMs instead of 15 slice pairs
    assert moduli_for(5, 131072) == 0       # int32 sums would overflow: slice products
    assert moduli_for(6, 47552) == 13


def test_floating_point_reductions_are_exact():
    """x - M rint(x / M) in FP64 for |x| <= 2^41 and the FP32 Garner step
    y - M rint(y / M) for |y| < 2^17 equal the centred integer residues."""
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.integers(-2 ** 41, 2 ** 41, 20000),
                         np.array([2 ** 41, -2 ** 41, 0, 1, -1, 2 ** 34, -2 ** 34])])
    for m in MODULI[1:]:
        x = xs.astype(np.float64)
        r = np.fma(-float(m), np.rint(x * (1.0 / m)), x) if hasattr(np, "fma") else \
            x - m * np.rint(x * (1.0 / m))
        want = np.array([((int(v) + m // 2) % m) - m // 2 for v in xs])
        assert np.array_equal(r.astype(np.int64), want), m
        y = np.arange(-(2 ** 17) + 1, 2 ** 17, dtype=np.int64)
        yf = y.astype(np.float32)
        inv = np.float32(1.0) / np.float32(m)
        t = yf - np.float32(m) * np.rint(yf * inv)   # every product and difference is exact
        wy = ((y + m // 2) % m) - m // 2
        assert np.array_equal(t.astype(np.int64), wy), m


def test_library_moduli_count_matches(built):
    """The library's own count (moao_debug_crt_moduli, host code) equals this
    restatement's, the fallback to slice products included."""
    from moao_b200._lib import lib
    for ns in range(1, 7):
        for K in (1, 2, 100, 4096, 47552, 100000, 131071, 131072, 10 ** 6):
            assert lib().moao_debug_crt_moduli(ns, K) == moduli_for(ns, K), (ns, K)


def test_kernel_reconstruction_path_in_floating_point():
    """The reconstruction as crt_combine_kernel runs it, restated in numpy:
    Garner digits by FP32 steps y = (t - v_j) m_j^-1, t = y - M round(y / M)
    (round by the 1.5 * 2^23 constant), then P = L + W_7 H from two int64
    Horner halves joined in FP64. Equal to the exact value within 2 ulp."""
    rng = np.random.default_rng(7)
    nmod = 11
    M = math.prod(MODULI[:nmod])
    # sums of K = 47552 products of 35-bit integers, spread over the whole range
    exact = [int(rng.integers(-2 ** 62, 2 ** 62)) * int(rng.integers(1, 2 ** 21)) for _ in range(3000)]
    exact += [0, 1, -1, 47552 * 2 ** 68, -47552 * 2 ** 68, M // 2 - 1, -(M // 2) + 1]
    magic = np.float32(12582912.0)
    z = np.array([[p % m for m in MODULI[:nmod]] for p in exact], dtype=np.float32)
    v = np.zeros_like(z)
    v[:, 0] = np.where(z[:, 0] >= 128, z[:, 0] - 256, z[:, 0])
    for i in range(1, nmod):
        m = MODULI[i]
        inv_m = np.float32(1.0) / np.float32(m)
        t = z[:, i].copy()
        for j in range(i):
            y = (t - v[:, j]) * np.float32(pow(MODULI[j] % m, -1, m))
            q = (y * inv_m + magic) - magic
            t = y - np.float32(m) * q
        v[:, i] = t
    vi = v.astype(np.int64)
    L = np.zeros(len(exact), dtype=np.int64)
    for i in reversed(range(7)):
        L = L * MODULI[i] + vi[:, i]
    H = np.zeros(len(exact), dtype=np.int64)
    for i in reversed(range(7, nmod)):
        H = H * MODULI[i] + vi[:, i]
    w7 = float(math.prod(MODULI[:7]))
    assert w7 == math.prod(MODULI[:7])  # exact in FP64
    for p, l, h in zip(exact, L.tolist(), H.tolist()):
        assert l + math.prod(MODULI[:7]) * h == p            # the digits are exact
        got = float(h) * w7 + float(l)                       # two roundings (the kernel fuses one)
        want = float(p)
        assert abs(got - want) <= 2 * np.spacing(abs(want)) + 0.0, (p, got, want)
