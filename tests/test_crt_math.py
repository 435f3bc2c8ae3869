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
