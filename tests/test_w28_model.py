"""Exact-integer model of the 28-bit-limb Montgomery product
(csrc/zg_field_w28.cuh), for both BN254 moduli (Fq and Fr).

The routine sums 28 x 28-bit limb products in 64-bit columns without carry
flags and reduces 9 x 28 + 4 = 256 bits Montgomery-style. This test restates
each step with Python integers, asserts that no 64-bit column overflows and
that the repacked result stays below 2p, and checks the value against
a * b / 2^256 mod p (the value of Fq::mul / Fr::mul). The device code itself
is checked against Fq::mul on the GPU by zg_selftest.
"""
import random

import pytest

import zgo

M28 = (1 << 28) - 1


def split(a):
    return [(a >> (28 * k)) & M28 for k in range(10)]


def mont_mul_model(a, b, P):
    P28 = [(P >> (28 * k)) & M28 for k in range(10)]
    PINV28 = (-pow(P, -1, 1 << 28)) % (1 << 28)
    PINV4 = (-pow(P, -1, 16)) % 16
    x, y = split(a), split(b)
    t = [0] * 20
    for i in range(10):
        for j in range(10):
            t[i + j] += x[i] * y[j]
    for i in range(9):
        m = ((t[i] & 0xFFFFFFFF) * PINV28) & M28
        for j in range(10):
            t[i + j] += m * P28[j]
        assert t[i] & M28 == 0
        t[i + 1] += t[i] >> 28
    m = ((t[9] & 0xFFFFFFFF) * PINV4) & 15
    for j in range(10):
        t[9 + j] += m * P28[j]
    assert all(v < 1 << 64 for v in t)
    r, c = [], 0
    for k in range(10):
        c += t[9 + k]
        r.append(c & M28)
        c >>= 28
    assert c == 0 and r[0] & 15 == 0
    v = sum(r[k] << (28 * k) for k in range(10)) >> 4
    assert v < 2 * P
    return v - P if v >= P else v


@pytest.mark.parametrize("P,pinv28,pinv4", [(zgo.Q_MOD, 0x4866389, 0x9), (zgo.R_MOD, 0xFFFFFFF, 0xF)])
def test_constants(P, pinv28, pinv4):
    """The constants csrc/zg_field_w28.cuh writes out."""
    P28 = [(P >> (28 * k)) & M28 for k in range(10)]
    assert sum(p << (28 * k) for k, p in enumerate(P28)) == P
    assert (P * pinv28 + 1) % (1 << 28) == 0 and (P * pinv4 + 1) % 16 == 0


@pytest.mark.parametrize("P", [zgo.Q_MOD, zgo.R_MOD])
def test_matches_montgomery_product(P):
    r_inv = pow(1 << 256, -1, P)
    rnd = random.Random(28)
    edges = [0, 1, 2, P - 1, P - 2, (1 << 253) % P, (P - 1) // 2]
    vals = edges + [rnd.randrange(P) for _ in range(400)]
    for k, a in enumerate(vals):
        b = vals[(k * 7 + 3) % len(vals)]
        assert mont_mul_model(a, b, P) == a * b * r_inv % P
    for a in edges:
        for b in edges:
            assert mont_mul_model(a, b, P) == a * b * r_inv % P
