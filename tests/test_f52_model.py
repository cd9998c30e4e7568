"""Exact-integer model of the FP64-pipe product (csrc/zg_field_f64.cuh), Fq and Fr.

The device routine splits every 52 x 52-bit limb product with two FMAs and
sums the bit patterns of the halves in 64-bit integer columns. This test
restates each step with Python integers (the FMA steps are exact by
construction, so their integer values are what the device computes) and
checks the result against a * b / 2^256 mod p, the value of Fp::mul, plus the
bounds the device code relies on, for both BN254 moduli (the MSM uses it over
Fq, the NTTs over Fr). The device routine itself is checked against Fq::mul
and Fr::mul on the GPU by zg_selftest (checks 1 and 8).
"""
import random

import pytest

import zgo

M52 = (1 << 52) - 1
M64 = (1 << 64) - 1
KL = 0x4330000000000000  # bit pattern of the double 2^52
KH = 0x4670000000000000  # bit pattern of the double 2^104
# the constants written in Limbs52<FqCfg> / Limbs52<FrCfg>
DEVICE_CONSTS = {
    zgo.Q_MOD: ([0x8C16D87CFD47, 0x916871CA8D3C2, 0x181585D97816A, 0xA029B85045B68, 0x30644E72E131],
                0x20782E4866389, 0x782E4866389),
    zgo.R_MOD: ([0x1F593F0000001, 0x4879B9709143E, 0x181585D2833E8, 0xA029B85045B68, 0x30644E72E131],
                0x1F593EFFFFFFF, 0xF593EFFFFFFF),
}


def nprod(c):
    return 0 if c < 0 or c > 8 else (c + 1 if c <= 4 else 9 - c)


def col_init(c):
    return (-(2 * nprod(c)) * KL - (2 * nprod(c - 1)) * KH) & M64


def fma_split(a, b, bits=52):
    """h = fma_rz(a, b, 2^(bits+52)), l = fma(a, b, 2^(bits+52) + 2^bits - h):
    the integer halves of a*b the device FMAs produce (exact)."""
    assert 0 <= a < 1 << 52 and 0 <= b < 1 << 52 and a * b < 1 << (bits + 52)
    return (a * b) >> bits, (a * b) & ((1 << bits) - 1)


def mont_mul_model(P, a, b, trace=None):
    PL = [(P >> (52 * k)) & M52 for k in range(5)]
    PINV52 = (-pow(P, -1, 1 << 52)) % (1 << 52)
    PINV48 = PINV52 & ((1 << 48) - 1)
    A = [(a >> (52 * k)) & M52 for k in range(5)]
    B = [(b >> (52 * k)) & M52 for k in range(5)]
    t = [col_init(c) for c in range(10)]
    true = [0] * 10  # the column values without offsets, for the bound check

    def add(i, j, x, y):
        hi, lo = fma_split(x, y)
        t[i + j] = (t[i + j] + KL + lo) & M64
        t[i + j + 1] = (t[i + j + 1] + KH + hi) & M64
        true[i + j] += lo
        true[i + j + 1] += hi

    for i in range(5):
        for j in range(5):
            add(i, j, A[i], B[j])
    for i in range(4):
        hi, m = fma_split(t[i] & M52, PINV52)
        for j in range(5):
            add(i, j, m, PL[j])
        assert t[i] & M52 == 0
        c = t[i] >> 52
        t[i + 1] = (t[i + 1] + c) & M64
        true[i + 1] += c
    hi, m = fma_split(t[4] & ((1 << 48) - 1), PINV48, bits=48)
    for j in range(5):
        add(4, j, m, PL[j])
    assert t[4] & ((1 << 48) - 1) == 0
    top = (t[4] >> 48) & 15
    for c in range(5, 10):
        t[c] = (t[c] + (t[c - 1] >> 52)) & M64
    n = [t[c] & M52 for c in range(5, 9)] + [t[9]]
    r = top + sum(x << (4 + 52 * k) for k, x in enumerate(n))
    if trace is not None:
        trace.append(max(true))
    return r - P if r >= P else r


@pytest.mark.parametrize("P", [zgo.Q_MOD, zgo.R_MOD])
def test_device_constants(P):
    limbs, pinv52, pinv48 = DEVICE_CONSTS[P]
    assert sum(x << (52 * k) for k, x in enumerate(limbs)) == P
    assert (P * pinv52 + 1) % (1 << 52) == 0
    assert (P * pinv48 + 1) % (1 << 48) == 0


@pytest.mark.parametrize("P", [zgo.Q_MOD, zgo.R_MOD])
def test_model_matches_montgomery_product(P):
    rng = random.Random(52)
    edge = [0, 1, 2, P - 1, P - 2, (1 << 253) - 1, 1 << 200]
    pairs = [(x, y) for x in edge for y in edge]
    pairs += [(rng.randrange(P), rng.randrange(P)) for _ in range(3000)]
    rinv = pow(2, -256, P)
    peak = []
    for a, b in pairs:
        assert mont_mul_model(P, a, b, peak) == a * b * rinv % P
    # column sums stay far below 2^64 (the device accumulates modulo 2^64)
    assert max(peak) < 1 << 58
