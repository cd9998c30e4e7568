"""CPU tests of the oracle (the checker): pinned against an independent pure-
Python restatement (tests/golden/), Python big integers, hashlib's SHA3
permutation, and the relations the reference's own tests check."""
import hashlib
import json
import os
import random
import sys

import numpy as np
import pytest

import zgo

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as mg  # noqa: E402

R_MOD, Q_MOD = zgo.R_MOD, zgo.Q_MOD
GOLDEN = json.load(open(os.path.join(HERE, "golden", "encode_3x5.json")))


def fr_bytes(vals):
    return b"".join(v.to_bytes(32, "little") for v in vals)


def fr_vals(buf):
    return [int.from_bytes(buf[32 * i:32 * i + 32], "little") for i in range(len(buf) // 32)]


# ---- pins --------------------------------------------------------------------
def test_keccak_permutation_matches_sha3(oracle):
    rng = random.Random(1)
    for n in (0, 1, 31, 32, 64, 135, 136, 137, 256, 300):
        m = bytes(rng.randrange(256) for _ in range(n))
        assert oracle.keccak256(m, pad=0x06) == hashlib.sha3_256(m).digest()


def test_golden_vectors(oracle):
    v = GOLDEN["vectors"]
    for m, h in v["keccak256"].items():
        assert oracle.keccak256(bytes.fromhex(m)).hex() == h
    for k, s in v["g1_mul"].items():
        assert oracle.g1_mul_gen(int(k, 16)).hex() == s
    assert v["coset_factor_16_1_eq_root_32"]
    assert oracle.root_of_unity(28) == int(v["root_of_unity_28"], 16)


# Published constants of the third-party crates the reference computes with,
# written out as literals: the oracle is pinned to the published values, not
# to a recomputation of its own.
# ark-bn254 0.4.0 FrConfig::TWO_ADIC_ROOT_OF_UNITY (TWO_ADICITY = 28)
ARK_BN254_FR_TWO_ADIC_ROOT = 19103219067921713944291392827692070036145651957329286315305642004821462161904
# the BN254 generators of ark-bn254 0.4.0 (g1::G1_GENERATOR_X/Y, g2::G2_GENERATOR_X/Y),
# the EIP-196 / EIP-197 generators: x = c0 + c1 u over Fq2 = Fq[u] / (u^2 + 1)
G1_GEN = (1, 2)
G2_GEN_X = (10857046999023057135944570762232829481370756359578518086990519993285655852781,
            11559732032986387107991004021392285783925812861821192530917403151452391805634)
G2_GEN_Y = (8495653923123431417604973247489272438418190587263600148770280649306958101930,
            4082367875863433681332203403145435568316851327593401208105741076214120093531)
# ark-serialize 0.4 SWFlags in the top bits of the last byte
SW_FLAG_Y_NEGATIVE, SW_FLAG_INFINITY = 0x80, 0x40


def test_published_constants(oracle):
    assert oracle.root_of_unity(28) == ARK_BN254_FR_TWO_ADIC_ROOT
    assert pow(ARK_BN254_FR_TWO_ADIC_ROOT, 1 << 28, R_MOD) == 1
    assert pow(ARK_BN254_FR_TWO_ADIC_ROOT, 1 << 27, R_MOD) == R_MOD - 1
    # G1 generator and its negation: x || y little-endian, flag bit 7 iff y > -y
    g = oracle.g1_mul_gen(1)
    assert g == G1_GEN[0].to_bytes(32, "little") + G1_GEN[1].to_bytes(32, "little")
    ng = oracle.g1_mul_gen(R_MOD - 1)
    assert ng[:63] == (G1_GEN[0].to_bytes(32, "little") + (Q_MOD - 2).to_bytes(32, "little"))[:63]
    assert ng[63] == ((Q_MOD - 2) >> 248) | SW_FLAG_Y_NEGATIVE
    assert oracle.g1_mul_gen(0) == bytes(63) + bytes([SW_FLAG_INFINITY])
    # the G2 generator as the mont params file carries it (ark uncompressed:
    # x.c0, x.c1, y.c0, y.c1 little-endian, flags in the last byte), and it
    # lies on the twist y^2 = x^3 + 3 / (9 + u)
    g2 = oracle.params(2, 3, 1).mont(0)[6:6 + 128]
    coords = [int.from_bytes(g2[32 * i:32 * i + 32], "little") for i in range(4)]
    coords[3] &= (1 << 254) - 1
    assert (coords[0], coords[1]) == G2_GEN_X and (coords[2], coords[3]) == G2_GEN_Y

    def f2mul(a, b):
        return ((a[0] * b[0] - a[1] * b[1]) % Q_MOD, (a[0] * b[1] + a[1] * b[0]) % Q_MOD)

    xi = (9, 1)
    xi_inv_n = pow(9 * 9 + 1, -1, Q_MOD)
    b2 = f2mul((3, 0), (9 * xi_inv_n % Q_MOD, (-xi_inv_n) % Q_MOD))
    x3 = f2mul(f2mul(G2_GEN_X, G2_GEN_X), G2_GEN_X)
    assert f2mul(G2_GEN_Y, G2_GEN_Y) == ((x3[0] + b2[0]) % Q_MOD, (x3[1] + b2[1]) % Q_MOD)
    assert f2mul(xi, (9 * xi_inv_n % Q_MOD, (-xi_inv_n) % Q_MOD)) == (1, 0)


@pytest.mark.parametrize("fixture", ["encode_3x5.json", "encode_6x5.json"])
def test_golden_encode(oracle, fixture):
    """Byte parity with the pure-Python restatement (tests/golden/make_golden.py)
    at 8 x 32 and at the reference's own 64 x 32 test setting."""
    e = json.load(open(os.path.join(HERE, "golden", fixture)))["encode"]
    op = oracle.params(e["log_row"], e["log_col"], e["seed"])
    ob = oracle.encode(op, bytes.fromhex(e["payload_hex"]))
    assert hex(oracle.tau(e["seed"])) == e["tau"]
    assert ob.commitment().hex() == e["erasure_commitment"]
    assert [ob.roots()[32 * i:32 * i + 32].hex() for i in range(3)] == e["roots"]
    assert ob.file_root().hex() == e["file_root"]
    assert hashlib.sha256(ob.data()).hexdigest() == e["encoded_data_sha256"]
    for i, h in enumerate(e["slice_sha256"]):
        s = ob.slice(i)
        assert len(s) == e["slice_size"]
        assert hashlib.sha256(s).hexdigest() == h, i


def test_fr_mul_matches_python(oracle):
    import ctypes
    rng = random.Random(2)
    out = ctypes.create_string_buffer(32)
    for _ in range(200):
        a, b = rng.randrange(R_MOD), rng.randrange(R_MOD)
        oracle.L.zgo_fr_mul(a.to_bytes(32, "little"), b.to_bytes(32, "little"), out)
        assert int.from_bytes(out.raw, "little") == a * b % R_MOD


@pytest.mark.parametrize("log_n", [1, 2, 4, 6])
def test_ntt_matches_naive_dft(oracle, log_n):
    rng = random.Random(log_n)
    n = 1 << log_n
    v = [rng.randrange(R_MOD) for _ in range(n)]
    w = pow(5, (R_MOD - 1) >> log_n, R_MOD)
    assert fr_vals(oracle.ntt(fr_bytes(v))) == mg.dft(v, w)
    assert fr_vals(oracle.ntt(oracle.ntt(fr_bytes(v)), inverse=True)) == v
    # coset: coefficient i scaled by coset_factor(n, 1)^i before the transform
    g = oracle.coset_factor(n, 1)
    assert fr_vals(oracle.ntt(fr_bytes(v), coset_idx=1, coset_len=n)) == \
        mg.dft([x * pow(g, i, R_MOD) % R_MOD for i, x in enumerate(v)], w)


def test_coset_factor(oracle):
    """test_coset_factor (crates/amt/src/blob/encode.rs:349-355) and the
    production cosets g1 = w_{2^21}, g2 = w_{2^22}."""
    assert oracle.coset_factor(16, 1) == oracle.root_of_unity(5)
    assert oracle.coset_factor(1 << 20, 1) == oracle.root_of_unity(21)
    assert oracle.coset_factor(1 << 20, 2) == oracle.root_of_unity(22)
    assert oracle.coset_factor(1 << 20, 3) == pow(oracle.root_of_unity(22), 3, R_MOD)


def test_pairing_bilinear(oracle):
    for seed in (3, 11):
        assert oracle.L.zgo_pairing_selftest(seed) == 1


def test_params_ec_domain_equals_scalar_domain(oracle):
    """AMTParams::from_pp restated with G1/G2 FFTs (generate.rs:139-263)
    equals the scalar-domain builder, mont file bytes included."""
    ec = oracle.params(3, 5, 42, ec_domain=True)
    sd = oracle.params(3, 5, 42)
    for c in range(3):
        assert ec.mont(c) == sd.mont(c)


def test_erasure_encoding(oracle):
    """test_erasure_encoding (crates/amt/src/blob/encode.rs:316-347): coset 0
    and coset 1 are the even / odd samples of the 2N-point transform of the
    data polynomial."""
    lr, lc = 3, 5
    n = 1 << (lr + lc)
    op = oracle.params(lr, lc, 5)
    payload = bytes(random.Random(5).randrange(256) for _ in range(7000))
    data = oracle.encode(op, payload).data()
    rows = lambda c: fr_vals(data[c * n * 32:(c + 1) * n * 32])
    col_major = lambda v: [v[r * (1 << lc) + j] for j in range(1 << lc) for r in range(1 << lr)]
    pts = col_major(rows(0))
    coeff = fr_vals(oracle.ntt(fr_bytes(pts), inverse=True))
    big = fr_vals(oracle.ntt(fr_bytes(coeff + [0] * n)))
    assert col_major(rows(0)) == big[0::2]
    assert col_major(rows(1)) == big[1::2]


# ---- verify and the reference's fault-injection table ------------------------
from slice_faults import fault_cases  # noqa: E402


@pytest.fixture(scope="module")
def blob_4x6(oracle):
    op = oracle.params(4, 6, 99)
    payload = bytes(random.Random(222).randrange(256) for _ in range(1234))
    ob = oracle.encode(op, payload)
    return op, ob, [ob.slice(i) for i in range(48)]


def test_every_slice_verifies(oracle, blob_4x6):
    """test_batcher_and_verify (crates/encoder/src/encoder/blob.rs:282-293)."""
    op, ob, slices = blob_4x6
    for i, s in enumerate(slices):
        rc, det = oracle.verify(op, s, ob.commitment(), ob.file_root())
        assert rc == zgo.V_OK, (i, rc, det)


@pytest.mark.parametrize("index", [0, 1, 15, 16, 37, 47])
def test_fault_injection_error_codes(oracle, blob_4x6, index):
    """gen_err_signer_map / get_invalid_row (crates/encoder/src/encoder/blob.rs:84-229,
    amt/blob.rs:61-96, merkle/blob.rs:60-106): each corruption yields exactly
    the reference's VerifierError variant."""
    op, ob, slices = blob_4x6
    com, root = ob.commitment(), ob.file_root()
    for buf, code, sub, a, b, c in fault_cases(slices, index, 4, 6):
        rc, det = oracle.verify(op, bytes(buf), com, root)
        assert rc == code, (index, rc, det)
        if code == zgo.V_AMT_INCORRECT_PROOF:
            assert det[0] == sub
        assert det[1:] == [a, b, c], (index, rc, det)


def test_too_large_blob(oracle):
    op = oracle.params(3, 5, 1)
    max_raw = 31 * 256 - 4
    oracle.encode(op, bytes(max_raw))
    with pytest.raises(zgo.TooLargeBlob):
        oracle.encode(op, bytes(max_raw + 1))


def test_zero_payload_is_infinity(oracle):
    op = oracle.params(3, 5, 1)
    ob = oracle.encode(op, b"")
    assert ob.commitment() == bytes(64)
    assert ob.slice(0)[16:80] == bytes(63) + b"\x40"
    rc, det = oracle.verify(op, ob.slice(5), ob.commitment(), ob.file_root())
    assert rc == zgo.V_OK


# ---- recovery (crates/recovery/src/data_poly.rs:164-256) -----------------------
@pytest.fixture(scope="module")
def recovery_blob(oracle):
    lr, lc = 4, 5
    op = oracle.params(lr, lc, 3)
    payload = bytes(random.Random(9).randrange(256) for _ in range(31 * (1 << (lr + lc)) - 4))
    data = oracle.encode(op, payload).data()
    C = 1 << lc
    rows = {i: data[i * C * 32:(i + 1) * C * 32] for i in range(3 << lr)}
    return lr, lc, payload, rows


def test_recovery_patterns(oracle, recovery_blob):
    lr, lc, payload, rows = recovery_blob
    R = 1 << lr
    pats = [
        range(1, 3 * R),
        list(range(0, R)) + list(range(R + 1, 3 * R)),
        range(R + 1, 3 * R),
        range(3 * R - R, 3 * R),
        range(0, R),
        range(1, 3 * R, 2),
    ]
    rng = random.Random(4)
    for k in (R, R + 1, 2 * R, 3 * R - 1, 3 * R):
        pats.append(rng.sample(range(3 * R), k))
    for p in pats:
        rc, out = oracle.recover(lr, lc, {i: rows[i] for i in p})
        assert rc == 0, (list(p)[:5], out)
        assert out == payload


def test_recovery_errors(oracle, recovery_blob):
    lr, lc, payload, rows = recovery_blob
    R = 1 << lr
    few = {i: rows[i] for i in range(2 * R + 2, 3 * R)}               # R - 2 rows
    assert oracle.recover(lr, lc, few) == (1, "Not enough valid lines")
    over = {i: rows[i] for i in range(2 * R + 1, 3 * R)}
    over[3 * R] = rows[0]                                                # row id >= BLOB_ROW_ENCODED
    assert oracle.recover(lr, lc, over) == (2, "Cannot recover data: RowIdOverflow")
    short = {i: rows[i] for i in range(R)}
    short[R] = rows[R][:-1]                                              # malformed rows are dropped
    rc, out = oracle.recover(lr, lc, short)
    assert rc == 0 and out == payload


def test_recovery_error_branches(oracle):
    """Codewords of invalid RawData and invalid inputs (tests/recovery_cases.py)."""
    from recovery_cases import bad_codewords
    lr, lc = 4, 5
    op = oracle.params(lr, lc, 3)
    cases = bad_codewords(lambda p: oracle.encode(op, p).data(), lr, lc)
    for name, rows, expected in cases:
        rc, out = oracle.recover(lr, lc, rows)
        if isinstance(expected, bytes):
            assert (rc, out) == (0, expected), name
        else:
            assert rc and out == expected, (name, rc, out)
