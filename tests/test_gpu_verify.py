"""GPU batched verification (zg_verify_slices) against the oracle's
EncodedSlice::verify, slice by slice: same verdict, same detail fields."""
import time

import numpy as np
import pytest

import zgo
from slice_faults import fault_cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def blob_4x6(gpu_pkg, oracle):
    params = gpu_pkg.ZgEncoderParams.from_seed(4, 6, 99)
    op = oracle.params(4, 6, 99)
    payload = np.random.default_rng(222).integers(0, 256, size=1234, dtype=np.uint8).tobytes()
    reply = gpu_pkg.EncoderService(params).process_data(payload, True)
    yield params, op, reply
    params.close()


def _oracle_verdicts(oracle, op, slices, com, root):
    out = []
    for s in slices:
        rc, det = oracle.verify(op, bytes(s), com, root)
        out.append((rc, det))
    return out


def _check_same(gpu_pkg, oracle, params, op, slices, com, root, seed=7):
    codes, det = gpu_pkg.verify_slices(params, slices, com, root, seed=seed)
    exp = _oracle_verdicts(oracle, op, slices, com, root)
    for i, (rc, d) in enumerate(exp):
        assert codes[i] == rc, (i, codes[i], det[i], rc, d)
        if rc == zgo.V_AMT_INCORRECT_PROOF:
            assert det[i][0] == d[0], (i, det[i], d)
        assert det[i][1:] == d[1:], (i, det[i], d)
    return codes


def test_every_slice_verifies(gpu_pkg, oracle, blob_4x6):
    """test_batcher_and_verify (crates/encoder/src/encoder/blob.rs:282-293):
    every slice of an encode verifies, in one batch."""
    params, op, reply = blob_4x6
    codes = _check_same(gpu_pkg, oracle, params, op, reply.encoded_slice, reply.erasure_commitment,
                        reply.storage_root)
    assert codes == [0] * len(reply.encoded_slice)


def test_full_payload_slices_verify(gpu_pkg, oracle):
    """A full payload (every row of every coset non-zero): all slices verify."""
    params = gpu_pkg.ZgEncoderParams.from_seed(5, 6, 41)
    op = oracle.params(5, 6, 41)
    payload = np.random.default_rng(9).integers(0, 256, size=params.dims.max_raw_data_size,
                                                dtype=np.uint8).tobytes()
    reply = gpu_pkg.EncoderService(params).process_data(payload, True)
    codes = _check_same(gpu_pkg, oracle, params, op, reply.encoded_slice, reply.erasure_commitment,
                        reply.storage_root)
    assert codes == [0] * len(reply.encoded_slice)
    params.close()


def test_fault_injection_in_one_batch(gpu_pkg, oracle, blob_4x6):
    """The reference's fault-injection table (gen_err_signer_map), every
    corrupted slice of several rows mixed with the valid slices in ONE call:
    the random linear combinations fail and bisection finds each bad slice
    with the oracle's verdict and details."""
    params, op, reply = blob_4x6
    slices = list(reply.encoded_slice)
    batch = list(slices)
    for index in (0, 1, 15, 16, 37, 47):
        batch += [c[0] for c in fault_cases(slices, index, 4, 6)]
    codes = _check_same(gpu_pkg, oracle, params, op, batch, reply.erasure_commitment, reply.storage_root)
    assert codes[:len(slices)] == [0] * len(slices)
    assert all(c != 0 for c in codes[len(slices):])


def test_kzg_layer_error(gpu_pkg, oracle, blob_4x6):
    """A wrong proof quotient at layer d fails KzgError(d) (checked from the
    deepest layer down, verify_params.rs:162-177)."""
    params, op, reply = blob_4x6
    s = reply.encoded_slice[21]
    lay_proof = 96 + 32 * 64 + 8
    bad = []
    for d in (0, 2, 3):
        q = lay_proof + 128 * d + 64  # quotient_d
        other = reply.encoded_slice[22][q:q + 64]
        bad.append(s[:q] + other + s[q + 64:])
    _check_same(gpu_pkg, oracle, params, op, bad + [s], reply.erasure_commitment, reply.storage_root)


def test_malformed_and_mismatched(gpu_pkg, oracle, blob_4x6):
    params, op, reply = blob_4x6
    s = reply.encoded_slice[3]
    cases = [s[:-1], s + b"\0", b"", bytes(len(s)), s[:96] + b"\xff" * 32 + s[128:]]
    codes, _ = gpu_pkg.verify_slices(params, cases + [s], reply.erasure_commitment, reply.storage_root)
    assert codes[:len(cases)] == [zgo.V_DESERIALIZE] * len(cases)
    assert codes[-1] == 0
    # another blob's commitment / root
    other = gpu_pkg.EncoderService(params).process_data(b"other payload", True)
    _check_same(gpu_pkg, oracle, params, op, [s, reply.encoded_slice[40]], other.erasure_commitment,
                reply.storage_root)
    _check_same(gpu_pkg, oracle, params, op, [s], reply.erasure_commitment, other.storage_root)


def test_zero_payload_commitment_at_infinity(gpu_pkg, oracle):
    params = gpu_pkg.ZgEncoderParams.from_seed(3, 5, 1)
    op = oracle.params(3, 5, 1)
    reply = gpu_pkg.EncoderService(params).process_data(b"", True)
    assert reply.erasure_commitment == bytes(64)  # the affine point at infinity, (0, 0)
    codes = _check_same(gpu_pkg, oracle, params, op, reply.encoded_slice, reply.erasure_commitment,
                        reply.storage_root)
    assert codes == [0] * len(reply.encoded_slice)
    params.close()


@pytest.fixture(scope="module")
def prod(gpu_pkg):
    seed = 2024
    params = gpu_pkg.ZgEncoderParams.from_seed(10, 10, seed)
    payload = np.random.default_rng(222).integers(0, 256, size=params.dims.max_raw_data_size,
                                                  dtype=np.uint8).tobytes()
    reply = gpu_pkg.EncoderService(params).process_data(payload, True)
    yield params, seed, payload, reply
    params.close()


def test_production_blob_verifies(prod, gpu_pkg, oracle):
    """All 3072 slices of the 1024 x 1024 blob verify in one call; a slice
    with a wrong row element among them is found (InconsistentCommitment)."""
    params, seed, payload, reply = prod
    slices = list(reply.encoded_slice)
    t0 = time.perf_counter()
    codes, _ = gpu_pkg.verify_slices(params, slices, reply.erasure_commitment, reply.storage_root, seed=3)
    dt = time.perf_counter() - t0
    assert codes == [0] * 3072
    print(f"verified 3072 slices in {dt:.3f} s")
    s = slices[1500]
    bad = s[:96 + 32 * 5] + bytes(32) + s[96 + 32 * 6:]
    codes, det = gpu_pkg.verify_slices(params, slices[:1500] + [bad] + slices[1501:], reply.erasure_commitment,
                                       reply.storage_root, seed=4)
    basis = b"".join(params.param_line(c, 10) for c in range(3))
    vp = oracle.verify_params(10, 10, seed, basis)
    rc, d = oracle.verify(vp, bad, reply.erasure_commitment, reply.storage_root)
    assert rc == zgo.V_AMT_INCORRECT_PROOF and d[0] == zgo.P_INCONSISTENT
    assert codes[1500] == rc and det[1500] == d
    assert codes[:1500] == [0] * 1500 and codes[1501:] == [0] * 1571


def test_mont_param_files(gpu_pkg, oracle, tmp_path):
    """ZgEncoderParams::from_dir_mont (crates/amt/src/blob/encode.rs:114-132):
    params read from the reference's mont files (G1 lines and the G2
    vanishing points / high_g2 the verifier needs) encode and verify exactly
    as the seeded context does."""
    lr, lc, seed = 4, 6, 57
    op = oracle.params(lr, lc, seed)
    for c in range(3):
        # the reference's file names: amt-prove-coset{c}-mont-<hash>-{LR:02}-{LR+LC:02}.bin
        (tmp_path / f"amt-prove-coset{c}-mont-5DWgDV-{lr:02d}-{lr + lc:02d}.bin").write_bytes(op.mont(c))
    params = gpu_pkg.ZgEncoderParams.from_dir_mont(str(tmp_path), lr, lc)
    seeded = gpu_pkg.ZgEncoderParams.from_seed(lr, lc, seed)
    for c in range(3):
        for line in range(lr + 2):
            assert params.param_line(c, line) == seeded.param_line(c, line)
    payload = np.random.default_rng(4).integers(0, 256, size=params.dims.max_raw_data_size,
                                                dtype=np.uint8).tobytes()
    reply = gpu_pkg.EncoderService(params).process_data(payload, True)
    ob = oracle.encode(op, payload)
    assert reply.erasure_commitment == ob.commitment() and reply.storage_root == ob.file_root()
    codes = _check_same(gpu_pkg, oracle, params, op, reply.encoded_slice, reply.erasure_commitment,
                        reply.storage_root)
    assert codes == [0] * len(reply.encoded_slice)
    params.close()
    seeded.close()
