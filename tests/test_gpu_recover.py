"""GPU erasure recovery (zg_recover) against the oracle's
recover_from_da_slice (crates/recovery/src/lib.rs:15-43): the same payload
bytes, or the same error message, for every received-row pattern."""
import numpy as np
import pytest

from recovery_cases import bad_codewords, patterns, split_rows

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(4, 5), (5, 4)])
def small(request, gpu_pkg):
    lr, lc = request.param
    params = gpu_pkg.ZgEncoderParams.from_seed(lr, lc, 11)
    svc = gpu_pkg.EncoderService(params)
    yield gpu_pkg, params, svc, lr, lc
    params.close()


def _gpu_recover(pkg, params, rows):
    try:
        return 0, pkg.recover_from_da_slice(params, rows)
    except pkg.RecoveryError as e:
        return 1, str(e)


def test_recover_patterns_match_oracle(small, oracle):
    pkg, params, svc, lr, lc = small
    payload = np.random.default_rng(3).integers(0, 256, params.dims.max_raw_data_size - 7,
                                                dtype=np.uint8).tobytes()
    rows = split_rows(svc.process_data(payload, True).encoded_data, lr, lc)
    for p in patterns(lr):
        sub = {i: rows[i] for i in p}
        out = pkg.recover_from_da_slice(params, sub)
        assert out == payload, p[:8]
        assert oracle.recover(lr, lc, sub) == (0, payload)


def test_recover_error_branches_match_oracle(small, oracle):
    pkg, params, svc, lr, lc = small
    cases = bad_codewords(lambda p: svc.process_data(p, True).encoded_data, lr, lc)
    for name, rows, expected in cases:
        got = _gpu_recover(pkg, params, rows)
        rc, want = oracle.recover(lr, lc, rows)
        if isinstance(expected, bytes):
            assert got == (0, expected) and (rc, want) == (0, expected), name
        else:
            assert got == (1, expected), (name, got)
            assert rc and want == expected, (name, rc, want)


def test_recover_empty_payload_and_repeat(small):
    """Zero-length payload; two calls in a row on one context give one answer."""
    pkg, params, svc, lr, lc = small
    rows = split_rows(svc.process_data(b"", True).encoded_data, lr, lc)
    R = 1 << lr
    sub = {i: rows[i] for i in range(R, 2 * R)}
    assert pkg.recover_from_da_slice(params, sub) == b""
    assert pkg.recover_from_da_slice(params, sub) == b""
