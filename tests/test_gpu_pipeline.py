"""The request pipeline (zg_submit / zg_wait / zg_encode_batch): every reply
bit-identical to the plain per-blob path, alone or mixed with recovery
requests, for uneven payload sizes."""
import random

import numpy as np
import pytest

from recovery_cases import split_rows

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def svc(gpu_pkg):
    params = gpu_pkg.ZgEncoderParams.from_seed(4, 6, 5)
    yield gpu_pkg, params, gpu_pkg.EncoderService(params)
    params.close()


def _payloads(max_raw, n, seed):
    rng = np.random.default_rng(seed)
    sizes = [0, 1, max_raw] + [int(x) for x in rng.integers(0, max_raw + 1, n - 3)]
    return [rng.integers(0, 256, s, dtype=np.uint8).tobytes() for s in sizes]


def test_batch_matches_plain(svc):
    pkg, params, s = svc
    payloads = _payloads(params.dims.max_raw_data_size, 9, 1)
    for require_data in (True, False):
        got = s.process_batch(payloads, require_data)
        for p, g in zip(payloads, got):
            assert g == s.process_data(p, require_data)


def test_batch_too_large_returns_nothing(svc):
    pkg, params, s = svc
    big = bytes(params.dims.max_raw_data_size + 1)
    with pytest.raises(pkg.TooLargeBlob):
        s.process_batch([b"abc", big], True)
    with pytest.raises(pkg.TooLargeBlob):
        s.submit(big, True)


def test_mixed_requests_match_alone(svc):
    """Encodes and recoveries interleaved in one queue: each result equals the
    same request run alone."""
    pkg, params, s = svc
    lr, lc = 4, 6
    R = 1 << lr
    payloads = _payloads(params.dims.max_raw_data_size, 6, 2)
    alone = [s.process_data(p, True) for p in payloads]
    rnd = random.Random(3)
    recs = []
    for p, a in zip(payloads[:3], alone[:3]):
        rows = split_rows(a.encoded_data, lr, lc)
        recs.append((p, {i: rows[i] for i in rnd.sample(range(3 * R), 3 * R // 2)}))
    bad = {i: rows[i] for i in range(R - 1)}
    tickets = []
    for i, p in enumerate(payloads):
        tickets.append(("enc", i, s.submit(p, True)))
        if i < 3:
            tickets.append(("rec", i, s.submit_recover(recs[i][1])))
    tickets.append(("bad", 0, s.submit_recover(bad)))
    rnd.shuffle(tickets)  # results are claimed in any order
    for kind, i, t in tickets:
        if kind == "enc":
            assert s.wait(t) == alone[i]
        elif kind == "rec":
            assert s.wait(t) == recs[i][0] == pkg.recover_from_da_slice(params, recs[i][1])
        else:
            with pytest.raises(pkg.RecoveryError, match="Not enough valid lines"):
                s.wait(t)


@pytest.mark.parametrize("blobs_per_launch", [2, 1])
def test_fused_launches_match_plain(svc, blobs_per_launch):
    """Requests waiting together are fused into one unit launch (one bucket
    accumulation over both blobs' MSM items) when blobs_per_launch is 2, and
    run one per launch when it is 1; every reply equals the plain path's."""
    pkg, params, s = svc
    params.set_pipeline(max_units=2, blobs_per_launch=blobs_per_launch)
    before = params.pipeline_stats()
    payloads = _payloads(params.dims.max_raw_data_size, 9, 5)
    alone = [s.process_data(p, True) for p in payloads]
    assert s.process_batch(payloads, True) == alone  # nine requests queued at once
    tickets = [s.submit(p, True) for p in payloads]
    for t, a in zip(tickets, alone):
        assert s.wait(t) == a
    st = params.pipeline_stats()
    fused = st["launches_by_blobs"][2] - before["launches_by_blobs"][2]
    if blobs_per_launch == 1:
        assert fused == 0
    else:
        assert fused >= 4  # the batch's nine requests fill at least four pairs
    assert st["max_in_flight"] >= 2
    params.set_pipeline()


def test_fused_launches_wide_windows(gpu_pkg):
    """Fused pairs at 32 x 1024, where each blob's MSM is six item sets (the
    chunk lines and five wide-window unit sizes), twelve in the shared launch."""
    params = gpu_pkg.ZgEncoderParams.from_seed(5, 10, 9)
    try:
        s = gpu_pkg.EncoderService(params)
        params.set_pipeline(max_units=1, blobs_per_launch=2)
        payloads = _payloads(params.dims.max_raw_data_size, 4, 6)
        alone = [s.process_data(p, False) for p in payloads]
        assert s.process_batch(payloads, False) == alone
        assert params.pipeline_stats()["launches_by_blobs"][2] >= 2
    finally:
        params.close()
