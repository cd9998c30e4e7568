"""The allocation-free MSM entry point against the allocating one.

zg_msm_chunks_noalloc exists for callers that cannot allocate device memory
on each call (a process whose HBM is already handed to another allocator, or
a loop that must not block on cudaMalloc). It keeps its scratch in a static
device array shared by all calls, so this test calls it twice in a row, with
different inputs, and checks both results bit for bit against zg_msm_chunks.
The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

import zgo

pytestmark = pytest.mark.gpu


def _dev(buf):
    import torch
    return torch.frombuffer(bytearray(buf), dtype=torch.uint8).cuda()


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy().tobytes()


def test_noalloc_msm_matches_allocating_entry_point(pkg, oracle):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    L = pkg.lib()
    lines, log_nchunks, log_chunk = 3, 4, 6          # 48 chunk MSMs of 64 points
    n = (1 << log_nchunks) << log_chunk
    bases = oracle.random_points(1234, lines * n)   # valid G1 points, mont x||y
    tb = _dev(bases)
    for call, seed in enumerate((11, 12)):
        rng = np.random.default_rng(seed)
        sc = rng.integers(0, 256, size=(n, 32), dtype=np.uint8)
        sc[:, 31] = rng.integers(0, 0x30, size=n, dtype=np.uint8)
        if call == 1:
            sc[:70] = 0                              # zero scalars: infinity results
        ts = _dev(sc.tobytes())
        ref = torch.empty(lines << log_nchunks << 6, dtype=torch.uint8, device="cuda")
        got = torch.empty_like(ref)
        assert L.zg_msm_chunks(tb.data_ptr(), ts.data_ptr(), lines, log_nchunks, log_chunk,
                               ref.data_ptr(), None) == 0, L.zg_last_error()
        assert L.zg_msm_chunks_noalloc(tb.data_ptr(), ts.data_ptr(), lines, log_nchunks, log_chunk,
                                       got.data_ptr(), None) == 0, L.zg_last_error()
        assert _host(got) == _host(ref), f"call {call}"


def test_noalloc_msm_at_the_scratch_limit(pkg, oracle):
    """Exactly 1024 chunk MSMs, the size of the static scratch (its last
    per-MSM result ends at the array's last byte), twice in a row."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    L = pkg.lib()
    lines, log_nchunks, log_chunk = 1, 10, 4         # 1024 chunk MSMs of 16 points
    n = (1 << log_nchunks) << log_chunk
    bases = oracle.random_points(4321, lines * n)
    tb = _dev(bases)
    for call, seed in enumerate((21, 22)):
        rng = np.random.default_rng(seed)
        sc = rng.integers(0, 256, size=(n, 32), dtype=np.uint8)
        sc[:, 31] = rng.integers(0, 0x30, size=n, dtype=np.uint8)
        ts = _dev(sc.tobytes())
        ref = torch.empty((lines << log_nchunks) * 64, dtype=torch.uint8, device="cuda")
        got = torch.empty_like(ref)
        assert L.zg_msm_chunks(tb.data_ptr(), ts.data_ptr(), lines, log_nchunks, log_chunk,
                               ref.data_ptr(), None) == 0, L.zg_last_error()
        assert L.zg_msm_chunks_noalloc(tb.data_ptr(), ts.data_ptr(), lines, log_nchunks, log_chunk,
                                       got.data_ptr(), None) == 0, L.zg_last_error()
        assert _host(got) == _host(ref), f"call {call}"


def test_noalloc_msm_rejects_oversized_requests(pkg):
    L = pkg.lib()
    dummy = ctypes.c_void_p(16)
    for lines, log_nchunks in ((2, 10), (1025, 0)):   # 2048 and 1025 > 1024 MSMs
        rc = L.zg_msm_chunks_noalloc(dummy, dummy, lines, log_nchunks, 6, dummy, None)
        assert rc != 0
        assert b"static scratch limit" in L.zg_last_error()
