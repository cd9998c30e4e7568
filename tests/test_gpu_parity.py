"""GPU parity: the CUDA path, called through the C ABI, against the CPU oracle.

Integer / field / byte work: every comparison is bit-exact.
"""
import ctypes
import random

import numpy as np
import pytest

import zgo

pytestmark = pytest.mark.gpu

R_MOD = zgo.R_MOD
Q_MOD = zgo.Q_MOD


def torch_mod():
    import torch
    return torch


def rand_fr_bytes(rng, n):
    """n canonical Fr elements, 32 B little-endian each (top byte < 0x30)."""
    b = rng.integers(0, 256, size=(n, 32), dtype=np.uint8)
    b[:, 31] = rng.integers(0, 0x30, size=n, dtype=np.uint8)
    return b.tobytes()


def dev(buf: bytes):
    torch = torch_mod()
    t = torch.frombuffer(bytearray(buf), dtype=torch.uint8).cuda()
    return t


def host(t) -> bytes:
    torch = torch_mod()
    torch.cuda.synchronize()
    return t.cpu().numpy().tobytes()


def empty(n):
    torch = torch_mod()
    return torch.empty(n, dtype=torch.uint8, device="cuda")


def device_view(ptr, n):
    """A uint8 tensor over n bytes of library-owned device memory."""
    torch = torch_mod()

    class _Cai:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_Cai(), device="cuda")


def mont_lines(mont: bytes, log_row, log_col):
    """Split a mont params file into its G1 lines (fast_serde_bn254.rs:20-53)."""
    n = 1 << (log_row + log_col)
    off = 6 + 256
    basis = mont[off:off + 64 * n]
    off += 64 * n
    quot = []
    for _ in range(log_row):
        quot.append(mont[off:off + 64 * n])
        off += 64 * n
    for d in range(log_row):
        off += 128 * (2 << d)
    high = mont[off:off + 64 * n]
    return quot + [basis, high]


# ---------------------------------------------------------------------------
def test_device_arithmetic_selftest(gpu_pkg):
    """Device field / curve routines against their host build, incl. the
    FP64-pipe Fq product the MSM pairs with the integer one and its Fr form."""
    fails = gpu_pkg.selftest()
    assert fails == {k: 0 for k in fails}, fails
    assert "fq_mul_f64" in fails and "fq_mul_w28" in fails and "fr_mul_f64" in fails


def test_measurement_probes(gpu_pkg):
    """The denominators of the bench's MSM fractions: the IMAD rate and the
    Fq product rate of every product kind are positive and physical (below
    one product per SM clock per lane)."""
    imad = gpu_pkg.probe_imad(0)
    assert 1e3 < imad < 1e5  # G IMAD/s
    for kind in gpu_pkg.MSM_PRODUCTS:
        g = gpu_pkg.probe_products(0, kind)
        assert 1.0 < g < imad / 100, kind  # a product is > 100 IMADs
    out = ctypes.c_double()
    assert gpu_pkg.lib().zg_probe_products(0, len(gpu_pkg.MSM_PRODUCTS), ctypes.byref(out)) != 0  # no such kind


@pytest.mark.parametrize("log_n,batch,inverse,coset", [
    (5, 4, 0, 0), (5, 4, 1, 0), (5, 3, 0, 1), (10, 8, 0, 0), (10, 8, 1, 0), (10, 2, 0, 2),
    (11, 2, 1, 0), (14, 1, 0, 0), (14, 1, 1, 0), (20, 1, 0, 1), (20, 1, 1, 0),
    (12, 4, 0, 1), (13, 3, 1, 0), (14, 5, 0, 2),  # batched four-step passes
    # the transform core's edge shapes: one stage, the fused first pass alone,
    # an odd last radix-2 stage, and odd four-step splits
    (1, 3, 0, 0), (1, 2, 1, 0), (1, 2, 0, 1), (2, 3, 0, 1), (2, 2, 1, 0), (3, 2, 0, 0), (3, 2, 1, 0),
    (4, 2, 0, 1), (7, 3, 0, 1), (9, 2, 1, 0), (15, 2, 0, 1), (17, 1, 1, 0),
])
def test_ntt_matches_oracle(gpu_pkg, oracle, log_n, batch, inverse, coset):
    rng = np.random.default_rng(log_n * 100 + batch + inverse)
    n = 1 << log_n
    data = rand_fr_bytes(rng, n * batch)
    t = dev(data)
    rc = gpu_pkg.lib().zg_ntt(t.data_ptr(), log_n, batch, inverse, coset, None)
    assert rc == 0, gpu_pkg.lib().zg_last_error()
    got = host(t)
    for b in range(batch):
        vec = data[b * n * 32:(b + 1) * n * 32]
        exp = oracle.ntt(vec, inverse=bool(inverse), coset_idx=coset, coset_len=n)
        assert got[b * n * 32:(b + 1) * n * 32] == exp, f"vector {b}"


def test_ntt_large_batches_match_oracle(gpu_pkg, oracle):
    """Batches of more vectors than the GPU holds resident CTAs (several waves
    of single-CTA transforms), first, middle and last vectors checked."""
    rng = np.random.default_rng(77)
    for log_n, batch, inverse, coset in ((10, 1500, 0, 0), (8, 3000, 1, 0), (6, 5000, 0, 1)):
        n = 1 << log_n
        data = rand_fr_bytes(rng, n * batch)
        t = dev(data)
        assert gpu_pkg.lib().zg_ntt(t.data_ptr(), log_n, batch, inverse, coset, None) == 0
        got = host(t)
        for b in (0, 1, batch // 2, batch - 1):
            vec = data[b * n * 32:(b + 1) * n * 32]
            exp = oracle.ntt(vec, inverse=bool(inverse), coset_idx=coset, coset_len=n)
            assert got[b * n * 32:(b + 1) * n * 32] == exp, (log_n, b)


def _neg_mont_point(p: bytes) -> bytes:
    y = int.from_bytes(p[32:], "little")
    return p[:32] + ((Q_MOD - y) % Q_MOD).to_bytes(32, "little")


@pytest.fixture(scope="module")
def small_params_mont(oracle):
    op = oracle.params(4, 6, 7)
    return [op.mont(c) for c in range(3)]


def test_msm_chunks_matches_oracle(gpu_pkg, oracle, small_params_mont):
    lines = mont_lines(small_params_mont[0], 4, 6)
    rng = np.random.default_rng(5)
    n = 1 << 10
    bases = b"".join(lines[:3])  # 3 lines of 1024 points
    scal = bytearray(rand_fr_bytes(rng, n))
    # edge scalars: zero, one, r - 1, small
    for i, v in enumerate([0, 1, R_MOD - 1, 2, 255, 256, 1 << 253]):
        scal[32 * i:32 * i + 32] = v.to_bytes(32, "little")
    scal = bytes(scal)
    out = empty(3 * 16 * 64)
    tb, ts = dev(bases), dev(scal)  # keep the device buffers alive across the call
    rc = gpu_pkg.lib().zg_msm_chunks(tb.data_ptr(), ts.data_ptr(), 3, 4, 6, out.data_ptr(), None)
    assert rc == 0, gpu_pkg.lib().zg_last_error()
    got = host(out)
    for l in range(3):
        for b in range(16):
            exp = oracle.msm(lines[l][64 * 64 * b:64 * 64 * (b + 1)], scal[32 * 64 * b:32 * 64 * (b + 1)])
            assert got[(l * 16 + b) * 64:(l * 16 + b + 1) * 64] == exp, (l, b)


@pytest.fixture(scope="module")
def ctx_4x6(gpu_pkg):
    params = gpu_pkg.ZgEncoderParams.from_seed(4, 6, 7)
    yield params
    params.close()


@pytest.mark.parametrize("n,coset,line,kind", [
    (64, 0, 4, "uniform"), (256, 1, 0, "uniform"), (1024, 0, 4, "uniform"), (1024, 2, 5, "blob"),
    (512, 0, 3, "edges"), (1024, 1, 4, "zero"),
])
def test_ctx_msm_matches_oracle(gpu_pkg, oracle, ctx_4x6, n, coset, line, kind):
    """zg_ctx_msm: one MSM over the first n points of a param line (fixed-base
    tables) against the oracle's Pippenger on the same points."""
    rng = np.random.default_rng(n + 7 * coset + line)
    if kind == "zero":
        scal = bytes(32 * n)
    elif kind == "blob":  # 31-byte scalars with a zero suffix (60 % of the points)
        b = np.zeros((n, 32), dtype=np.uint8)
        k = int(n * 0.4)
        b[:k, :31] = rng.integers(0, 256, size=(k, 31), dtype=np.uint8)
        scal = b.tobytes()
    else:
        scal = bytearray(rand_fr_bytes(rng, n))
        if kind == "edges":
            for i, v in enumerate([0, 1, R_MOD - 1, 2, R_MOD - 2, 1 << 252, (1 << 248) - 1]):
                scal[32 * i:32 * i + 32] = v.to_bytes(32, "little")
        scal = bytes(scal)
    bases = ctx_4x6.param_line(coset, line, 0, n)
    out = empty(64)
    ts = dev(scal)
    rc = gpu_pkg.lib().zg_ctx_msm(ctx_4x6.handle, coset, line, ts.data_ptr(), n, out.data_ptr(), None)
    assert rc == 0, gpu_pkg.lib().zg_last_error()
    assert host(out) == oracle.msm(bases, scal)


def test_ctx_msm_rejects_bad_sizes(gpu_pkg, ctx_4x6):
    out = empty(64)
    ts = dev(bytes(32 * 2048))
    L = gpu_pkg.lib()
    for n, coset, line in [(32, 0, 0), (96, 0, 0), (2048, 0, 0), (64, 3, 0), (64, 0, 6)]:
        assert L.zg_ctx_msm(ctx_4x6.handle, coset, line, ts.data_ptr(), n, out.data_ptr(), None) != 0


@pytest.fixture(scope="module")
def ctx_5x10(gpu_pkg):
    params = gpu_pkg.ZgEncoderParams.from_seed(5, 10, 9)
    yield params
    params.close()


@pytest.mark.parametrize("n,coset,line", [(1 << 11, 0, 6), (1 << 13, 1, 0), (1 << 15, 2, 5)])
def test_ctx_msm_small_chunks_match_oracle(gpu_pkg, oracle, ctx_5x10, n, coset, line):
    """On a 1024-column context zg_ctx_msm cuts MSMs that would give few
    1024-point chunks into smaller chunks (here 128 points for 2^11 and 2^13
    points, 512 for 2^15, capped by the context's chunk buffers); the result
    is the oracle's Pippenger on the same points."""
    rng = np.random.default_rng(n + coset)
    scal = bytearray(rand_fr_bytes(rng, n))
    for i, v in enumerate([0, 1, R_MOD - 1, 2, 1 << 252]):
        scal[32 * i:32 * i + 32] = v.to_bytes(32, "little")
    scal = bytes(scal)
    bases = ctx_5x10.param_line(coset, line, 0, n)
    out = empty(64)
    ts = dev(scal)
    rc = gpu_pkg.lib().zg_ctx_msm(ctx_5x10.handle, coset, line, ts.data_ptr(), n, out.data_ptr(), None)
    assert rc == 0, gpu_pkg.lib().zg_last_error()
    assert host(out) == oracle.msm(bases, scal)


def test_msm_special_cases(gpu_pkg, oracle, small_params_mont):
    """Doubling and cancellation inside buckets: repeated and negated bases."""
    line = mont_lines(small_params_mont[0], 4, 6)[0]
    pts = [line[64 * i:64 * i + 64] for i in range(8)]
    chunk = []
    for i in range(32):
        p = pts[i % 4]
        chunk.append(_neg_mont_point(p) if (i // 4) % 2 else p)
    bases = b"".join(chunk)
    scal = b"".join(((i % 3) + 5).to_bytes(32, "little") for i in range(32))
    zero = bytes(32 * 32)
    out = empty(2 * 64)
    b2 = bases + bases
    s2 = scal + zero
    tb, ts = dev(b2), dev(s2)
    rc = gpu_pkg.lib().zg_msm_chunks(tb.data_ptr(), ts.data_ptr(), 1, 1, 5, out.data_ptr(), None)
    assert rc == 0
    got = host(out)
    assert got[:64] == oracle.msm(bases, scal)
    assert got[64:] == oracle.msm(bases, zero)
    assert got[127] == 0x40  # zero scalars give the point at infinity


@pytest.mark.parametrize("log_row,log_col", [(4, 6), (6, 5), (3, 5)])
def test_params_match_oracle(gpu_pkg, oracle, log_row, log_col):
    seed = 1234 + log_row
    params = gpu_pkg.ZgEncoderParams.from_seed(log_row, log_col, seed)
    op = oracle.params(log_row, log_col, seed)
    for c in range(3):
        lines = mont_lines(op.mont(c), log_row, log_col)
        for l, exp in enumerate(lines):
            assert params.param_line(c, l) == exp, (c, l)
    params.close()


def _check_against_oracle(pkg, oracle, params, op, payload, verify_all=False):
    reply = pkg.EncoderService(params).process_data(payload, True)
    ob = oracle.encode(op, payload)
    assert reply.version == 0
    assert reply.erasure_commitment == ob.commitment()
    assert reply.storage_root == ob.file_root()
    assert reply.encoded_data == ob.data()
    d = params.dims
    assert len(reply.encoded_slice) == d.rows_encoded
    for i, s in enumerate(reply.encoded_slice):
        assert len(s) == d.slice_size
        assert s == ob.slice(i), f"slice {i}"
    if verify_all:
        for i, s in enumerate(reply.encoded_slice):
            rc, det = oracle.verify(op, s, reply.erasure_commitment, reply.storage_root)
            assert rc == zgo.V_OK, (i, rc, det)
    return reply


@pytest.mark.parametrize("log_row,log_col", [(4, 6), (6, 5)])
def test_encode_matches_oracle(gpu_pkg, oracle, log_row, log_col):
    """EncodedBlob::build parity for payload sizes 0, 1, 1234, MAX and MAX+1
    (the cases of test_batcher_and_verify, crates/encoder/src/encoder/blob.rs:282-293)."""
    seed = 99
    params = gpu_pkg.ZgEncoderParams.from_seed(log_row, log_col, seed)
    op = oracle.params(log_row, log_col, seed)
    d = params.dims
    rng = np.random.default_rng(222)
    for n in (0, 1, 1234, d.max_raw_data_size):
        payload = rng.integers(0, 256, size=n, dtype=np.uint8).tobytes()
        _check_against_oracle(gpu_pkg, oracle, params, op, payload, verify_all=(n == 1234))
    with pytest.raises(gpu_pkg.TooLargeBlob) as ei:
        gpu_pkg.EncoderService(params).process_data(bytes(d.max_raw_data_size + 1), False)
    assert ei.value.actual == d.max_raw_data_size + 1
    assert ei.value.expected_max == d.max_raw_data_size
    params.close()


@pytest.mark.parametrize("product,cpb,threads,task", [
    ("imad", 1, 128, 64), ("hybrid", 4, 512, 32), ("fp64", 2, 256, 48), ("imad", 2, 512, 96),
    ("fp64", 4, 128, 64), ("w28", 1, 256, 32), ("w28_hybrid", 2, 128, 96), ("w28_hybrid", 4, 256, 64),
])
def test_tuning_choices_match_oracle(gpu_pkg, oracle, product, cpb, threads, task):
    """Every kernel choice the tuning can make (MSM product kind, bucket task
    size, RS column tile and block size) gives the oracle's bytes, on the
    plain path and on the request pipeline (whose CUDA graphs are re-captured
    on a change)."""
    params = gpu_pkg.ZgEncoderParams.from_seed(5, 6, 17)
    op = oracle.params(5, 6, 17)
    payload = np.random.default_rng(cpb * threads).integers(0, 256, size=params.dims.max_raw_data_size - 3,
                                                            dtype=np.uint8).tobytes()
    exp = oracle.encode(op, payload)
    # the pipeline first runs (and captures its graphs) with the default choice
    first = gpu_pkg.EncoderService(params).process_batch([payload], True)[0]
    assert first.storage_root == exp.file_root()
    params.set_tuning(product, cpb, threads, msm_task=task)
    t = params.tuning()
    assert (t["msm_product"], t["ntt_cols_per_cta"], t["ntt_threads"], t["msm_task"]) == \
        (product, cpb, threads, task)
    _check_against_oracle(gpu_pkg, oracle, params, op, payload)
    again = gpu_pkg.EncoderService(params).process_batch([payload], True)[0]
    assert again.encoded_slice == [exp.slice(i) for i in range(params.dims.rows_encoded)]
    assert again.erasure_commitment == exp.commitment()
    with pytest.raises(RuntimeError):
        params.set_tuning(product, 3, threads)
    with pytest.raises(RuntimeError):
        params.set_tuning(product, cpb, threads, msm_task=40)
    params.close()


@pytest.mark.parametrize("log_row", [5, 6])
def test_wide_class_choices_match_oracle(gpu_pkg, oracle, log_row):
    """At 32 x 1024 the context holds five wide-window classes (units of 2^15
    .. 2^11 points); at 64 x 1024 six, the first for the high line's 2^16-point
    nodes as pairs of 2^15-point sort units (the 2^15 class then reads that
    class's sort). Every number of them in use (the lines of the others on
    11-bit chunk windows) gives the oracle's bytes."""
    params = gpu_pkg.ZgEncoderParams.from_seed(log_row, 10, 13)
    op = oracle.params(log_row, 10, 13)
    avail = params.tuning()["msm_wide_avail"]
    assert avail == log_row
    payload = np.random.default_rng(13).integers(0, 256, size=params.dims.max_raw_data_size // 3,
                                                 dtype=np.uint8).tobytes()
    exp = oracle.encode(op, payload)
    lines = []
    for k in range(avail + 1):
        params.set_tuning("hybrid", 2, 256, msm_task=64, msm_wide_classes=k)
        lines.append(params.tuning()["msm_wide_lines"])
        r = gpu_pkg.EncoderService(params).process_data(payload, False)
        assert r.erasure_commitment == exp.commitment(), k
        assert r.encoded_slice == [exp.slice(i) for i in range(params.dims.rows_encoded)], k
    assert lines == sorted(lines) and lines[0] == 0 and lines[-1] == log_row
    params.close()


def test_autotune_then_encode(gpu_pkg, oracle):
    """zg_ctx_autotune times every candidate and keeps the default (hybrid
    kind, task 64) unless another is more than 1 % faster, else the fastest;
    the encodes after it still give the oracle's bytes."""
    params = gpu_pkg.ZgEncoderParams.from_seed(6, 5, 23)
    op = oracle.params(6, 5, 23)
    t = params.autotune()
    assert t["msm_product"] in gpu_pkg.MSM_PRODUCTS
    assert all(x > 0 for x in t["msm_ms"]) and all(x > 0 for x in t["ntt_ms"])
    assert all(x > 0 for x in t["task_ms"])

    def picked(times, chosen, default):
        fastest = min(range(len(times)), key=times.__getitem__)
        if times[fastest] < 0.99 * times[default]:
            return chosen == fastest
        return chosen == default

    assert picked(t["msm_ms"], gpu_pkg.MSM_PRODUCTS.index(t["msm_product"]), gpu_pkg.MSM_PRODUCTS.index("hybrid"))
    assert picked(t["task_ms"], gpu_pkg.MSM_TASK_SIZES.index(t["msm_task"]), gpu_pkg.MSM_TASK_SIZES.index(64))
    assert params.tuning()["msm_product"] == t["msm_product"]
    assert params.tuning()["msm_task"] == t["msm_task"]
    payload = np.random.default_rng(5).integers(0, 256, size=4321, dtype=np.uint8).tobytes()
    _check_against_oracle(gpu_pkg, oracle, params, op, payload)
    params.close()


@pytest.mark.parametrize("bits", [8, 11])
def test_encode_msm_variants_match_oracle(gpu_pkg, oracle, bits):
    """Both MSM variants (8-bit windows with doublings; 11-bit fixed-base
    window tables) give the oracle's bytes."""
    params = gpu_pkg.ZgEncoderParams.from_seed(5, 6, 31, msm_window_bits=bits)
    op = oracle.params(5, 6, 31)
    payload = np.random.default_rng(bits).integers(0, 256, size=params.dims.max_raw_data_size - 7,
                                                   dtype=np.uint8).tobytes()
    _check_against_oracle(gpu_pkg, oracle, params, op, payload)
    params.close()


def test_device_encode_then_host_encode_are_ordered(gpu_pkg, oracle):
    """zg_encode_device on a caller stream followed at once by zg_encode on the
    context stream: both share the context scratch and must not overlap."""
    torch = torch_mod()
    params = gpu_pkg.ZgEncoderParams.from_seed(4, 6, 77)
    op = oracle.params(4, 6, 77)
    L = gpu_pkg.lib()
    rng = np.random.default_rng(9)
    a = rng.integers(0, 256, size=5000, dtype=np.uint8).tobytes()
    b = rng.integers(0, 256, size=3000, dtype=np.uint8).tobytes()
    s = torch.cuda.Stream()
    ta = dev(a)
    db = gpu_pkg._DeviceBlob()
    for _ in range(3):
        rc = L.zg_encode_device(params.handle, ctypes.c_void_p(ta.data_ptr()), len(a),
                                ctypes.c_void_p(s.cuda_stream), ctypes.byref(db))
        assert rc == 0
    reply = gpu_pkg.EncoderService(params).process_data(b, True)
    ob = oracle.encode(op, b)
    assert reply.encoded_data == ob.data()
    assert reply.encoded_slice[5] == ob.slice(5)
    params.close()


@pytest.mark.parametrize("offset", [0, 1, 3, 8, 16])
def test_device_encode_unaligned_payload(gpu_pkg, oracle, offset):
    """zg_encode_device reads the caller's payload in place: at 16-byte
    aligned addresses as 16-byte words, elsewhere byte by byte, with the
    payload end, zero padding and length trailer byte by byte in both cases.
    Every offset gives the oracle's encoded data, slices and roots."""
    params = gpu_pkg.ZgEncoderParams.from_seed(4, 6, 19)
    op = oracle.params(4, 6, 19)
    L = gpu_pkg.lib()
    d = params.dims
    rng = np.random.default_rng(offset)
    for size in (d.max_raw_data_size, 5003, 1984 * 3 + 17):
        payload = rng.integers(0, 256, size=size, dtype=np.uint8).tobytes()
        buf = dev(bytes(offset) + payload + bytes(32))
        db = gpu_pkg._DeviceBlob()
        assert L.zg_encode_device(params.handle, ctypes.c_void_p(buf.data_ptr() + offset), size, None,
                                  ctypes.byref(db)) == 0, L.zg_last_error()
        ob = oracle.encode(op, payload)
        n_enc = 3 * d.raw_blob_size * 32
        assert host(device_view(db.encoded_data, n_enc)) == ob.data(), (offset, size)
        slices = host(device_view(db.slices, 3 * 16 * db.slice_size))
        for i in (0, 17, 47):
            assert slices[i * db.slice_size:(i + 1) * db.slice_size] == ob.slice(i), (offset, size, i)
        assert host(device_view(db.file_root, 32)) == ob.file_root(), (offset, size)
    params.close()


@pytest.mark.parametrize("log_row", [5, 6])
def test_encode_wide_windows_match_oracle(gpu_pkg, oracle, log_row):
    """With 1024 columns every AMT line whose nodes hold more than 1024 points
    runs on wide fixed-base windows: units of 2^min(15, log2 node) points and
    (log2 unit + 1)-bit digits. At 32 and 64 rows all five unit sizes
    (2^11 .. 2^15) occur; only the last quotient line and the basis line stay
    on 1024-point chunks. Both a random payload and a constant one (every data
    scalar equal: whole units in one bucket per window, the adaptive task size
    of the bucket kernel) give the oracle's bytes, and the 11-bit-only context
    gives the same reply."""
    seed = 41
    params = gpu_pkg.ZgEncoderParams.from_seed(log_row, 10, seed)
    narrow = gpu_pkg.ZgEncoderParams.from_seed(log_row, 10, seed, msm_window_bits=11)
    assert params.tuning()["msm_wide_lines"] == log_row  # L - 2 of the L = log_row + 2 lines
    assert narrow.tuning()["msm_wide_lines"] == 0
    op = oracle.params(log_row, 10, seed)
    d = params.dims
    rng = np.random.default_rng(log_row)
    for payload in (rng.integers(0, 256, size=d.max_raw_data_size, dtype=np.uint8).tobytes(),
                    b"\xff" * d.max_raw_data_size):
        reply = _check_against_oracle(gpu_pkg, oracle, params, op, payload)
        other = gpu_pkg.EncoderService(narrow).process_data(payload, False)
        assert other.erasure_commitment == reply.erasure_commitment
        assert list(other.encoded_slice) == list(reply.encoded_slice)
    narrow.close()
    params.close()


def test_encode_zero_blob_is_infinity(gpu_pkg, oracle):
    """An empty payload encodes to the all-zero blob: every commitment and
    proof is the point at infinity (ark flag bit 6)."""
    params = gpu_pkg.ZgEncoderParams.from_seed(4, 6, 5)
    reply = gpu_pkg.EncoderService(params).process_data(b"", False)
    assert reply.erasure_commitment == bytes(64)
    assert reply.encoded_data == b""
    s = reply.encoded_slice[0]
    assert s[16:80] == bytes(63) + b"\x40"
    params.close()


def test_merkle_roots_match_oracle(gpu_pkg, oracle):
    rng = np.random.default_rng(3)
    log_row, log_col = 5, 6
    n = 3 << (log_row + log_col)
    items = rng.integers(0, 256, size=32 * n, dtype=np.uint8).tobytes()
    out = empty(96)
    ti = dev(items)
    rc = gpu_pkg.lib().zg_merkle_roots(ti.data_ptr(), n, out.data_ptr(), None)
    assert rc == 0
    assert host(out) == oracle.merkle_roots(log_row, log_col, items)


# ---------------------------------------------------------------------------
# production shape: 1024 x 1024, full payload
@pytest.fixture(scope="module")
def prod(gpu_pkg):
    seed = 2024
    params = gpu_pkg.ZgEncoderParams.from_seed(10, 10, seed)
    rng = np.random.default_rng(222)
    payload = rng.integers(0, 256, size=params.dims.max_raw_data_size, dtype=np.uint8).tobytes()
    reply = gpu_pkg.EncoderService(params).process_data(payload, True)
    yield params, seed, payload, reply
    params.close()


@pytest.fixture(scope="module")
def prod_oracle(prod, oracle):
    """The oracle's own params of the same seeded tau (built on the CPU) and
    its full encode of the production payload (the reference CPU
    decomposition of prove.rs, every MSM ark-ec's signed-digit method)."""
    _, seed, payload, _ = prod
    op = oracle.params(10, 10, seed)
    ob = oracle.encode(op, payload)
    return op, ob


def test_production_params_full(prod, prod_oracle):
    """Every point of every G1 param line of the three cosets (12 lines of
    2^20 points each) equals the oracle's, byte for byte."""
    params = prod[0]
    op = prod_oracle[0]
    for c in range(3):
        for line, exp in enumerate(mont_lines(op.mont(c), 10, 10)):
            assert params.param_line(c, line) == exp, (c, line)


def test_production_params_sample(prod, oracle):
    """Sampled param points against the scalar-domain oracle (s * G1 of the
    param scalars of the seeded tau), independent of the oracle's EC builder."""
    params, seed, _, _ = prod
    idx = [0, 1, 2, 777, 65535, 524288, 1048575]
    for c in range(3):
        for line in (0, 9, 10, 11):
            got = params.param_line(c, line)
            exp = oracle.param_points(10, 10, seed, c, line, idx)
            for k, i in enumerate(idx):
                assert got[64 * i:64 * i + 64] == exp[64 * k:64 * k + 64], (c, line, i)


def test_production_full_blob_matches_oracle(prod, prod_oracle):
    """The whole 1024 x 1024 reply equals the oracle's full encode of the same
    payload: erasure commitment, storage root, the 96 MiB of encoded data and
    all 3072 serialized slices (every AMT sibling pair, high commitment, row,
    Merkle root, path and leaf of every row)."""
    _, _, _, reply = prod
    ob = prod_oracle[1]
    assert reply.erasure_commitment == ob.commitment()
    assert reply.storage_root == ob.file_root()
    assert reply.encoded_data == ob.data()
    exp = ob.all_slices()
    size = len(exp) // 3072
    assert len(reply.encoded_slice) == 3072
    for i, s in enumerate(reply.encoded_slice):
        assert s == exp[i * size:(i + 1) * size], f"slice {i}"


def test_production_encoded_data(prod, oracle):
    params, seed, payload, reply = prod
    d = params.dims
    N = d.raw_blob_size
    data = reply.encoded_data
    assert len(data) == 3 * N * 32
    # coset 0 is the raw blob: 31-byte chunks + a zero byte
    raw = gpu_mod_raw(payload, d)
    c0 = np.frombuffer(data[:N * 32], dtype=np.uint8).reshape(N, 32)
    assert np.array_equal(c0[:, :31], np.frombuffer(raw, dtype=np.uint8).reshape(N, 31))
    assert not c0[:, 31].any()
    # cosets 1, 2: to_coset_blob of the column-major points (encode.rs:135-158)
    pts = c0.reshape(d.rows, d.cols, 32).transpose(1, 0, 2).copy().tobytes()
    coeff = oracle.ntt(pts, inverse=True)
    for c in (1, 2):
        ev = oracle.ntt(coeff, coset_idx=c, coset_len=N)
        ev = np.frombuffer(ev, dtype=np.uint8).reshape(d.cols, d.rows, 32).transpose(1, 0, 2).copy().tobytes()
        assert data[c * N * 32:(c + 1) * N * 32] == ev, f"coset {c}"


def gpu_mod_raw(payload, d):
    buf = bytearray(d.max_blob_size)
    buf[:len(payload)] = payload
    buf[d.max_raw_data_size:] = len(payload).to_bytes(4, "little")
    return bytes(buf)


def test_production_merkle(prod, oracle):
    params, _, _, reply = prod
    roots = oracle.merkle_roots(10, 10, reply.encoded_data)
    s = reply.encoded_slice[0]
    off = 96 + 32 * 1024 + 8 + 128 * 10 + 64
    assert s[off:off + 96] == roots
    assert reply.storage_root == oracle.keccak256(oracle.keccak256(roots[:64]) + roots[64:])


def test_production_amt_scalar_domain(prod, prod_oracle, gpu_pkg, oracle):
    """Every AMT output of all three cosets -- the commitment tree, the ten
    proof layers and the high commitment, 3 x (4R - 2) nodes -- equals
    (sum_t scalar_t * s_t) * G1 with s_t the param scalars of the seeded tau,
    both as the device wrote them (zg_encode_device) and as the oracle's
    EC-domain encode computed them, and the commitment is the reply's."""
    params, seed, payload, reply = prod
    N = params.dims.raw_blob_size
    R = 1024
    exp = [oracle.amt_scalar_domain(10, 10, seed, c, reply.encoded_data[c * N * 32:(c + 1) * N * 32])
           for c in range(3)]
    assert exp[0][:64] == exp[1][:64] == exp[2][:64]
    com = exp[0][:64]
    assert reply.erasure_commitment[:63] == com[:63]
    assert reply.erasure_commitment[63] == com[63] & 0x3f
    torch = torch_mod()
    L = gpu_pkg.lib()
    tp = dev(payload)
    db = gpu_pkg._DeviceBlob()
    assert L.zg_encode_device(params.handle, ctypes.c_void_p(tp.data_ptr()), len(payload), None,
                              ctypes.byref(db)) == 0, L.zg_last_error()
    nodes = host(device_view(db.amt_outputs, 3 * (4 * R - 2) * 64))
    ob = prod_oracle[1]
    for c in range(3):
        got = nodes[c * (4 * R - 2) * 64:(c + 1) * (4 * R - 2) * 64]
        for k in range(4 * R - 2):
            assert got[64 * k:64 * k + 64] == exp[c][64 * k:64 * k + 64], (c, k)
        assert ob.amt_outputs(c) == exp[c], c


def test_production_slices_verify(prod, oracle):
    params, seed, _, reply = prod
    basis = b"".join(params.param_line(c, 10) for c in range(3))
    vp = oracle.verify_params(10, 10, seed, basis)
    rnd = random.Random(7)
    for i in [0, 1023, 1024, 3071] + rnd.sample(range(3072), 4):
        rc, det = oracle.verify(vp, reply.encoded_slice[i], reply.erasure_commitment, reply.storage_root)
        assert rc == zgo.V_OK, (i, rc, det)


def test_production_recovery_round_trip(prod, gpu_pkg):
    """1024 x 1024 blob: the payload back from a seeded random half of the
    3072 rows, from the two parity cosets alone and from exactly R rows."""
    params, _, payload, reply = prod
    R, C = 1024, 1024
    data = reply.encoded_data
    rows = {i: data[i * C * 32:(i + 1) * C * 32] for i in range(3 * R)}
    rnd = random.Random(21)
    for ids in (rnd.sample(range(3 * R), 3 * R // 2), range(R, 3 * R), rnd.sample(range(3 * R), R)):
        assert gpu_pkg.recover_from_da_slice(params, {i: rows[i] for i in ids}) == payload
    bad = {i: rows[i] for i in rnd.sample(range(3 * R), R - 1)}
    with pytest.raises(gpu_pkg.RecoveryError, match="Not enough valid lines"):
        gpu_pkg.recover_from_da_slice(params, bad)


def test_production_batch_uneven(prod, gpu_pkg):
    """Uneven payloads through the pipelined batch path: every reply equals the
    plain per-blob path's (the full-size payload's reply is the fixture's)."""
    params, _, payload, reply = prod
    rng = np.random.default_rng(44)
    sizes = [65536, 20_000_000, 0]
    payloads = [payload] + [rng.integers(0, 256, n, dtype=np.uint8).tobytes() for n in sizes]
    svc = gpu_pkg.EncoderService(params)
    got = svc.process_batch(payloads, True)
    assert got[0] == reply
    for p, g in zip(payloads[1:], got[1:]):
        assert g == svc.process_data(p, True)


@pytest.mark.parametrize("fixture", ["encode_3x5.json", "encode_6x5.json"])
def test_encode_matches_golden_fixture(gpu_pkg, fixture):
    """The CUDA path against the independent pure-Python restatement's bytes
    (tests/golden/make_golden.py): an 8 x 32 blob and the reference's own
    64 x 32 test setting with a full payload."""
    import hashlib
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", fixture)))["encode"]
    params = gpu_pkg.ZgEncoderParams.from_seed(g["log_row"], g["log_col"], g["seed"])
    reply = gpu_pkg.EncoderService(params).process_data(bytes.fromhex(g["payload_hex"]), True)
    assert reply.erasure_commitment.hex() == g["erasure_commitment"]
    assert reply.storage_root.hex() == g["file_root"]
    assert hashlib.sha256(reply.encoded_data).hexdigest() == g["encoded_data_sha256"]
    assert [hashlib.sha256(s).hexdigest() for s in reply.encoded_slice] == g["slice_sha256"]
    params.close()
