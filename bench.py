#!/usr/bin/env python
"""Throughput benchmark of the B200 blob encoder.

Workload: the plain per-blob GPU path at production shape -- one blob of
1024 x 1024 BN254 Fr scalars built from a full MAX_RAW_DATA_SIZE payload of
seeded random bytes, RS-extended to 3 cosets (3072 rows), AMT commitment and
proofs for every row (G1 MSMs against device-resident params of a seeded
tau), keccak Merkle tree, and the 3072 serialized EncodedSlices.

  value : blobs/s with the payload already in HBM (zg_encode_device), each
          step timed with CUDA events on the launching stream; L2 is flushed
          between steps (256 MiB write, outside the events)
  e2e   : blobs/s through the C ABI's request pipeline (zg_submit / zg_wait,
          the serving path behind EncoderService) with the payload in pinned
          host memory: H2D of the payload, the encode and the D2H of the full
          reply (3072 slices + 96 MiB encoded data), each reply consumed and
          freed as it completes; `plain_value` is the same through the
          blocking per-blob zg_encode (process_data)
  batched_uneven : blobs/s of the pipelined path over blobs of uneven
          payload size L ~ U[64 KiB, MAX_RAW_DATA_SIZE] (seeded)
  serving : Poisson arrivals of requests (payload log-uniform on [4 KiB,
          MAX_RAW_DATA_SIZE], 10 % recovery requests from 1536 of the 3072
          rows, each result checked) through the pipeline: completed
          requests/s and p50 / p99 latency from arrival to result

  cpu_baseline : one full blob of the C++ restatement of the reference CPU
          path (oracle/, all host threads, the reference's prove.rs
          decomposition and ark-ec's signed-digit MSM), on the same payload;
          its file root is checked against the GPU's

Multi-GPU: one process per GPU, independent replicas (weak scaling), max of
the per-rank times. `--impl reference` times the same CPU restatement on full
blobs, one coset per step (three steps make one blob; the reference itself is
Rust and cannot be built here).
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "encoded blobs/s (1024x1024 Fr blob)"
UNIT = "blobs/s"
LOG_ROW = LOG_COL = 10
PARAM_SEED = 2024
DATA_SEED = 222
R = 1 << LOG_ROW
N = 1 << (LOG_ROW + LOG_COL)
PAYLOAD = 31 * N - 4                      # MAX_RAW_DATA_SIZE
SLICE_SIZE = 312 + 32 * (1 << LOG_COL) + 160 * LOG_ROW
# algorithmic work per blob: the reference GPU-plugin decomposition (36 864 chunk MSMs of 1024 points)
MSM_ADDS = 36864 * 40960                  # 36 864 MSMs x 1024 pts, signed 8-bit windows
MSM_IMAD = MSM_ADDS * 10 * 264            # 10 Fq mul per mixed add, 264 32-bit IMAD per Fq mul
RS_BYTES = 201_326_592                    # 3 transforms x (read + write 32 MiB)
RS_FR_MULS = 37_224_448                   # Fr products of the three RS passes (counted from the kernels)
KECCAK_F = 1_179_645                      # 393 216 x 2 leaf permutations + 393 213 node permutations
MERKLE_BYTES = 138_411_744                # 393 216 x 256 B leaves + 393 213 x 96 B nodes
D2H_BYTES = 3 * R * SLICE_SIZE + 3 * N * 32 + 64 * 3 + 96 + 32
CONFIG = {
    "workload": "plain per-blob GPU path: 1 blob of 1024x1024 Fr (full 32505852-byte payload), "
                "3-coset RS extension, AMT commitment + 3072 slice proofs, keccak Merkle, slice serialization",
    "log_row": LOG_ROW, "log_col": LOG_COL, "payload_bytes": PAYLOAD, "params": "seeded tau (seed 2024)",
    "l2": "flushed between timed steps (256 MiB device write outside the CUDA events); "
          "each step also streams 2.25 GiB of params",
}


def _line_unit_logs(lr, lc):
    """Per AMT line (quotients 0 .. lr - 1, the basis, the high line): the
    log2 of its node size and of its wide unit, min(16, log2 node) (units of
    2^16 points are pairs of 2^15-point sort units sharing 2^15 buckets)."""
    n = 1 << (lr + lc)
    out = []
    for line in range(lr + 2):
        node = n if line == lr + 1 else (1 << lc if line == lr else n >> (line + 1))
        lg = node.bit_length() - 1
        out.append((lg, min(16, lg)))
    return out


def _wide(lc, lg, u, wide_classes):
    # classes by unit size, largest first: class index 16 - u
    return lc == 10 and lg > 10 and 16 - u < wide_classes


def executed_mixed_adds(lr, lc, wide_classes=6):
    """Bucket additions of table points this build runs per blob (random
    scalars): the lines whose nodes are single chunks use 24 windows per
    point; with 1024 columns every other line uses units of 2^u points, u =
    min(16, log2 node), and floor(254 / c) + 1 windows of c = min(u, 15) + 1
    bits, when its class (index 16 - u, largest unit first) is among the first
    `wide_classes` in use, else 11-bit windows per chunk."""
    n, total = 1 << (lr + lc), 0
    for lg, u in _line_unit_logs(lr, lc):
        if _wide(lc, lg, u, wide_classes):
            total += 3 * n * (254 // (min(u, 15) + 1) + 1)
        else:
            total += 3 * n * 24
    return total


def executed_full_adds(lr, lc, wide_classes=6):
    """XYZZ + XYZZ additions of the bucket reductions per blob: per MSM work
    item (1024 buckets each: 3 x rows per line, half as many on the lines of
    2^16-point units) the running sums of its 128 threads (two per bucket;
    the merges of a bucket's extra task partials are not counted) and the
    combine of the 128 (T, S) partials (2 x 127 additions plus 3
    doublings)."""
    items = 0
    for lg, u in _line_unit_logs(lr, lc):
        merged = _wide(lc, lg, u, wide_classes) and u == 16
        items += 3 * ((1 << lr) >> (1 if merged else 0))
    return items * (2 * 1024 + 2 * 127 + 3)


def ntt_muls(logn):
    """Twiddle products of one 2^logn-point transform of the device core: the
    first two stages (twiddles 1 and w^(n/4)) cost n/4 products, every later
    stage n/2."""
    n = 1 << logn
    return logn if logn < 2 else n // 4 + (logn - 2) * n // 2


def zg_ntt_products(batch, logn, inverse, coset):
    """Fr products of one zg_ntt call: up to 2^11 points one transform per
    vector (coset shift 1 product per element from a full table, 1/n 1
    product); above, the four-step split (lc = ceil(logn / 2)): column
    transforms, 2 products per element for the twiddles between the passes,
    row transforms (coset shift 2 products per element from split tables)."""
    n = 1 << logn
    if logn <= 11:
        per = ntt_muls(logn) + (n if coset else 0) + (n if inverse else 0)
    else:
        lc = (logn + 1) // 2
        lr = logn - lc
        per = (1 << lc) * ntt_muls(lr) + 2 * n + (1 << lr) * ntt_muls(lc) \
            + (2 * n if coset else 0) + (n if inverse else 0)
    return batch * per


def set_dims(lr, lc):
    """Switch the module constants to another blob shape (profiling runs)."""
    global LOG_ROW, LOG_COL, R, N, PAYLOAD, SLICE_SIZE, MSM_ADDS, MSM_IMAD, RS_BYTES, MERKLE_BYTES, D2H_BYTES, \
        RS_FR_MULS, KECCAK_F
    if (lr, lc) == (LOG_ROW, LOG_COL):
        return
    LOG_ROW, LOG_COL = lr, lc
    R, N = 1 << lr, 1 << (lr + lc)
    PAYLOAD = 31 * N - 4
    SLICE_SIZE = 312 + 32 * (1 << lc) + 160 * lr
    MSM_ADDS = 3 * (lr + 2) * R * 32 * ((1 << lc) + 256)
    MSM_IMAD = MSM_ADDS * 10 * 264
    RS_BYTES = 3 * 2 * N * 32
    C_ = 1 << lc
    # rows pass: NTT + 2 twiddle products per element; column pass: iNTT, then
    # per coset 2 scale + NTT + 2 twiddle products; rows NTT (the passes run
    # on canonical values, with no conversion products)
    RS_FR_MULS = R * (ntt_muls(lc) + 2 * C_) + C_ * (ntt_muls(lr) + 2 * (4 * R + ntt_muls(lr))) \
        + 2 * R * ntt_muls(lc)
    KECCAK_F = 3 * N // 8 * 2 + 3 * N // 8 - 3
    leaves = 3 * N // 8
    MERKLE_BYTES = leaves * 256 + (leaves - 3) * 96
    D2H_BYTES = 3 * R * SLICE_SIZE + 3 * N * 32 + 64 * 3 + 96 + 32
    CONFIG["workload"] = f"profiling shape {R}x{1 << lc} (not the benchmark workload)"
    CONFIG["log_row"], CONFIG["log_col"], CONFIG["payload_bytes"] = lr, lc, PAYLOAD


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-blobs", type=int, default=32, help="blobs in the batched-uneven sample")
    ap.add_argument("--serve-rate", default="3,6,9",
                    help="Poisson arrival rates of the serving sample (1/s, comma-separated sweep)")
    ap.add_argument("--serve-requests", type=int, default=128, help="requests per serving sample (0 = skip)")
    ap.add_argument("--no-serve-plain", action="store_true",
                    help="skip serving the same arrivals through the blocking per-blob path")
    ap.add_argument("--verify-sample", type=int, default=4,
                    help="slices of the CPU verification sample (0 = skip the verification measurement)")
    ap.add_argument("--micro", action="store_true",
                    help="kernel microbenchmarks instead of the blob benchmark: single MSMs of 2^16/2^18/2^20 "
                         "points (uniform and blob-like scalars), NTTs (1024 x 2^10, 64 x 2^14, 1 x 2^20; "
                         "forward, inverse, coset), Keccak Merkle over 3072 x 1024 x 32 B")
    ap.add_argument("--micro-cases", default="msm,ntt,merkle",
                    help="which microbenchmarks --micro runs (comma-separated subset of msm,ntt,merkle; without "
                         "msm no encoder context or params are built: profiling captures of the NTT kernels)")
    ap.add_argument("--tuning", default="",
                    help="PRODUCT,COLS,THREADS[,TASK[,WIDE_CLASSES]] (e.g. hybrid,1,256,64,6): use these kernel "
                         "choices instead of autotuning "
                         "(profiling runs, where the autotuner's own timings would be distorted)")
    ap.add_argument("--msm-window-bits", type=int, default=0,
                    help="0 = the context's choice (11-bit fixed-base tables when they fit), 8 = 8-bit windows "
                         "without tables (a few GB on the device: profiling captures of the RS / Merkle kernels)")
    ap.add_argument("--dims", default="10,10",
                    help="LOG_ROW,LOG_COL of the blob; the default 10,10 is the benchmark workload, smaller "
                         "shapes are for profiling captures")
    return ap.parse_args()


def load_pkg():
    import __graft_entry__
    return __graft_entry__.load_package()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "of measured"
    except Exception:
        return 6650.0, "of fallback"


def profile_traffic():
    """dram bytes per MSM launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "msm_fb_accum_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch="):
                    return int(line.split("=", 1)[1].strip())
    except OSError:
        pass
    return None


class ClockSampler:
    FIELDS = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.tmp.flush()
        self.tmp.seek(0)
        rows = [l.strip().split(", ") for l in self.tmp.read().splitlines() if l.strip()]
        os.unlink(self.tmp.name)
        if self.uuid:
            mine = [r for r in rows if len(r) > 1 and r[1].replace("GPU-", "") == self.uuid.replace("GPU-", "")]
            rows = mine or rows
        sm = [float(r[2]) for r in rows if len(r) > 3 and r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if len(r) > 3 and r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, name in enumerate(names):
                if len(r) > 6 + k and r[6 + k].strip() == "Active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


class Ranks:
    """Barrier and max-over-ranks around the timed regions (one process per
    GPU over NCCL; gloo and CPU tensors in the multi-rank tests). Every rank
    takes the same collective steps in the same order."""

    def __init__(self, dist, device):
        self.dist, self.device = dist, device

    def _sync(self):
        if self.device == "cuda":
            import torch
            torch.cuda.synchronize()

    def barrier(self):
        self._sync()
        if self.dist is not None:
            self.dist.barrier()
        self._sync()

    def max(self, x):
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())


def job_value(world, steps, max_seconds):
    """Whole-job throughput: every rank processed `steps` blobs; the job took
    the slowest rank's time."""
    return world * steps / max_seconds


def dist_setup():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


CPU_SAMPLE = ("full 1024x1024 blobs of the C++ restatement of the reference CPU path (oracle/), one coset per "
              "step, 3 steps = 1 blob: RawData -> RawBlob -> 3-coset RS extension (to_coset_blob, ark-poly style "
              "radix-2), AMT commitment + proofs with the reference CPU decomposition (prove.rs:58-102: layer d = "
              "2^d MSMs of 2^(20-d) points, 1024 x 1024 commitment tree, one 2^20 high MSM; each MSM ark-ec's "
              "signed-digit bucket method, windows in parallel), keccak Merkle tree, 3072 serialized slices; "
              "params of the seeded tau built on the CPU; nothing sampled or scaled (the Rust reference cannot "
              "be built here)")


def cpu_blob_steps(o, params, payload, warmup, steps):
    """Times `steps` coset steps of the restated CPU path after `warmup`
    untimed ones, starting each timed run on a blob boundary. Returns
    (blobs/s, total seconds, per-step seconds, file root of the last blob)."""
    job = o.cpu_job(params, payload)
    done = 0
    root = None
    while done < warmup or done % 3:
        _, r, _ = job.step()
        root = r or root
        done += 1
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        _, r, _ = job.step()
        times.append(time.perf_counter() - t0)
        root = r or root
    total = sum(times)
    return (steps / 3.0) / total, total, times, root


def cpu_oracle():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import zgo
    return zgo.Oracle()


def reference_arm(args, rank):
    """The reference's CPU path (its C++ restatement, oracle/) on all host
    threads, full blobs, one coset per step."""
    if rank != 0:
        return
    o = cpu_oracle()
    t0 = time.perf_counter()
    params = o.params(LOG_ROW, LOG_COL, PARAM_SEED)
    t_params = time.perf_counter() - t0
    payload = np.random.default_rng(DATA_SEED).integers(0, 256, size=PAYLOAD, dtype=np.uint8).tobytes()
    value, total, times, _ = cpu_blob_steps(o, params, payload, args.warmup, args.steps)
    cores = o.L.zgo_num_threads()
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded random payload bytes)",
        "config": CONFIG, "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": CPU_SAMPLE + f"; value = ({args.steps} steps / 3) blobs / timed seconds",
                         "params_build_s": t_params,
                         "step_s": {"min": min(times), "max": max(times)}},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


class Pipe:
    """The C ABI's request pipeline, driven without Python-side reply copies."""

    def __init__(self, pkg, params):
        self.pkg, self.L, self.h = pkg, pkg.lib(), params.handle

    def _submit(self, q):
        t = ctypes.c_uint64()
        rc = self.L.zg_submit(self.h, ctypes.byref(q), ctypes.byref(t))
        assert rc == 0, self.L.zg_last_error()
        return t.value

    def submit_encode(self, ptr, n, require_data=1):
        q = self.pkg._Request()
        q.kind, q.data, q.len, q.require_data = 0, ptr, n, require_data
        return self._submit(q)

    def submit_recover(self, rec):
        ids, bufs, lens, n, _ = rec
        q = self.pkg._Request()
        q.kind, q.row_ids, q.rows, q.row_lens, q.n_rows = 1, ids, bufs, lens, n
        return self._submit(q)

    def wait(self, t):
        r = ctypes.c_void_p()
        rc = self.L.zg_wait(self.h, t, -1, ctypes.byref(r))
        assert rc == 0, self.L.zg_last_error()
        return r

    def payload(self, r):
        n = ctypes.c_size_t()
        p = self.L.zg_reply_payload(r, ctypes.byref(n))
        return ctypes.string_at(p, n.value) if n.value else b""

    def free(self, r):
        self.L.zg_reply_free(r)


def recovery_inputs(rows, seeds):
    """ctypes arrays of 1536 of the 3072 rows (seeded erasures), built once."""
    out = []
    for sd in seeds:
        ids = sorted(np.random.default_rng(sd).choice(3 * R, size=3 * R // 2, replace=False).tolist())
        keep = [rows[i] for i in ids]
        arr = (ctypes.c_uint64 * len(ids))(*ids)
        bufs = (ctypes.c_char_p * len(ids))(*keep)
        lens = (ctypes.c_size_t * len(ids))(*[len(x) for x in keep])
        out.append((arr, bufs, lens, len(ids), keep))
    return out


def serving_run(pkg, params, pipe, h_ptr, full_payload, recs, rate, n, seed, plain=False):
    """Poisson arrivals (rate per s) of n requests: 10 % recovery requests (one
    of `recs`, checked against the original payload), the rest encodes of a
    payload log-uniform on [4 KiB, MAX_RAW_DATA_SIZE] (a prefix of the pinned
    payload). Pipeline: a submitter thread submits at each arrival and the
    caller collects results in order. Plain: one worker serves the arrivals
    in order through the blocking zg_encode / zg_recover."""
    import queue
    import threading
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, n)
    arrive = np.cumsum(gaps) - gaps[0]
    kinds = rng.random(n) < 0.10
    sizes = np.exp(rng.uniform(np.log(4096), np.log(PAYLOAD), n)).astype(np.int64)
    which = rng.integers(0, len(recs), n)
    L = pkg.lib()
    lat = [0.0] * n
    bad = []
    t0 = time.perf_counter() + 0.05
    if not plain:
        q = queue.Queue()

        def submitter():
            for i in range(n):
                d = t0 + arrive[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                t = pipe.submit_recover(recs[which[i]]) if kinds[i] else pipe.submit_encode(h_ptr, int(sizes[i]))
                q.put((i, t))

        th = threading.Thread(target=submitter)
        th.start()
        for _ in range(n):
            i, t = q.get()
            r = pipe.wait(t)
            done = time.perf_counter()
            if kinds[i] and pipe.payload(r) != full_payload:
                bad.append(i)
            pipe.free(r)
            lat[i] = done - (t0 + arrive[i])
        th.join()
    else:
        for i in range(n):
            d = t0 + arrive[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            if kinds[i]:
                ids, bufs, lens, k, _ = recs[which[i]]
                out = ctypes.create_string_buffer(PAYLOAD)
                olen = ctypes.c_size_t()
                rc = L.zg_recover(params.handle, ids, bufs, lens, k, out, PAYLOAD, ctypes.byref(olen))
                assert rc == 0, L.zg_last_error()
                if out.raw[:olen.value] != full_payload:
                    bad.append(i)
            else:
                r = ctypes.c_void_p()
                rc = L.zg_encode(params.handle, ctypes.cast(ctypes.c_void_p(h_ptr), ctypes.c_char_p),
                                 int(sizes[i]), 1, ctypes.byref(r))
                assert rc == 0, L.zg_last_error()
                L.zg_reply_free(r)
            lat[i] = time.perf_counter() - (t0 + arrive[i])
    span = max(arrive[i] + lat[i] for i in range(n))
    lat_ms = np.array(lat) * 1000.0
    return {
        "path": "plain per-blob (blocking zg_encode / zg_recover)" if plain else "pipeline (zg_submit / zg_wait)",
        "arrival_rate_per_s": rate, "requests": n, "recovery_requests": int(kinds.sum()),
        "completed_per_s": n / span, "p50_ms": float(np.percentile(lat_ms, 50)),
        "p99_ms": float(np.percentile(lat_ms, 99)), "mean_ms": float(lat_ms.mean()),
        "payload_mean_bytes": float(sizes[~kinds].mean()) if (~kinds).any() else 0.0,
        "recovery_mismatches": len(bad),
    }


def micro(args):
    """Kernel microbenchmarks on one GPU, one JSON line. Each case: 3 warm-up
    calls, then `steps` calls timed one by one with CUDA events on the
    launching stream, L2 flushed (256 MiB write) between calls outside the
    events; the median is reported."""
    import torch
    pkg = load_pkg()
    L = pkg.lib()
    cases = set(args.micro_cases.split(","))
    params = pkg.ZgEncoderParams.from_seed(LOG_ROW, LOG_COL, PARAM_SEED) if "msm" in cases else None
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234)
    hbm, hbm_tag = measured_peaks()
    steps = max(3, args.steps)

    def timed(fn):
        for _ in range(3):
            fn()
        ts = []
        for k in range(steps):
            flush.fill_(k & 0xff)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    def rand_bytes(n):
        return torch.randint(0, 256, (n,), dtype=torch.uint8, device="cuda", generator=gen)

    out = {"msm": [], "ntt": [], "keccak_merkle": None}
    d_out = torch.empty(64, dtype=torch.uint8, device="cuda")
    basis_line = LOG_ROW  # lines: quotients 0..LOG_ROW-1, basis, high basis
    rng = np.random.default_rng(3)
    for logn in ((16, 18, 20) if "msm" in cases else ()):
        n = 1 << logn
        for kind in ("uniform", "blob"):
            sc = rand_bytes(32 * n).view(n, 32)
            z = 0.0
            if kind == "uniform":
                sc[:, 31] &= 0x1f  # below 2^253 < r
            else:  # 31-byte scalars (< 2^248), zero suffix of a fraction z ~ U[0, 0.9]
                z = float(rng.uniform(0, 0.9))
                sc[:, 31] = 0
                sc[int(np.ceil((1 - z) * n)):] = 0
            sc = sc.contiguous()

            def run():
                rc = L.zg_ctx_msm(params.handle, 0, basis_line, ctypes.c_void_p(sc.data_ptr()), n,
                                  ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
                assert rc == 0, L.zg_last_error()

            ms = timed(run)
            nz = int((1 - z) * n) if kind == "blob" else n
            out["msm"].append({"points": n, "scalars": kind, "zero_fraction": round(z, 3), "ms": ms,
                               "points_per_s": n / (ms / 1000.0), "nonzero_points_per_s": nz / (ms / 1000.0)})
    fr_probe = pkg.probe_products(0, "imad") * 1e9 if "ntt" in cases else 0.0  # G/s -> /s
    for batch, logn in (((1024, 10), (64, 14), (1, 20)) if "ntt" in cases else ()):
        n = 1 << logn
        for mode, inv, coset in (("forward", 0, 0), ("inverse", 1, 0), ("coset1", 0, 1)):
            v = rand_bytes(32 * n * batch).view(n * batch, 32)
            v[:, 31] &= 0x2f  # canonical: below r

            def run():
                rc = L.zg_ntt(ctypes.c_void_p(v.data_ptr()), logn, batch, inv, coset,
                              ctypes.c_void_p(stream.cuda_stream))
                assert rc == 0, L.zg_last_error()

            ms = timed(run)
            byts = 2 * n * batch * 32
            prods = zg_ntt_products(batch, logn, inv, coset)
            out["ntt"].append({"batch": batch, "log_n": logn, "mode": mode, "ms": ms,
                               "algorithmic_bytes": byts, "achieved_gbs": byts / (ms / 1000) / 1e9,
                               "hbm_frac": byts / (ms / 1000) / 1e9 / hbm,
                               "butterfly_mul_per_s": batch * (n // 2) * logn / (ms / 1000),
                               "fr_products": prods, "fr_products_per_s": prods / (ms / 1000),
                               "product_frac": prods / (ms / 1000) / fr_probe})
    if "merkle" not in cases:
        res = {"micro": out, "fr_product_probe_per_s": fr_probe, "hbm_peak_gbs": hbm, "hbm_peak_src": hbm_tag,
               "timing": f"median of {steps} calls, CUDA events on the launching stream, L2 flushed between calls"}
        print(json.dumps(res), flush=True)
        if params:
            params.close()
        return
    items = rand_bytes(3 * N * 32)
    roots = torch.empty(96, dtype=torch.uint8, device="cuda")

    def run():
        rc = L.zg_merkle_roots(ctypes.c_void_p(items.data_ptr()), 3 * N, ctypes.c_void_p(roots.data_ptr()),
                               ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.zg_last_error()

    ms = timed(run)
    out["keccak_merkle"] = {"rows": 3 * R, "row_bytes": 32 << LOG_COL, "ms": ms,
                            "algorithmic_bytes": MERKLE_BYTES,
                            "achieved_gbs": MERKLE_BYTES / (ms / 1000) / 1e9,
                            "hbm_frac": MERKLE_BYTES / (ms / 1000) / 1e9 / hbm,
                            "keccak_f_per_s": (3 * N // 8 * 2 + 3 * N // 8 - 3) / (ms / 1000)}
    res = {"micro": out, "imad_probe_gimad_s": pkg.probe_imad(0), "fr_product_probe_per_s": fr_probe,
           "hbm_peak_gbs": hbm, "hbm_peak_src": hbm_tag,
           "timing": f"median of {steps} calls, CUDA events on the launching stream, L2 flushed between calls",
           "params": "seeded tau (seed 2024), 1024 x 1024, MSM bases = coset-0 basis line"}
    print(json.dumps(res), flush=True)
    if params:
        params.close()


def main():
    args = parse()
    set_dims(*[int(x) for x in args.dims.split(",")])
    rank, world, local = dist_setup()
    if args.micro:
        micro(args)
        return
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    pkg = load_pkg()
    L = pkg.lib()
    params = pkg.ZgEncoderParams.from_seed(LOG_ROW, LOG_COL, PARAM_SEED, device=local,
                                           msm_window_bits=args.msm_window_bits)
    # the kernels' free choices (MSM product kind, RS tile shape), timed on a
    # synthetic blob before any measurement
    if args.tuning:
        f = args.tuning.split(",")
        params.set_tuning(f[0], int(f[1]), int(f[2]), msm_task=int(f[3]) if len(f) > 3 else 64,
                          msm_wide_classes=int(f[4]) if len(f) > 4 else None)
        tuning = dict(params.tuning(), source="--tuning")
    else:
        tuning = params.autotune()
    payload = np.random.default_rng(DATA_SEED + rank).integers(0, 256, size=PAYLOAD, dtype=np.uint8)
    d_payload = torch.from_numpy(payload.copy()).cuda()
    h_payload = torch.from_numpy(payload.copy()).pin_memory()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()  # the encode, its events and the L2 flush share this stream
    torch.cuda.set_stream(stream)
    db = pkg._DeviceBlob()

    def encode_device():
        rc = L.zg_encode_device(params.handle, ctypes.c_void_p(d_payload.data_ptr()), PAYLOAD,
                                ctypes.c_void_p(stream.cuda_stream), ctypes.byref(db))
        assert rc == 0, L.zg_last_error()

    pipe = Pipe(pkg, params)
    h_ptr = h_payload.data_ptr()

    def encode_e2e_plain():
        r = ctypes.c_void_p()
        rc = L.zg_encode(params.handle, ctypes.cast(ctypes.c_void_p(h_ptr), ctypes.c_char_p),
                         PAYLOAD, 1, ctypes.byref(r))
        assert rc == 0, L.zg_last_error()
        L.zg_reply_free(r)  # the reply is host-resident once zg_encode returns

    def pipeline(sizes):
        ts = [pipe.submit_encode(h_ptr, int(n)) for n in sizes]
        for t in ts:
            pipe.free(pipe.wait(t))  # the reply is host-resident once zg_wait returns

    ranks = Ranks(dist, "cuda")
    barrier, max_over_ranks = ranks.barrier, ranks.max

    # warm-up (the pipeline's first blobs also capture its graphs and fill the
    # pinned reply pool)
    for _ in range(args.warmup):
        encode_device()
    encode_e2e_plain()
    pipeline([PAYLOAD] * max(3, args.warmup))
    torch.cuda.synchronize()

    # phase profile (one untimed encode with events between phases)
    params.set_profiling(True)
    encode_device()
    torch.cuda.synchronize()
    phases = params.phase_times()
    params.set_profiling(False)
    imad = pkg.probe_imad(local)

    # timed: device-resident
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    launches0 = params.launches()
    clocks.start()
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        starts[k].record(stream)
        encode_device()
        ends[k].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = params.launches() - launches0
    barrier()
    total_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    total_ms = max_over_ranks(total_ms)
    value = job_value(world, args.steps, total_ms / 1000.0)

    # timed: end to end through the public API (pipeline), then the blocking path
    barrier()
    t0 = time.perf_counter()
    pipeline([PAYLOAD] * args.steps)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    barrier()
    e2e_value = job_value(world, args.steps, e2e_s)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        encode_e2e_plain()
    torch.cuda.synchronize()
    plain_s = max_over_ranks(time.perf_counter() - t0)
    barrier()
    e2e_plain = job_value(world, args.steps, plain_s)

    # batched uneven payloads (one zg_encode_batch call of all the blobs) and
    # a serving sample (single-GPU runs)
    extra = {}
    if world == 1 and args.batch_blobs > 0:
        sizes = np.random.default_rng(4).integers(64 << 10, PAYLOAD + 1, args.batch_blobs)
        n = len(sizes)
        ptrs = (ctypes.c_void_p * n)(*([h_ptr] * n))
        lens = (ctypes.c_size_t * n)(*[int(x) for x in sizes])
        outs = (ctypes.c_void_p * n)()

        def batch_call():
            rc = L.zg_encode_batch(params.handle, n, ptrs, lens, 1, outs)
            assert rc == 0, L.zg_last_error()
            for i in range(n):
                L.zg_reply_free(outs[i])

        modes = {}
        for name, fuse in (("fused_pairs", 2), ("one_blob_per_launch", 1)):
            params.set_pipeline(blobs_per_launch=fuse)
            batch_call()  # units and their graphs come up
            st0 = params.pipeline_stats()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            batch_call()
            bt = time.perf_counter() - t0
            st1 = params.pipeline_stats()
            modes[name] = {"value": n / bt, "seconds": bt, "units": st1["units"],
                           "launches_by_blobs": {k: st1["launches_by_blobs"][k] - st0["launches_by_blobs"][k]
                                                 for k in st1["launches_by_blobs"]},
                           "max_in_flight": st1["max_in_flight"]}
        params.set_pipeline()
        t0 = time.perf_counter()
        for x in sizes:
            r = ctypes.c_void_p()
            rc = L.zg_encode(params.handle, ctypes.cast(ctypes.c_void_p(h_ptr), ctypes.c_char_p), int(x), 1,
                             ctypes.byref(r))
            assert rc == 0, L.zg_last_error()
            L.zg_reply_free(r)
        plain_bt = time.perf_counter() - t0
        extra["batched_uneven"] = {
            "blobs": n, "value": modes["fused_pairs"]["value"], "unit": UNIT,
            "payload_mean_bytes": float(sizes.mean()),
            "path": "zg_encode_batch: pipeline units of 2 blob slots, each pair fused into one launch sequence "
                    "(one bucket accumulation over both blobs' MSMs) from a captured CUDA graph; pinned host "
                    "payloads, full replies",
            "modes": modes,
            "plain_value": n / plain_bt, "plain_path": "blocking zg_encode per blob",
            "fused_over_plain": modes["fused_pairs"]["value"] / (n / plain_bt),
        }
    if world == 1 and args.serve_requests > 0:
        rows_reply = pkg.EncoderService(params).process_data(payload.tobytes(), True)
        rows = [rows_reply.encoded_data[i * (32 << LOG_COL):(i + 1) * (32 << LOG_COL)] for i in range(3 * R)]
        recs = recovery_inputs(rows, [11, 12, 13])
        full = payload.tobytes()
        extra["serving"] = []
        for rate in [float(x) for x in str(args.serve_rate).split(",") if x]:
            st0 = params.pipeline_stats()
            row = serving_run(pkg, params, pipe, h_ptr, full, recs, rate, args.serve_requests, 5)
            st1 = params.pipeline_stats()
            row["pipeline"] = {"units": st1["units"], "max_in_flight": st1["max_in_flight"],
                               "launches_by_blobs": {k: st1["launches_by_blobs"][k] - st0["launches_by_blobs"][k]
                                                     for k in st1["launches_by_blobs"]}}
            extra["serving"].append(row)
            if not args.no_serve_plain:
                extra["serving"].append(serving_run(pkg, params, pipe, h_ptr, full, recs, rate,
                                                    args.serve_requests, 5, plain=True))

    # batched verification of every slice of one blob (EncodedSlice::verify for
    # 3072 slices through zg_verify_slices), beside the oracle's per-slice
    # verifier on a sample
    if world == 1 and args.verify_sample > 0 and args.msm_window_bits != 8:  # needs the fixed-base tables
        rep = pkg.EncoderService(params).process_data(payload.tobytes(), True)
        times = []
        for k in range(2):
            t0 = time.perf_counter()
            codes, _ = pkg.verify_slices(params, rep.encoded_slice, rep.erasure_commitment, rep.storage_root,
                                         seed=11 + k)
            times.append(time.perf_counter() - t0)
        ver = {"slices": len(rep.encoded_slice), "seconds": min(times),
               "slices_per_s": len(rep.encoded_slice) / min(times), "all_ok": all(c == 0 for c in codes),
               "path": "zg_verify_slices (host slice bytes in, verdicts out; GPU Merkle paths, MSM and Miller "
                       "loops, host final exponentiation)"}
        if not args.no_cpu_baseline:
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            import zgo
            o = zgo.Oracle()
            basis = b"".join(params.param_line(cs, LOG_ROW) for cs in range(3))
            vp = o.verify_params(LOG_ROW, LOG_COL, PARAM_SEED, basis)
            ids = list(range(0, 3 * R, max(1, 3 * R // args.verify_sample)))[:args.verify_sample]
            t0 = time.perf_counter()
            for i in ids:
                o.verify(vp, rep.encoded_slice[i], rep.erasure_commitment, rep.storage_root)
            dt = time.perf_counter() - t0
            ver["cpu_oracle"] = {"slices": len(ids), "seconds": dt, "slices_per_s": len(ids) / dt,
                                 "cores": o.L.zgo_num_threads(),
                                 "note": "C++ restatement of EncodedSlice::verify, one slice at a time"}
        extra["verify"] = ver

    hbm, hbm_tag = measured_peaks()
    t_msm = phases["msm"] / 1000.0
    achieved = MSM_IMAD / t_msm / 1e9
    wide_on = tuning.get("msm_wide_classes", 6)
    ex_mixed = executed_mixed_adds(LOG_ROW, LOG_COL, wide_on)
    ex_full = executed_full_adds(LOG_ROW, LOG_COL, wide_on)
    ex_prod = ex_mixed * 10 + ex_full * 14
    ex_imad = ex_prod * 264
    prod_by_kind = {k: pkg.probe_products(local, k) for k in pkg.MSM_PRODUCTS}
    prod_peak = prod_by_kind[tuning.get("msm_product", "hybrid")]
    roofline = {
        "kernel": "k_fb_accum", "bound": "imad", "achieved": achieved, "peak": imad, "unit": "G IMAD/s",
        "frac": achieved / imad, "traffic": profile_traffic(),
        "note": "work = 1509949440 mixed adds/blob x 10 Fq mul x 264 IMAD (reference decomposition; "
                f"this build executes {ex_mixed} table-point additions plus "
                "the bucket reductions, half of the products on the FP64 pipe, so frac may exceed 1); "
                "peak = live mad.lo.u32 probe on this GPU (of measured); traffic = dram bytes per launch "
                "from the committed ncu summary",
        "executed_mixed_adds": ex_mixed, "executed_full_adds": ex_full,
        "executed_frac": ex_imad / t_msm / 1e9 / imad,
        "executed_products_per_s": ex_prod / t_msm,
        "product_peak_per_s": prod_peak * 1e9,
        "product_frac": ex_prod / t_msm / 1e9 / prod_peak,
        "product_probe_by_kind": {k: v * 1e9 for k, v in prod_by_kind.items()},
        "product_note": "executed Fq products (mixed additions x 10 + XYZZ additions x 14) per second of the MSM "
                        "phase / the live product-throughput probe of the same product kind at the bucket "
                        "kernel's launch shape (zg_probe_products): how close the bucket loop runs to the rate "
                        "its field products can be issued",
        "executed_note": "the additions this build runs (mixed x 10 Fq products + XYZZ x 14) x 264 IMAD per "
                         "product / MSM phase time / the live IMAD probe: a utilisation of the integer pipe as if "
                         "every product ran there (the FP64-pipe share of the hybrid kinds counts as IMAD work)",
    }
    phase_roofs = {
        "rs_extension": {"bound": "hbm", "bytes": RS_BYTES, "ms": phases["rs"],
                         "achieved_gbs": RS_BYTES / (phases["rs"] / 1000) / 1e9, "peak_gbs": hbm,
                         "frac": RS_BYTES / (phases["rs"] / 1000) / 1e9 / hbm, "peak_src": hbm_tag,
                         # the passes are bound by their Fr products, not by HBM: the same
                         # IMAD-credited figure as the MSM roofline
                         "fr_muls": RS_FR_MULS,
                         "achieved_gimad": RS_FR_MULS * 264 / (phases["rs"] / 1000) / 1e9,
                         "imad_frac": RS_FR_MULS * 264 / (phases["rs"] / 1000) / 1e9 / imad},
        "merkle": {"bound": "hbm", "bytes": MERKLE_BYTES, "ms": phases["merkle"],
                   "achieved_gbs": MERKLE_BYTES / (phases["merkle"] / 1000) / 1e9, "peak_gbs": hbm,
                   "frac": MERKLE_BYTES / (phases["merkle"] / 1000) / 1e9 / hbm, "peak_src": hbm_tag,
                   "keccak_f": KECCAK_F, "keccak_f_per_s": KECCAK_F / (phases["merkle"] / 1000)},
        "phase_ms": phases,
    }
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded random payload bytes; params from a seeded tau)",
        "config": dict(CONFIG, tuning=tuning),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": PAYLOAD, "d2h_bytes_per_step": D2H_BYTES,
                "path": "zg_submit / zg_wait request pipeline", "plain_value": e2e_plain,
                "plain_path": "blocking zg_encode per blob"},
        "gpu_launches": launches, "clocks": clk, "roofline": roofline, "phase_rooflines": phase_roofs,
    }
    out.update(extra)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # one full blob (3 coset steps) of the restated CPU path on all host
        # threads, the same payload: its file root must equal the GPU's
        o = cpu_oracle()
        t0 = time.perf_counter()
        oparams = o.params(LOG_ROW, LOG_COL, PARAM_SEED)
        t_params = time.perf_counter() - t0
        v, total, times, root = cpu_blob_steps(o, oparams, payload.tobytes(), 0, 3)
        gpu_root = pkg.EncoderService(params).process_data(payload.tobytes(), False).storage_root
        out["cpu_baseline"] = {
            "value": v, "unit": UNIT, "cores": o.L.zgo_num_threads(), "kind": "port",
            "sample": "1 full blob (3 coset steps): " + CPU_SAMPLE,
            "detail": {"blob_s": total, "coset_step_s": times, "params_build_s": t_params,
                       "file_root_matches_gpu": root == gpu_root},
        }
    if rank == 0:
        print(json.dumps(out), flush=True)
    params.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
