"""The multi-GPU harness of bench.py (independent replicas, weak scaling) on
CPU: two gloo ranks take the barrier and the max-over-ranks steps of the
timed region, and the reference arm does no work on ranks other than 0."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    r = bench.Ranks(dist, "cpu")
    r.barrier()
    t = r.max(1.0 + rank)  # per-rank timed seconds
    r.barrier()
    q.put((rank, t, bench.job_value(world, 5, t)))
    dist.destroy_process_group()


def test_two_gloo_ranks_max_over_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank sees the slowest rank's time; 2 ranks x 5 blobs in 2 s
    assert res == [(0, 2.0, 5.0), (1, 2.0, 5.0)]


def test_reference_arm_only_on_rank0(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class A:
        cpu_sample = 8
        warmup = 0
        steps = 1
        gpus = 2
    bench.reference_arm(A(), 1)
    assert capsys.readouterr().out == ""
