"""The multi-GPU path of bench.py is replicas only: each rank renders its own
disjoint noise sequence of the full frame, and the job is timed by the
slowest rank. These checks run the host side of that with two gloo ranks on
the CPU (the oracle stands in for a GPU)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import bench
from oracle.binding import OracleTracer
from stargaze_b200 import workloads as W


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank: int, world: int, port: int, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # Per-rank timings: the job takes the slowest rank's.
        step_ms = [10.0 + rank, 20.0 - 5.0 * rank]
        total = bench.max_over_ranks(step_ms, dist, "cpu")
        # Each rank's image of the same frame from its own noise keys.
        wl = W.spheres_256(width=16, height=16, spp=8)
        t = OracleTracer((16, 16), W.render_options(wl, 8, noise_seed=bench.rank_noise_seed(rank)), threads=1)
        t.encode(wl.frame)
        out.put((rank, total, t.read_pixels()))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank_and_render_disjoint_noise():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict((r, (total, image)) for r, total, image in (out.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results[0][0] == results[1][0] == [11.0, 20.0]
    a, b = results[0][1], results[1][1]
    assert not np.array_equal(a, b)  # disjoint noise keys
    # Same expectation: the replicas estimate the same image.
    assert abs(a[:, :3].mean() - b[:, :3].mean()) < 0.2 * max(a[:, :3].mean(), 1e-6)


def test_rank_noise_keys_never_overlap():
    # A bench run renders (warmup + 2 * steps) * spp keys per rank; the
    # stride leaves room for far more.
    per_rank = (3 + 2 * 5) * 256 + 4096
    starts = [bench.rank_noise_seed(r) for r in range(8)]
    for i in range(8):
        for j in range(i + 1, 8):
            assert abs(starts[i] - starts[j]) >= per_rank
    assert bench.job_msamples_per_s(2, 1_000_000, 5, 1000.0) == 10.0
