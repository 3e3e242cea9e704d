"""The multi-GPU path of bench.py (replicas, one process per GPU) on two CPU processes over gloo.

Each rank plays a replica with its own device times and work; the job's figures must be the
units of all ranks over the slowest rank's time, on every rank, and the reference arm must run on
rank 0 only.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, queue):
    import datetime
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import numpy as np
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        # Replica figures: rank r solved 10 + r LM iterations in (2 + r) seconds of device time.
        reports = [{"solve_ms": 1000.0 * (2 + rank), "lm_iterations": 10 + rank, "cg_iterations": 100 * (rank + 1),
                    "refinements": 0}]

        class Scene:
            C, P = 2, 3

        out = np.zeros(12 * 2 + 3 * 3 + 27)
        out[12 * 2 + 3 * 3 + 6] = 5.0 + rank
        summary = bench.form_summary(world, Scene, reports, [3.0 + rank], out)
        maxed = bench.max_over_ranks(world, float(rank))
        summed = bench.sum_over_ranks(world, float(rank + 1))
        # The reference arm: only rank 0 runs and prints.
        class Args:
            config, scale, warmup, steps, gpus = "invdepth", 0.0001, 0, 1, world

        import contextlib
        import io
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            bench.run_reference(Args, world, rank)
        queue.put((rank, summary["value"], summary["e2e"], summary["t_max"], maxed, summed, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_replica_figures_over_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    for rank, value, e2e, t_max, maxed, summed, printed in results:
        # 21 LM iterations over both ranks, over the slower rank's 3 s (device) and 4 s (wall).
        assert value == pytest.approx(21 / 3.0) and e2e == pytest.approx(21 / 4.0) and t_max == 3.0
        assert maxed == 1.0 and summed == 3.0
        assert (printed.strip() != "") == (rank == 0)
    assert '"impl": "reference"' in results[0][6]
