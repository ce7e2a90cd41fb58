"""The multi-GPU bench path on CPU: replicas with no data-path collective, timed as the slowest rank.

bench.py --gpus N runs one independent replica of the workload per rank (the runs of an ensemble are
independent); the only collective is the max over ranks of the timed milliseconds.  Here two gloo
ranks stand in for two GPUs.
"""
import os
import socket
from datetime import timedelta

import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        ms = 10.0 + 5.0 * rank                      # rank 1 is the slow one
        m = bench.max_over_ranks(ms, True, device="cpu")
        q.put((rank, m, bench.whole_job_rate(world, 576, 200, m)))
    finally:
        torch.distributed.destroy_process_group()


def test_replicas_are_timed_by_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [m for _, m, _ in out] == [15.0, 15.0]
    # whole-job value: both replicas' orbital-steps over the slowest replica's time
    assert out[0][2] == pytest.approx(2 * 576 * 200 / 0.015)


def test_single_rank_needs_no_collective():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, False) == 12.5
    assert bench.whole_job_rate(1, 576, 200, 12.5) == pytest.approx(576 * 200 / 0.0125)
