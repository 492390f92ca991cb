"""Multi-GPU runs are replicas: one independent scene per rank, no exchange
in the data path; the only collectives are the barrier and the max over ranks
of the device time.  These host-side rules run here on CPU ranks over gloo
(world size 2), exactly as bench.py uses them over NCCL."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
        ms = bench.reduce_max(dist, local_ms, device="cpu")
        dist.barrier()
        q.put((rank, ms, bench.replica_value(world, 64 ** 3, 10, ms)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    # every rank sees the slowest rank's time, and the whole-job value counts
    # both replicas' cells over that time
    for rank, ms, val in got:
        assert ms == 150.0
        assert val == pytest.approx(2 * 64 ** 3 * 10 / 0.150 / 1e6)


def test_single_rank_is_identity():
    assert bench.reduce_max(None, 3.5) == 3.5
    assert bench.replica_value(1, 1000, 10, 10.0) == pytest.approx(1.0)
