"""The replica path of bench.py on CPU: two ranks over gloo.

The solve does not shard, so `bench.py --gpus N` runs one independent solve per GPU and reports
the whole job: the slowest rank's device time and the sum of every rank's voxel-iterations
(bench.aggregate_replicas).  Two processes on the gloo backend check that reduction, and that
`--impl reference` leaves ranks other than 0 without work.
"""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    secs, vi = bench.aggregate_replicas(dist, 1.5 + rank, 1000.0 * (rank + 1), "cpu")
    ref_rc = bench.run_reference(type("A", (), {"n": 8})(), world, rank) if rank != 0 else None
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, secs, vi, ref_rc))


@pytest.mark.timeout(180)
def test_two_replicas_aggregate_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=150) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, secs, vi, ref_rc in res:
        assert secs == 2.5 and vi == 3000.0  # max of 1.5, 2.5 s; 1000 + 2000 voxel-iters
    assert res[1][3] == 0  # rank 1 of the reference arm: no work, exit 0


def test_single_process_is_its_own_job():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.aggregate_replicas(None, 2.0, 7.0, "cpu") == (2.0, 7.0)
