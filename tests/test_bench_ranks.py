"""bench.py's multi-rank arithmetic on two gloo ranks (CPU): units summed over ranks, time the
slowest rank's, every rank getting the same answer -- the replicas / sharded-worlds path that
`torchrun --nproc-per-node N bench.py` takes on N GPUs."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    units = 1000 * (rank + 1)           # ranks step different amounts of work (batched worlds)
    ms = 100.0 + 50.0 * rank             # and take different times
    out[rank] = bench.job_throughput(units, ms, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_agree_and_reduce():
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    v0, v1 = out[0], out[1]
    assert v0 == v1
    value, ms_max, total = v0
    assert total == 3000.0 and ms_max == 150.0
    assert value == pytest.approx(3000.0 / 0.150)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    value, ms_max, total = bench.job_throughput(500, 250.0)
    assert (total, ms_max) == (500.0, 250.0) and value == pytest.approx(2000.0)
