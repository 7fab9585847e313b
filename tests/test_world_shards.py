"""The batched-worlds table split across ranks (riftphys-rust_b200/shards.py) on two gloo ranks (CPU):
each rank steps its contiguous range of one table -- every world a CPU-restatement World, as each
world of a device batch steps bit for bit like it alone -- and the per-world hashes gathered once at
the window's end equal one process stepping the whole table."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N_WORLDS, TICKS = 9, 20


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _step_worlds(lo, hi):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import oracle_lib, rp, scenes
    lib = oracle_lib()
    hashes = []
    for k in range(lo, hi):
        d = scenes.batch_world_descs(rp, k, n_min=16, n_max=64)
        w = lib.world(len(d), len(d))
        dt = scenes.batch_setup(w)
        w.add_bodies_array(d)
        w.step_n(dt, TICKS)
        hashes.append(w.hash())
        w.close()
    return hashes


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import rp  # noqa: F401  (imports the package and its submodules)
    import riftphys_rust_b200.shards as shards
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    lo, hi = shards.world_range(rank, world, N_WORLDS)
    out[rank] = shards.gather_world_hashes(_step_worlds(lo, hi), N_WORLDS, dist)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gather_the_single_rank_hashes():
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    whole = _step_worlds(0, N_WORLDS)
    assert out[0] == out[1] == whole
    assert len(set(whole)) == N_WORLDS


def test_world_ranges_cover_the_table():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import rp  # noqa: F401
    import riftphys_rust_b200.shards as shards
    for n in (1, 7, 4096):
        for ws in (1, 2, 3, 8):
            rs = [shards.world_range(r, ws, n) for r in range(ws)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(rs[i][1] == rs[i + 1][0] for i in range(ws - 1))
