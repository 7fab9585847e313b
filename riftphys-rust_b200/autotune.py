"""Autotuner of the velocity solve's launch shapes (rphys_ext_set_tuning): the rows up to which
islands are packed into shared solve groups, and the threads of a packed group's block and of a
single island's block. It times every combination on a world's own state -- restored from one
snapshot, a few ticks each, CUDA events on the world's stream -- checks that every combination
gives the same tick hash (launch shapes change no result bit), and records the table in
tuning.json beside this file, keyed by workload. The library's compiled defaults are the terrain
workload's entry."""
import itertools
import json
import os

GRID = {"group_rows": (8, 16, 32, 64, 128), "packed_threads": (32, 64, 128), "island_threads": (32, 64, 128, 256)}
TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")


def tune(world, dt, snap, ticks, torch, stream):
    """Times every launch shape over `ticks` ticks from snapshot `snap`; leaves the fastest set.
    Returns (best, rows) with one row per shape: its ms per tick and whether its hash matched."""
    rows, ref = [], None
    for gr, pt, it in itertools.product(GRID["group_rows"], GRID["packed_threads"], GRID["island_threads"]):
        world.set_tuning(gr, pt, it)
        world.restore_exact(snap)
        world.step_n(dt, 1)                      # first use of a shape: attributes, scratch growth
        world.restore_exact(snap)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        world.step_n(dt, ticks)
        e1.record(stream)
        torch.cuda.synchronize()
        h = world.hash()
        ref = h if ref is None else ref
        rows.append({"group_rows": gr, "packed_threads": pt, "island_threads": it,
                     "ms_per_tick": e0.elapsed_time(e1) / ticks, "same_bits": h == ref})
    best = min(rows, key=lambda r: r["ms_per_tick"])
    world.set_tuning(best["group_rows"], best["packed_threads"], best["island_threads"])
    return best, rows


def record(path, workload, best, rows, note):
    """Writes the workload's entry (the best shape, every timed shape) into the JSON table."""
    table = load(path)
    table[workload] = {"best": {k: best[k] for k in GRID}, "ms_per_tick": best["ms_per_tick"], "timed": rows,
                       "note": note}
    with open(path, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)


def load(path=TABLE):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def apply(world, workload, path=TABLE):
    """Sets the recorded best shape for `workload` on `world`; returns it (None without an entry)."""
    e = load(path).get(workload)
    if not e:
        return None
    b = e["best"]
    world.set_tuning(b["group_rows"], b["packed_threads"], b["island_threads"])
    return b
