"""Benchmark: body-ticks/s of the rigid-body tick at PGS residual <= 1e-4 (or the sweep cap) on one B200.

Workload (default ``--config terrain``): 100,000 bodies (40% spheres, 30% capsules, 30% boxes,
density 1000) falling onto a 512x512 heightfield (1 m spacing), dt 1/60, 20 iterations; each solve
island sweeps until its residual (largest |delta impulse| / effective mass over its rows in a
sweep, m/s) is <= 1e-4, or 80 sweeps (4x the iteration count). Seeded synthetic scene (no
dataset). A "step" is one tick of the whole world. The scene is first advanced ``--settle`` ticks
(untimed) so the timed ticks sit in the contact-rich part of the 600-tick run; then W warm-up
ticks, then exactly K timed ticks, bracketed by a barrier + device synchronize, timed with CUDA
events recorded on the world's own stream. ``--config box_drop`` is the 1,000-box drop
(8 iterations).

value   whole-job body-ticks/s (bodies x K summed over ranks / max over ranks of the timed span).
e2e     the same metric through the C ABI's rphys_world_step_ex with the tick's state read back to
        host memory (rphys_ext_get_body_states: pos, rot, lin, ang) every tick, timed on the host,
        over the same K ticks (replayed from a snapshot taken before the timed region).
roofline  the stage with the most device time in a profiled replay of the same K ticks (CUDA events
        around each stage on the world's stream): its algorithmic bytes per launch / its mean
        duration, against the measured HBM copy bandwidth in MEASURED_PEAKS.json.
cpu_baseline  the CPU restatement of the reference step (C++, OpenMP, all host threads or
        --cpu-threads) on the benchmark's own state: it loads the GPU world's state blob from the
        timed region's start and steps --cpu-ticks ticks of the full workload; ``one_thread``: the
        first of those ticks again on one thread.
parity  those ticks' hashes and the final body states, GPU against the CPU restatement.
solve   the last timed tick's velocity solve: sweeps, residual, islands still above the tolerance
        at the cap and their rows, and a histogram of the islands' last-sweep residuals.
batched (terrain) the 4,096-world batch stepped as one device world against the same worlds
        stepped one by one through their own RPhysWorld, and against the CPU restatement on every
        128th world (whose hashes must equal the batch's), plus the rollback window.

Multi-GPU: a single world does not shard (its contacts couple every body), so for the terrain and
box-drop workloads N ranks run N independent replicas (one per GPU, scaling "weak"). ``--config
batch`` splits one world table across the ranks (contiguous world ranges, riftphys-rust_b200/shards.py)
and gathers the per-world hashes once per rollback window; no collective touches the ticks.
``--impl reference`` times the CPU restatement alone on the same workload: the full scene settled
on the CPU, then the same warm-up and timed ticks (rank 0 only).
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))


def _import_pkg():
    import importlib.util
    pkg = os.path.join(ROOT, "riftphys-rust_b200")
    if "riftphys_rust_b200" in sys.modules:
        return sys.modules["riftphys_rust_b200"]
    spec = importlib.util.spec_from_file_location("riftphys_rust_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["riftphys_rust_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


rp = _import_pkg()
import riftphys_rust_b200.scenes as scenes  # noqa: E402
import riftphys_rust_b200.shards as shards  # noqa: E402
import riftphys_rust_b200.autotune as autotune  # noqa: E402

TOL = 1.0e-4
# algorithmic bytes per unit of each stage (counted once per required HBM read or write)
BYTES = {
    "forces": ("bodies", 24), "aabb_sweep": ("colliders", 92), "integrate": ("bodies", 152),
    "vel_solve": ("row_sweeps", 280), "pos_iter": ("pos_row_sweeps", 152), "narrow_pairs": ("pairs", 88 + 4 * 28),
    "stage6": ("bodies", 120),
}


ITERS = {"terrain": 20, "box_drop": 8, "batch": 16, "ragdolls": 24}
# DRAM bytes the velocity-solve kernels read and write per scheduled row and tick, from an ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum over the vel_solve kernels of 2 timed ticks of the
# terrain workload at 20,000 bodies: 48.8 MB over 175,676 rows; profiles/vel_solve_dram_terrain20k.md):
# the one-time staging of rows and bodies into shared memory, which grows with the rows
TRAFFIC_PER_ROW = {"vel_solve": 278.0}


def build_scene(lib, config, n_bodies=None, area=None, hf_n=None, worlds=4096, rank=0, world_size=1):
    if config == "batch":
        # one world table from one seed; this rank steps its contiguous range of it (no exchange
        # during the ticks; the hashes are gathered at the rollback window's end)
        lo, hi = shards.world_range(rank, world_size, worlds)
        descs = [scenes.batch_world_descs(rp, k, seed=3) for k in range(lo, hi)]
        total = sum(len(d) for d in descs)
        w = lib.world(total + 16, total + 16)
        dt = scenes.batch_setup(w)
        for d in descs:
            w.add_world(d)
        return w, dt, total, (f"batch: {worlds} independent worlds stepped together (worlds {lo}-{hi - 1} on this "
                              f"rank, {total:,} bodies), body counts log-uniform in [16, 4096], alternately square box "
                              "pyramids and random box piles (half-extents U[0.25, 0.75] m, 1000 kg/m^3) on 50x0.5x50 "
                              "ground boxes, dt 1/60, 16 iters")
    if config == "ragdolls":
        # worlds of 5 ragdolls each (15 capsules, 14 ball / hinge joints with limits), all on the same
        # 128^2 heightfield; the worlds' joints added in world order in one call
        import numpy as np
        per = 5
        h, origin = scenes.heightfield(128, 1.0, 5)
        parts = [scenes.ragdoll_arrays(rp, per, 1000 * (rank + 1) + k, 0.8 * 127, base_id=1,
                                       y0=float(h.max()) + 1.0) for k in range(worlds)]
        total = sum(len(b) for b, _, _ in parts)
        w = lib.world(total + 16, total + 16)
        w.set_heightfield(h, 128, 128, 1.0, 1.0, origin, origin, material=4)
        w.set_pair_props(0, 0, 0.6, 0.5, 0.0, 0.08)
        w.set_pair_props(0, 4, 0.883176, 0.724569, 0.0, 0.1)
        w.set_iterations(24, 24)
        jds, lds, nj = [], [], 0
        for bd, jd, ld in parts:
            _, first = w.add_world(bd)
            jd[:, 2:4].view(np.uint32)[:] += first - 1
            ld[:, 0].view(np.uint32)[:] += nj
            nj += len(jd)
            jds.append(jd); lds.append(ld)
        w.add_joint_array(np.concatenate(jds))
        w.set_joint_limit_array(np.concatenate(lds))
        return w, 1.0 / 120.0, total, (f"ragdolls: {worlds} independent worlds of {per} ragdolls ({total:,} capsule "
                                       f"bodies, {nj:,} joints: balls with +-45 deg swing limits, hinges limited to "
                                       "[-120, 0] deg; capsule r U[0.05, 0.12] m, segment U[0.2, 0.5] m, 1-8 kg) on one "
                                       "128^2 heightfield, dt 1/120, 24 iters")
    if config == "box_drop":
        side = max(1, round((n_bodies or 1000) ** (1.0 / 3.0)))
        w = lib.world(side ** 3 + 24, side ** 3 + 24)
        dt, n = scenes.box_drop(rp, w, n_side=side)
        return w, dt, n, (f"box_drop: {side ** 3:,} boxes (he 0.5 m, 1 kg) on a static 50x0.5x50 ground box, dt 1/60, "
                          "8+8 iters")
    n_bodies = n_bodies or 100_000
    w = lib.world(n_bodies + 16, n_bodies + 16)
    dt, n = scenes.terrain(rp, w, n_bodies=n_bodies, hf_n=hf_n or 512, area=area or 400.0)
    return w, dt, n, (f"terrain: {n} bodies (40% spheres, 30% capsules, 30% boxes, 1000 kg/m^3) starting in a "
                      f"{area or 400.0:g} m square over a {hf_n or 512}^2 heightfield at 1 m spacing, dt 1/60, 20 iters")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = "clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index, self.samples, self.proc = index, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 6:
                self.samples.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=2)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit())
        mx = max(float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[2 + k].strip() == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons}


def peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def job_throughput(local_units, local_ms, dist=None, device="cpu"):
    """Whole-job throughput over the ranks: units summed over ranks (each rank steps its own worlds
    or replica) over the slowest rank's device time. Returns (units per second, max ms, total units).
    Every rank makes the same two collective calls."""
    import torch
    units = torch.tensor([float(local_units)], dtype=torch.float64, device=device)
    ms = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(units, op=dist.ReduceOp.SUM)
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    total, ms_max = float(units.item()), float(ms.item())
    return total / (ms_max / 1000.0), ms_max, total


def peak_bf16():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def run_model(args, lib, torch):
    """The learned warm start's MLP alone: predictions for --rows device-resident rows per step
    (the inference a tick runs for its contact rows), timed on the device; tensor roofline."""
    rows = args.rows
    m = lib.model(seed=2)
    g = torch.Generator(device="cuda").manual_seed(1)
    feats = torch.randn(rows, 24, device="cuda", generator=g, dtype=torch.float32)
    out = torch.empty(rows, 3, device="cuda", dtype=torch.float32)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        m.predict_device(feats.data_ptr(), rows, out.data_ptr(), stream.cuda_stream)
    launches0 = lib.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        m.predict_device(feats.data_ptr(), rows, out.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    padded = (rows + 127) // 128 * 128
    flops = 2.0 * padded * (32 * 128 + 2 * 128 * 128 + 128 * 16)  # the padded products the GEMMs run
    peak, kind = peak_bf16()
    achieved = flops / (ms / 1000.0) / 1e12
    line = {"metric": "warm-start model rows/s", "value": rows / (ms / 1000.0), "unit": "rows/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": f"MLP 24-128-128-128-3 (SiLU) forward on {rows:,} rows, bf16 x bf16 -> f32 on tcgen05"},
            "roofline": {"kernel": "k_tc_gemm (4 products + activations)", "bound": "tensor", "unit": "TFLOP/s",
                         "achieved": achieved, "peak": peak, "peak_source": kind, "frac": achieved / peak,
                         "traffic": None, "flops_per_step": flops},
            "gpu_launches": lib.launch_count() - launches0}
    print(json.dumps(line), flush=True)


def oracle_path():
    p = os.path.join(ROOT, "oracle", "build", "liboracle_rphys.so")
    if not os.path.exists(p):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    return p


def oracle_world(lib, args, threads):
    """The CPU restatement's world of the benchmark scene (terrain or box drop), all threads."""
    w, dt, nb, desc = build_scene(lib, args.config, n_bodies=args.bodies, area=args.area)
    if args.mode == "residual":
        w.set_residual_mode(TOL, 4 * ITERS[args.config])
    lib.dll.rphys_oracle_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.dll.rphys_oracle_set_threads(w.h, threads)
    return w, dt, nb, desc


def run_reference(args):
    """--impl reference: the CPU restatement of the reference step (the reference itself is Rust and
    cannot be built here) on the same workload as our arm: the full scene, settled on the CPU, then
    W warm-up and K timed ticks, all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    if args.config not in ("terrain", "box_drop"):
        print(json.dumps({"impl": "reference", "unavailable": f"--impl reference covers the terrain and box_drop "
                                                             f"workloads, not {args.config}"}), flush=True)
        return
    args.mode = args.mode or "residual"
    lib = rp.Lib(oracle_path())
    threads = args.cpu_threads or os.cpu_count() or 1
    w, dt, nb, desc = oracle_world(lib, args, threads)
    t0 = time.perf_counter()
    w.step_n(dt, args.settle + args.warmup)
    t_settle = time.perf_counter() - t0
    t0 = time.perf_counter()
    w.step_n(dt, args.steps)
    el = time.perf_counter() - t0
    value = nb * args.steps / el
    sample = (f"the whole workload: ticks {args.settle + args.warmup + 1}-{args.settle + args.warmup + args.steps} "
              f"after {args.settle + args.warmup} settle and warm-up ticks on the CPU ({t_settle:.0f} s), "
              f"{threads} threads, islands solved in parallel")
    print(json.dumps({"impl": "reference", "metric": metric_name(args.config), "value": value, "unit": "body-ticks/s",
                      "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": el * 1000.0 / args.steps, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                      "config": run_config(args, desc, world_size),
                      "cpu_baseline": {"value": value, "unit": "body-ticks/s", "cores": threads, "kind": "port",
                                       "sample": sample},
                      "e2e": {"value": value, "unit": "body-ticks/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)


def cpu_sample_from_state(olib, args, blob, gpu_world, dt, ticks, threads):
    """The CPU baseline on the benchmark's own state: a CPU-restatement world of the same scene loads
    the GPU world's state blob taken at the timed region's start and steps `ticks` ticks (timed);
    the GPU world, restored to the same snapshot by the caller, steps the same ticks. Returns the
    CPU throughput, the sample's description and whether every tick's hash and the final body
    states agreed."""
    import numpy as np
    w, _, nb, _ = oracle_world(olib, args, threads)
    w.state_import(blob)
    same = w.hash() == gpu_world.hash()
    hs = []
    el = 0.0
    for _ in range(ticks):
        t0 = time.perf_counter()
        w.step_n(dt, 1)
        el += time.perf_counter() - t0
        hs.append(w.hash())
    for k in range(ticks):
        gpu_world.step_n(dt, 1)
        same = same and gpu_world.hash() == hs[k]
    same = same and np.array_equal(w.body_states().view(np.uint32), gpu_world.body_states().view(np.uint32))
    first = args.settle + args.warmup + 1
    sample = (f"the benchmark's own {nb}-body state at its timed region's start (loaded from the GPU world's state "
              f"blob), ticks {first}-{first + ticks - 1}, {threads} threads, islands solved in parallel")
    w.close()
    return nb * ticks / el, sample, same


def batched_record(lib, torch, n_worlds, settle=30, ticks=10, every=32, cpu_every=128, cpu_threads=1):
    """The batched-worlds workload (n_worlds worlds of 16-4096 boxes, residual <= 1e-4 or 64 sweeps)
    stepped as one device batch, against the plain path -- each world its own RPhysWorld stepped by
    its own calls, as the reference steps one World per call -- on every `every`-th world (the worlds'
    sizes are independent draws, so the sample has the table's size distribution). Both from tick 0:
    `settle` ticks untimed, then `ticks` timed; the batch on the device clock, the plain worlds on the
    host clock around each world's completed ticks (its launches and waits are its cost). Plus the
    8-tick rollback window of the batch: restore, re-simulate, every world's hash compared. Plus the
    CPU restatement on every `cpu_every`-th world, stepped the same ticks (host-timed over the timed
    ticks) with each world's final hash compared with the batch's hash of that world."""
    tol, cap = TOL, 4 * ITERS["batch"]
    descs = [scenes.batch_world_descs(rp, k, seed=3) for k in range(n_worlds)]
    total = sum(len(d) for d in descs)
    b = lib.world(total + 16, total + 16)
    dt = scenes.batch_setup(b)
    for d in descs:
        b.add_world(d)
    b.set_residual_mode(tol, cap)
    b.step_n(dt, settle)
    snap = b.snapshot()
    stream = torch.cuda.ExternalStream(b.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    b.step_n(dt, ticks)
    e1.record(stream)
    torch.cuda.synchronize()
    bms = e0.elapsed_time(e1)
    sb = b.stats()
    t0 = time.perf_counter()
    h_first = b.world_hashes()
    hash_ms = (time.perf_counter() - t0) * 1000.0
    b.restore_exact(snap)
    b.step_n(dt, ticks)
    rollback_ok = b.world_hashes() == h_first
    b.free_snapshot(snap)
    b.close()
    plain_s, plain_bodies, sample = 0.0, 0, list(range(0, n_worlds, every))
    for k in sample:
        d = descs[k]
        w = lib.world(len(d), len(d))
        scenes.batch_setup(w)
        w.add_bodies_array(d)
        w.set_residual_mode(tol, cap)
        w.step_n(dt, settle)
        t0 = time.perf_counter()
        w.step_n(dt, ticks)
        plain_s += time.perf_counter() - t0
        plain_bodies += len(d)
        w.close()
    cpu_s, cpu_bodies, cpu_same, cpu_sample = 0.0, 0, True, list(range(0, n_worlds, cpu_every))
    olib = rp.Lib(oracle_path())
    olib.dll.rphys_oracle_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
    for k in cpu_sample:
        d = descs[k]
        o = olib.world(len(d), len(d))
        scenes.batch_setup(o)
        o.add_bodies_array(d)
        o.set_residual_mode(tol, cap)
        olib.dll.rphys_oracle_set_threads(o.h, cpu_threads)
        o.step_n(dt, settle)
        t0 = time.perf_counter()
        o.step_n(dt, ticks)
        cpu_s += time.perf_counter() - t0
        cpu_bodies += len(d)
        cpu_same = cpu_same and o.hash() == h_first[k]
        o.close()
    batched_v = total * ticks / (bms / 1000.0)
    plain_v = plain_bodies * ticks / plain_s
    return {"workload": f"{n_worlds} worlds, {total:,} boxes, ticks {settle + 1}-{settle + ticks} from rest, residual "
                        f"<=1e-4 or {cap} sweeps per island, previous-tick warm start",
            "batched": {"value": batched_v, "unit": "body-ticks/s", "ms_per_tick": bms / ticks,
                        "levels_last_tick": sb["levels"], "sweeps_last_tick": sb["sweeps"],
                        "islands_capped_last_tick": sb["islands_capped"]},
            "plain": {"value": plain_v, "unit": "body-ticks/s", "worlds": len(sample), "bodies": plain_bodies,
                      "s_per_tick_all_sampled_worlds": plain_s / ticks,
                      "note": "one RPhysWorld per world stepped through rphys_ext_step_n, host-timed"},
            "batched_over_plain": batched_v / plain_v,
            "cpu": {"value": cpu_bodies * ticks / cpu_s, "unit": "body-ticks/s", "cores": cpu_threads, "kind": "port",
                    "worlds": len(cpu_sample), "bodies": cpu_bodies, "hashes_match_batch": cpu_same,
                    "note": f"the CPU restatement stepping every {cpu_every}th world alone, host-timed over the "
                            f"timed ticks; each world's hash after them compared with the batch's"},
            "rollback_window": {"ticks": ticks, "hashes_match": rollback_ok,
                                "all_world_hashes_ms": hash_ms,
                                "note": "every world's tick hash in one rphys_ext_batch_get_hashes call (kernels over the "
                                        "world table), host-timed"}}


def metric_name(config):
    """The headline metric: throughput with every solve island sweeping until its residual is
    <= 1e-4 m/s or the sweep cap (4x the configuration's iteration count) stops it."""
    return f"body-ticks/s at PGS residual <=1e-4 or {4 * ITERS[config]} sweeps per island"


def run_config(args, desc, world_size):
    """The workload's configuration, identical in both arms' lines (measured values live elsewhere)."""
    return {"workload": desc, "settle_ticks": args.settle, "warmup_ticks": args.warmup, "mode": args.mode,
            "tolerance": TOL if args.mode == "residual" else None,
            "max_sweeps": 4 * ITERS[args.config] if args.mode == "residual" else ITERS[args.config],
            "parallelism": f"replicas{world_size}", "l2": "inputs larger than L2 (126 MB)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--settle", type=int, default=240)
    ap.add_argument("--config", default="terrain", choices=["terrain", "box_drop", "batch", "ragdolls", "model"])
    ap.add_argument("--rows", type=int, default=1 << 20, help="model: rows per step")
    ap.add_argument("--worlds", type=int, default=None, help="batch / ragdolls: number of worlds (4096 / 2000)")
    ap.add_argument("--learned", type=int, default=1, help="terrain: also time the learned warm start (1/0)")
    ap.add_argument("--mode", default=None, choices=["residual", "fixed"],
                    help="velocity-solve stop: residual <= 1e-4 (default), or the reference's fixed iteration count "
                         "(default for ragdolls, whose articulations stay above 1e-4 for most islands)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--bodies", type=int, default=None)
    ap.add_argument("--area", type=float, default=None,
                    help="terrain: side of the square the bodies start in (default 400 m; the workload's density "
                         "for n bodies is 400 * sqrt(n / 100000))")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-ticks", type=int, default=3, help="ticks of the CPU sample (and of the parity check)")
    ap.add_argument("--cpu-threads", type=int, default=0, help="threads of the CPU restatement (0: all host threads)")
    ap.add_argument("--coloured", type=int, default=1, help="also replay the timed ticks in coloured order (1/0)")
    ap.add_argument("--autotune", type=int, default=0, help="time every velocity-solve launch shape first (1/0)")
    ap.add_argument("--batched", type=int, default=1,
                    help="terrain: also measure the batched-worlds workload against stepping its worlds one by one")
    ap.add_argument("--batched-worlds", type=int, default=4096)
    ap.add_argument("--tuning-out", default=autotune.TABLE, help="where --autotune records its table")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world_size > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    lib = rp.load_product()
    if args.config == "model":
        return run_model(args, lib, torch)
    worlds = args.worlds or (2000 if args.config == "ragdolls" else 4096)
    w, dt, nb, desc = build_scene(lib, args.config, n_bodies=args.bodies, area=args.area, worlds=worlds, rank=rank,
                                  world_size=world_size)
    args.mode = args.mode or ("fixed" if args.config == "ragdolls" else "residual")
    if args.mode == "residual":
        w.set_residual_mode(TOL, 4 * ITERS[args.config])
    # settle into the contact regime, then warm up
    t_settle = time.perf_counter()
    learn_f, learn_t = [], []
    learned_on = args.learned and args.config == "terrain"
    if args.settle:
        if learned_on and args.settle > 60:
            # the learned warm start's training rows: every row of every 3rd of the last 60 settle
            # ticks (about 8M rows of this workload), with the impulses the plain solver converged to
            w.step_n(dt, args.settle - 60)
            w.set_feature_logging(True)
            for k in range(60):
                w.step_n(dt, 1)
                if k % 3 == 2:
                    f, t = w.row_features()
                    learn_f.append(f); learn_t.append(t)
            w.set_feature_logging(False)
        else:
            w.step_n(dt, args.settle)
    print(f"[bench] {nb} bodies, settle {args.settle} ticks in {time.perf_counter() - t_settle:.2f}s", file=sys.stderr)
    for _ in range(args.warmup):
        w.step_n(dt, 1)
    stream = torch.cuda.ExternalStream(w.stream_handle())
    # the e2e and profiled passes replay exactly the timed ticks from this snapshot (the restore is
    # bit-exact, so all three passes see the same contacts, islands and sweeps)
    snap = w.snapshot()
    tuning_note = None
    if args.autotune:
        # time every launch shape on this state (same bits for all), record the table, keep the best
        best, rows = autotune.tune(w, dt, snap, 5, torch, stream)
        autotune.record(args.tuning_out, args.config, best, rows,
                        f"{desc}; 5 ticks from the state after {args.settle + args.warmup} ticks, per shape")
        tuning_note = "autotuned in this run"
        print(f"[bench] autotune: best {best}; all same bits: {all(r['same_bits'] for r in rows)}", file=sys.stderr)
        w.restore_exact(snap)  # the tuner stepped on from the snapshot: back to it
    else:
        tuning_note = "recorded table" if autotune.apply(w, args.config) else "compiled defaults"
    # the same state as a host blob, for the CPU restatement's sample of the same ticks
    blob = w.state_export() if args.config in ("terrain", "box_drop") else None
    launches0 = lib.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    torch.cuda.nvtx.range_push("timed")  # lets a profiler select exactly the timed ticks
    e0.record(stream)
    w.step_n(dt, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    clk = clocks.stop()
    launches = lib.launch_count() - launches0
    if world_size > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    st = w.stats()
    value, ms_max, _ = job_throughput(nb * args.steps, ms, dist, "cuda")

    # e2e: the drop-in C-ABI call with the tick's state read back to host memory every tick
    import numpy as np
    host = torch.empty((nb, 13), dtype=torch.float32, pin_memory=True)  # page-locked: the fast D2H path
    e2e_ticks = args.steps
    w.restore_exact(snap)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_ticks):
        w.step(dt)
        w.c("rphys_ext_get_body_states", 0, nb, ctypes.c_void_p(host.data_ptr()))
    e2e_s = time.perf_counter() - t0
    e2e = {"value": nb * e2e_ticks / e2e_s, "unit": "body-ticks/s", "h2d_bytes_per_step": 20,
           "d2h_bytes_per_step": 52 * nb,
           "note": "each tick one rphys_world_step_ex call whose input is its 20-byte RPhysStepParams (the world "
                   "state lives in the library between calls, as behind the reference's FFI), then "
                   "rphys_ext_get_body_states reads every body's pos, rot, lin, ang (52 B) back into pinned host "
                   "memory"}

    # roofline: the stage with the most device time, in a separate profiled pass
    w.restore(snap)
    w.profile(True)
    units = {"bodies": 0, "colliders": 0, "row_sweeps": 0, "pos_row_sweeps": 0, "pairs": 0}
    for _ in range(args.steps):
        w.step_n(dt, 1)
        s = w.stats()
        units["bodies"] += nb
        units["colliders"] += nb
        units["row_sweeps"] += s["row_sweeps"]
        units["pos_row_sweeps"] += s["rows_scheduled"] * ITERS[args.config]
        units["pairs"] += s["pairs"]
    prof = w.profile_read()
    w.profile(False)
    for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0]):
        print(f"[bench] stage {k:14s} {v[0] / max(1, v[1]):9.4f} ms/tick", file=sys.stderr)
    outer = {k: v for k, v in prof.items() if "." not in k}  # "a.b" phases are nested inside "a"
    total_ms = sum(v[0] for v in outer.values())
    top = max(outer.items(), key=lambda kv: kv[1][0])
    peak, peak_kind = peak_hbm()
    stage, (stage_ms, stage_calls) = top
    roof = {"kernel": stage, "bound": "hbm", "unit": "GB/s", "peak": peak, "peak_source": peak_kind,
            "traffic": None, "share_of_tick": stage_ms / total_ms if total_ms else None}
    if stage in BYTES and stage_calls:
        unit, per = BYTES[stage]
        bytes_per_launch = per * units[unit] / stage_calls
        achieved = bytes_per_launch / (stage_ms / stage_calls / 1000.0) / 1e9
        roof.update({"achieved": achieved, "frac": achieved / peak, "bytes_per_launch": bytes_per_launch,
                     "ms_per_launch": stage_ms / stage_calls})
    if stage in TRAFFIC_PER_ROW and stage_calls:
        roof["traffic"] = TRAFFIC_PER_ROW[stage] * (units["pos_row_sweeps"] / ITERS[args.config]) / stage_calls
        roof["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the vel_solve kernels at 20,000 "
                                  "bodies, scaled by this run's rows (profiles/vel_solve_dram_terrain20k.md)")
    if stage == "vel_solve" and stage_calls:
        # the bound that holds: the serial chain of the deepest island, sweeps x its levels dependent
        # row updates (a level step: one row update plus a block barrier)
        chain = st["sweeps"] * st["levels"]
        roof["latency"] = {"level_steps_last_tick": chain, "ms_per_launch": stage_ms / stage_calls,
                           "ns_per_level_step": stage_ms / stage_calls * 1e6 / chain if chain else None,
                           "note": "vel_solve time over the deepest island's chain (sweeps x levels of the last "
                                   "timed tick); the kernel is latency-bound, not HBM-bound"}
    else:
        roof.update({"achieved": None, "frac": None, "ms_per_launch": stage_ms / max(1, stage_calls)})
    stages = {k: round(v[0] / max(1, v[1]), 4) for k, v in prof.items() if v[1]}

    cpu, parity = None, None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline and blob is not None:
        # the CPU restatement on the benchmark's own state: timed (cpu_baseline), and every tick's
        # hash and the final body state compared with the GPU's replay of the same ticks (parity)
        olib = rp.Lib(oracle_path())
        threads = args.cpu_threads or os.cpu_count() or 1
        w.restore_exact(snap)
        v, sample, same = cpu_sample_from_state(olib, args, blob, w, dt, args.cpu_ticks, threads)
        cpu = {"value": v, "unit": "body-ticks/s", "cores": threads, "kind": "port", "sample": sample}
        if threads > 1:
            # the first of those ticks again on one thread (the reference's single-core figure)
            w.restore_exact(snap)
            v1, _, same1 = cpu_sample_from_state(olib, args, blob, w, dt, 1, 1)
            cpu["one_thread"] = {"value": v1, "ticks": 1, "same_bits": bool(same1)}
        parity = {"bit_exact": bool(same), "ticks": args.cpu_ticks,
                  "checked": "tick hash every tick and all body states after the last, GPU vs CPU restatement "
                             "from the same state"}

    coloured = None
    if args.config in ("terrain", "box_drop", "batch") and args.coloured:
        # the same timed ticks replayed in coloured order (rphys_ext_set_solve_order): steps per sweep,
        # device time, and the first tick's divergence from the serial order's (same state)
        import numpy as np
        w.restore_exact(snap)
        w.step_n(dt, 1)
        ser1 = w.body_states()
        w.restore_exact(snap)
        w.set_coloured(True)
        w.step_n(dt, 1)
        col1 = w.body_states()
        w.restore_exact(snap)
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        c0.record(stream)
        w.step_n(dt, args.steps)
        c1.record(stream)
        torch.cuda.synchronize()
        cms = c0.elapsed_time(c1)
        cs = w.stats()
        w.set_coloured(False)

        def rel(a, b):
            return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
        coloured = {"value": nb * args.steps / (cms / 1000.0), "unit": "body-ticks/s", "ms_per_step": cms / args.steps,
                    "levels_last_tick": cs["levels"], "levels_last_tick_serial": st["levels"],
                    "sweeps_last_tick": cs["sweeps"], "row_sweeps_last_tick": cs["row_sweeps"],
                    "islands_capped_last_tick": cs["islands_capped"],
                    "first_tick_rel_divergence": {"pos": rel(col1[:, 0:3], ser1[:, 0:3]),
                                                  "lin": rel(col1[:, 7:10], ser1[:, 7:10]),
                                                  "ang": rel(col1[:, 10:13], ser1[:, 10:13])},
                    "note": "same timed ticks replayed from the snapshot in coloured order; divergence: relative L2 "
                            "difference of one tick from the same state, coloured vs serial"}

    learned = None
    if learned_on and learn_f:
        # train on the settle rows (targets clipped to +-20 units: the rows of infeasible contact
        # sets carry impulses thousands of units large), then replay the timed ticks with the model
        # offering a start to every row (each row keeps the prediction only where it starts better
        # than the previous tick's impulse) and, separately, only to rows the cache has nothing for
        import numpy as np
        F, T = np.concatenate(learn_f), np.clip(np.concatenate(learn_t), -20.0, 20.0)
        del learn_f, learn_t
        model = lib.model(seed=2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        epochs = 2
        loss = model.train(F, T, epochs=epochs, batch=4096, lr=1e-3)
        t_train = time.perf_counter() - t0
        w.set_warm_model(model)
        runs = {}
        for policy, cold in (("all_rows", False), ("cold_rows", True)):
            w.set_warm_policy(cold)
            w.restore_exact(snap)
            l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            l0.record(stream)
            w.step_n(dt, args.steps)
            l1.record(stream)
            torch.cuda.synchronize()
            lms = l0.elapsed_time(l1)
            # the same ticks again, stats read after each (row updates, starts taken) and staged
            w.restore_exact(snap)
            w.profile(True)
            rs = pu = capped = 0
            for _ in range(args.steps):
                w.step_n(dt, 1)
                s_ = w.stats()
                rs += s_["row_sweeps"]; pu += s_["pred_used"]; capped += s_["rows_capped"]
            lprof = w.profile_read()
            w.profile(False)
            runs[policy] = {"value": nb * args.steps / (lms / 1000.0), "ms_per_step": lms / args.steps,
                            "row_updates": rs, "rows_in_capped_islands": capped,
                            "rows_started_from_prediction": pu,
                            "stage_ms": {k: round(v[0] / max(1, v[1]), 4) for k, v in lprof.items()
                                         if k in ("warm_match", "vel_solve")}}
        w.set_warm_model(None)
        learned = dict(runs["all_rows"], unit="body-ticks/s", policies=runs,
                       row_updates_previous_tick_start=units["row_sweeps"], train_rows=int(len(F)),
                       train_epochs=epochs, train_seconds=t_train, train_loss=loss,
                       note="same timed ticks replayed from the snapshot; value and ms from a replay with no host "
                            "reads, row counts from a second replay with stats read after each tick")

    rollback = None
    if args.config in ("batch", "ragdolls"):
        # the rollback workload: back to the snapshot, re-simulate 8 ticks twice from it (the first
        # pass and the replay), the replay timed on the device; every world's hash must match
        # (ragdoll worlds stay per rank; batch worlds are one table: its hashes gathered over ranks)
        w.restore_exact(snap)
        w.step_n(dt, 8)
        local_first = w.world_hashes()
        w.restore_exact(snap)
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        r0.record(stream)
        w.step_n(dt, 8)
        r1.record(stream)
        torch.cuda.synchronize()
        local_again = w.world_hashes()
        if args.config == "batch":
            h_first = shards.gather_world_hashes(local_first, worlds, dist, "cuda")
            h_again = shards.gather_world_hashes(local_again, worlds, dist, "cuda")
        else:
            h_first, h_again = local_first, local_again
        rollback = {"ticks": 8, "ms": r0.elapsed_time(r1), "worlds": len(h_first),
                    "hashes_match": h_first == h_again}

    # the riftnet wire snapshot of the final state (riftphys-riftnet/src/wire.rs): packed on the
    # device and copied to the host, as a server does every tick; host-timed over a few calls
    batched = None
    if args.config == "terrain" and args.batched and rank == 0 and world_size == 1:
        batched = batched_record(lib, torch, args.batched_worlds, cpu_threads=args.cpu_threads or os.cpu_count() or 1)

    wire = None
    if args.config == "terrain":
        import time as _time
        w.pack_snapshot(0, 0)
        t0 = _time.perf_counter()
        reps = 10
        for k in range(reps):
            data, chunks = w.pack_snapshot(k, 0)
        wire_ms = (_time.perf_counter() - t0) * 1000.0 / reps
        wire = {"bodies": nb, "chunks": chunks, "bytes": len(data), "ms": wire_ms,
                "gb_per_s": len(data) / (wire_ms * 1e-3) / 1e9, "note": "host-timed, device pack + copy to pageable memory"}
        # batched scene queries on the same state (queries.rs:18-116): 16,384 seeded rays down onto
        # the scene, AABB and exact, through the C ABI; host-timed, rays/s
        qrng = np.random.default_rng(5)
        nq = 16384
        qo = np.column_stack([qrng.uniform(-190, 190, nq), qrng.uniform(20, 70, nq), qrng.uniform(-190, 190, nq)])
        qd = np.column_stack([qrng.normal(size=nq) * 0.3, -np.ones(nq), qrng.normal(size=nq) * 0.3])
        qo, qd = qo.astype(np.float32), qd.astype(np.float32)
        rays = {}
        for name, exact in (("aabb", False), ("exact", True)):
            w.raycast_batch(qo, qd, 120.0, exact=exact)
            t0 = _time.perf_counter()
            for _ in range(3):
                hits = w.raycast_batch(qo, qd, 120.0, exact=exact)
            ms = (_time.perf_counter() - t0) * 1000.0 / 3
            rays[name] = {"rays": nq, "ms": ms, "rays_per_s": nq / (ms * 1e-3),
                          "hits": int(hits[:, 0].view(np.uint32).sum())}
        wire["ray_batch"] = dict(rays, note="host-timed through rphys_ext_raycast_batch / _exact_batch, "
                                             "one 256-thread block per ray over every collider")

    if rank == 0:
        rows, capped = st["rows_scheduled"], st["rows_capped"]
        solve = {"sweeps": st["sweeps"], "residual": st["residual"], "rows": rows, "contacts": st["contacts"],
                 "islands": st["islands"], "levels": st["levels"], "islands_capped": st["islands_capped"],
                 "rows_in_capped_islands": capped,
                 "rows_converged_frac": (rows - capped) / rows if rows else None,
                 "island_residual_hist": dict(zip(["<=1e-4", "<=1e-3", "<=1e-2", "<=1e-1", "<=1", ">1"],
                                                  st["res_hist"])),
                 "row_sweeps": st["row_sweeps"],
                 "solve_groups": {"shared_memory": st["groups_shared"], "global_memory": st["groups_global"],
                                  "max_rows": st["max_group_rows"], "max_bodies": st["max_group_bodies"]},
                 "note": "the last timed tick's velocity solve"}
        rows_total = units["pos_row_sweeps"] / ITERS[args.config]  # rows present, summed over the K ticks
        rates = {"constraint_rows_per_s": rows_total / (ms / 1000.0), "row_updates_per_s": units["row_sweeps"] / (ms / 1000.0),
                 "note": "rows present per tick and velocity row updates run, summed over the timed ticks (from the "
                         "profiled replay of the same ticks) over the timed span"}
        line = {"metric": metric_name(args.config), "value": value, "unit": "body-ticks/s", "n_gpus": world_size,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": run_config(args, desc, world_size), "solve": solve, "rates": rates, "parity": parity,
                "e2e": e2e, "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
                "gpu_launches": launches, "stage_ms": stages,
                "tuning": dict(w.tuning(), source=tuning_note)}
        if batched is not None:
            line["batched"] = batched
        if rollback is not None:
            line["rollback"] = rollback
        if learned is not None:
            line["learned_warm_start"] = learned
        if coloured is not None:
            line["coloured_order"] = coloured
        if wire is not None:
            line["wire_snapshot"] = wire
        print(json.dumps(line), flush=True)
    w.free_snapshot(snap)
    w.close()
    if world_size > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
