#!/usr/bin/env python
"""Benchmark of MARL's per-tick field-and-cell path on B200.

Workload: the reference default run — 128x128x64 grid, 12 external species,
Winogradsky boundary priming, 3 x 30 seeded starter cells, host RNG seed 42,
10 diffusion substeps per tick, f32.  One step = one tick of marl_sim::run's
loop: boundary sources, diffusion, light, the sequential cell loop (device),
then the change list to the host, fate/division/mutation on the host, and the
edit list back.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --case {diffusion,cells,light,mlp,engine} [...]   (one kernel, for ncu)

Printed (rank 0, one JSON line):
  value       ticks/s with all state resident in HBM: K ticks / summed device
              time of the ticks (CUDA events on the engine's stream around the
              tick kernels + change-list copy and around the edit copy +
              kernels); the host fate step between them is excluded here.
  e2e         ticks/s through the public C-ABI engine call (marl_engine_step):
              wall time of the whole tick including the device->host change
              list, the host fate step and the host->device edit list.
  roofline    the dominant kernel (diffusion substep): algorithmic bytes
              (97 B/voxel: 48 read + 48 written + 1 mask) / CUDA-event time.
  cpu_baseline  the CPU oracle (restatement of the reference) on this host.
Multi-GPU: independent replicas (one run per GPU, no collective on the data
path); value = total ticks of all ranks / max over ranks of the device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "marl-ochre_b200"))

DIMS = (128, 128, 64)
SEED = 42
SEED_COUNT = 30
METRIC = "ticks/s at 128x128x64 (plain vs batched/surrogate, <=1e-3 rel err); HBM GB/s"
BYTES_PER_VOXEL_SUBSTEP = 97  # 48 B read + 48 B written + 1 B occupancy
L2_FLUSH_BYTES = 256 << 20
REFERENCE_TICKS_PER_S = 1.9  # reference CPU engine, 128x128x64 (recorded in the reference's notes)
WORKLOAD = ("reference default run: 128x128x64 grid, 12 species, Winogradsky boundary priming, "
            "3 starters x 30 seeded cells, host RNG seed 42, 10 diffusion substeps/tick, f32")


def peaks() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(name: str):
    """DRAM bytes per launch from a committed ncu summary, if one exists."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed loop runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = max(smax, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(values, dist, device) -> list:
    """Element-wise maximum of per-rank timings (the slowest replica sets the
    job's time); identity without a process group."""
    if dist is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def replica_rates(steps: int, world: int, dev_s: float, wall_s: float) -> tuple[float, float]:
    """Whole-job ticks/s of `world` independent replicas of `steps` ticks each,
    from the maximum device time and the maximum wall time over ranks."""
    total = steps * world
    return total / dev_s, total / wall_s


def cpu_baseline(budget_s: float = 15.0, max_ticks: int = 60) -> dict:
    """The CPU oracle (restatement of the reference) on the same workload, this host's cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    w = oracle.World(DIMS, seed=SEED, seed_count=SEED_COUNT)
    w.tick(1)  # warm-up (page-in, thread pool)
    n, t0 = 0, time.perf_counter()
    while n < max_ticks and time.perf_counter() - t0 < budget_s:
        w.tick(1)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "ticks/s", "cores": threads, "kind": "port",
            "sample": f"{n} ticks (ticks 1..{n}) of the same seed-42 default run; diffusion over z on "
                      f"{threads} OpenMP threads as rayon does, light and cells single-threaded"}


def run_reference(args) -> int:
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    w = oracle.World(DIMS, seed=SEED, seed_count=SEED_COUNT)
    w.tick(max(args.warmup, 0))
    budget = 120.0
    n, t0 = 0, time.perf_counter()
    while n < args.steps and time.perf_counter() - t0 < budget:
        w.tick(1)
        n += 1
    dt = time.perf_counter() - t0
    v = n / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "ticks/s", "n_gpus": args.gpus, "steps": n,
        "warmup": args.warmup, "ms_per_step": 1000.0 * dt / max(n, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": v / REFERENCE_TICKS_PER_S, "dtype": "f32",
        "data": "synthetic (seeded Winogradsky initial condition)",
        "config": {"workload": WORKLOAD, "grid": list(DIMS), "seed": SEED, "seed_count": SEED_COUNT},
        "cpu_baseline": {"value": v, "unit": "ticks/s", "cores": threads, "kind": "port",
                         "sample": f"{n} ticks after {args.warmup} warm-up ticks (at most {budget:.0f} s); CPU "
                                   f"restatement of the reference (the Rust engine cannot be built here)"},
        "e2e": {"value": v, "unit": "ticks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def diffusion_roofline(marl, torch, engine, stream, fixed_tile=None) -> dict:
    """Times the diffusion substep on the engine's current state with CUDA events."""
    ctx = marl.Context(DIMS, engine.params, cell_capacity=max(int(engine.stats()["population"]), 1) + 16)
    ctx.set_stream(stream.cuda_stream)
    ctx.upload_field(engine.field())
    ctx.upload_cells(engine.cells())
    if fixed_tile is None:
        us = ctx.autotune(5)
    else:
        ctx.set_tile(*fixed_tile)
        us = None
    tile, zc = ctx.get_tile()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    groups, per_group = 20, 10
    for _ in range(3):
        ctx.diffuse(per_group)
    total_ms = 0.0
    for _ in range(groups):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.diffuse(per_group)
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    t_sub = total_ms / 1000.0 / (groups * per_group)
    V = DIMS[0] * DIMS[1] * DIMS[2]
    bytes_per_launch = BYTES_PER_VOXEL_SUBSTEP * V
    achieved = bytes_per_launch / t_sub / 1e9
    peak, src = peaks()
    traffic = ncu_traffic("diffusion_traffic.json")
    tr = None
    if traffic and traffic.get("grid") == list(DIMS):
        tr = traffic.get("dram_bytes_per_launch")
    ctx.close()
    tiles = ["16x8 (4 stages)", "16x16 (4 stages)", "16x4 (4 stages)", "16x32 (4 stages)",
             "16x8 (3 stages)", "16x16 (3 stages)", "16x4 (3 stages)", "16x32 (3 stages)",
             "16x4 (3 stages, direct stores)", "16x8 (3 stages, direct stores)",
             "16x16 (3 stages, direct stores)", "16x32 (3 stages, direct stores)"]
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": tr, "kernel": "k_diffuse (diffusion substep, TMA z-march)", "peak_source": src,
            "algorithmic_bytes_per_launch": bytes_per_launch, "us_per_launch": t_sub * 1e6,
            "tile": f"{tiles[tile]} columns, z-chunk {zc}", "autotune_us_per_substep": us,
            "l2": "flushed between groups of 10 substeps (one tick's worth)"}


ENSEMBLE_GRIDS = [(64, 64, 32), (96, 96, 48), (128, 128, 64), (128, 128, 96)]
MLP_FLOP_PER_CELL = 2 * (93 * 256 + 256 * 256 + 256 * 16)  # algorithmic forward FLOPs (93 inputs)
TICK_COMPARE = 1000  # the surrogate's tick comparison starts from this tick of the seed-42 run


def device_fate_leg(marl, torch, stream, steps: int, warmup: int, flush) -> dict:
    """The same default run with fate on the device (per-division streams keyed
    by the run seed): every tick through marl_engine_step with an L2 flush
    between ticks, then `steps` more ticks enqueued by one marl_engine_step call."""
    eng = marl.Engine(DIMS, marl.default_params(), rng_seed=SEED, seed_count=SEED_COUNT, cell_capacity=1 << 20)
    eng.set_stream(stream.cuda_stream)
    eng.autotune(5)
    eng.set_device_fate(True)
    eng.step(warmup)
    torch.cuda.synchronize()
    c0 = eng.counters()
    wall = 0.0
    h2d = d2h = 0
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.step(1)
        torch.cuda.synchronize()
        wall += time.perf_counter() - t0
        s = eng.stats()
        h2d += s["h2d_bytes_last_tick"]
        d2h += s["d2h_bytes_last_tick"]
    c1 = eng.counters()
    st = eng.stats()
    dev_s = (c1["device_us"] - c0["device_us"]) / 1e6
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    eng.step(steps)
    torch.cuda.synchronize()
    wall_one_call = time.perf_counter() - t0
    st2 = eng.stats()
    eng.close()
    return {"e2e_ticks_per_s": steps / wall, "device_ticks_per_s": steps / dev_s,
            "one_call_ticks_per_s": steps / wall_one_call,
            "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps,
            "launches_per_tick": (c1["kernel_launches"] - c0["kernel_launches"]) / steps,
            "population_end": int(st["population"]), "divisions": int(st["total_divisions"]),
            "deaths": int(st["total_deaths"]),
            "one_call_ticks": f"{warmup + steps + 1}..{warmup + 2 * steps}",
            "one_call_population_end": int(st2["population"]),
            "api": "marl_engine_step (C ABI) with marl_engine_set_device_fate: per tick, wall clock incl. the "
                   "64-byte fate-counter read; one_call: all ticks in one call, one synchronisation",
            "note": "fate on the device draws from per-division streams, so the run's trajectory differs from "
                    "the host-fate run (same model, different random numbers)"}


def ensemble_leg(marl, torch, stream, ticks: int = 1000, window: int = 20, surrogate=None) -> dict:
    """Batched ensemble as configured: 64 runs, seeds 0-63, 16 each of four grid
    sizes, default seeding, one launch per phase for all runs and a
    graph-captured device tick, advanced `ticks` ticks from seeding with host
    fate and timed over all of them (device time and end to end); from the
    tick-`ticks` state, `window` more plain ticks and then, with a trained
    surrogate, `window` ticks gated at 1e-3; and the same ensemble with fate on
    the device, `ticks` ticks from seeding."""
    # Table capacity: half the voxels of the run's grid (the seeded runs hold
    # about a quarter of their voxels at most by tick 1000).
    runs = [(g, i, SEED_COUNT, g[0] * g[1] * g[2] // 2) for i, g in ((i, ENSEMBLE_GRIDS[i // 16]) for i in range(64))]

    def make(device_fate):
        b = marl.Batch(runs, marl.default_params(), seed_count=SEED_COUNT)
        b.set_stream(stream.cuda_stream)
        us = b.autotune(3)
        if device_fate:
            b.set_device_fate(True)
        return b, us

    def timed(b, n):
        torch.cuda.synchronize()
        c0 = b.counters()
        t0 = time.perf_counter()
        b.step(n)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        c1 = b.counters()
        return (c1["device_us"] - c0["device_us"]) / 1e6, wall

    def population(b):
        return int(sum(b.stats(r)["population"] for r in range(len(runs))))

    def whole_run(b, us):
        dev = wall = 0.0
        trajectory = []
        chunk = max(ticks // 10, 1)
        done = 0
        while done < ticks:
            n = min(chunk, ticks - done)
            d, w = timed(b, n)
            dev += d
            wall += w
            done += n
            trajectory.append({"tick": done, "population": population(b),
                               "run_ticks_per_s": len(runs) * n / d})
        return {"ticks": f"1..{ticks}", "run_ticks_per_s": len(runs) * ticks / dev,
                "e2e_run_ticks_per_s": len(runs) * ticks / wall, "ms_per_batch_tick": 1000.0 * dev / ticks,
                "population_end": population(b), "population_trajectory": trajectory,
                "autotune_us_per_batched_substep": us}

    b, us = make(False)
    res = whole_run(b, us)
    res["workload"] = ("64 runs, seeds 0-63, 16 each of 64x64x32, 96x96x48, 128x128x64, 128x128x96, default "
                       f"seeding; ticks 1..{ticks} from seeding, host fate")
    res["note"] = ("device time: CUDA events on the batch stream around the graph-replayed device ticks and edit "
                   "copies; e2e adds the host fate step of all runs on worker threads")
    d, w = timed(b, window)
    res["plain_window"] = {"ticks": f"{ticks + 1}..{ticks + window}", "run_ticks_per_s": len(runs) * window / d,
                           "e2e_run_ticks_per_s": len(runs) * window / w, "population_end": population(b)}
    if surrogate is not None:
        b.set_surrogate(surrogate, marl.SURR_GATED, 1e-3)
        d, w = timed(b, window)
        cnt = b.surrogate_counters()
        res["gated_1e-3_window"] = {
            "ticks": f"{ticks + window + 1}..{ticks + 2 * window}", "run_ticks_per_s": len(runs) * window / d,
            "e2e_run_ticks_per_s": len(runs) * window / w, "population_end": population(b),
            "surrogate_counters": {k: (float(v) if isinstance(v, float) else int(v)) for k, v in cnt.items()},
            "note": "max_err: largest normwise error, over the 16 species, of an accepted cell's final state "
                    "(after maintenance and effectors) against the plain kernel's"}
        b.set_surrogate(None, marl.SURR_OFF)
    b.close()
    bd, us = make(True)
    res["with_device_fate"] = whole_run(bd, us)
    res["with_device_fate"]["note"] = ("fate of every run on the device: one CUDA graph per batch tick, one "
                                       "synchronisation per step call; per-division random streams, so the "
                                       "trajectories differ from the host-fate runs")
    bd.close()
    return res


def surrogate_leg(marl, torch, stream, budget_s: float = 45.0, target_pairs: int = 10_000_000):
    """Learned reaction surrogate: pairs captured from the plain cell kernel on
    seeded 128x128x64 default runs, trained on the GPU, evaluated on held-out
    rows and in the tick (gated at 1e-3 and trusted), against the plain tick
    from the same state.  Returns (trained surrogate, result)."""
    t_start = time.perf_counter()
    p = marl.default_params()
    s = marl.Surrogate(max_pairs=target_pairs, batch=8192, lr=2e-3, seed=5)
    s.set_stream(stream.cuda_stream)
    seed, cap_ticks = 100, 0
    while s.pair_count() < target_pairs and time.perf_counter() - t_start < budget_s / 3:
        e = marl.Engine(DIMS, p, rng_seed=seed, seed_count=SEED_COUNT, cell_capacity=1 << 20)
        e.set_stream(stream.cuda_stream)
        e.step(20)
        marl.ctx_set_surrogate(e.lib.marl_engine_ctx(e.h), s, marl.SURR_CAPTURE)
        while s.pair_count() < target_pairs and time.perf_counter() - t_start < budget_s / 3:
            e.step(20)
            cap_ticks += 20
            if e.stats()["tick"] >= 600:
                break
        marl.ctx_set_surrogate(e.lib.marl_engine_ctx(e.h), None, marl.SURR_OFF)
        e.close()
        seed += 1
    t_cap = time.perf_counter() - t_start
    n = s.pair_count()
    n_train = int(0.95 * n)
    s.prepare(n_train)
    # A fixed number of Adam steps with a stepped learning rate (2e-3, 5e-4,
    # then 1e-4 to settle): acceptance at 1e-3 is sensitive to where the last
    # steps leave the weights.
    t0 = time.perf_counter()
    steps = 0
    losses = []
    for lr, n_steps in ((2e-3, 16000), (5e-4, 16000), (1e-4, 8000)):
        s.set_lr(lr)
        losses.append(s.train(n_steps))
        steps += n_steps
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    held = s.evaluate(n_train, n - n_train, tol=1e-3)
    raw = s.download_pairs(n_train, min(n - n_train, 200_000))
    d = raw[:, 93:109]
    plain = raw[:, :16] + d
    zero_ok = float(((np.abs(d).max(1) / np.maximum(np.abs(plain).max(1), 1e-6)) <= 1e-3).mean())

    # Inference kernels alone: three tcgen05 GEMM launches on n_cells rows.
    n_cells = 300_000
    x = torch.randn(n_cells, 128, device="cuda").to(torch.bfloat16)
    x[:, 93:] = 0
    y = torch.empty(16, n_cells, device="cuda")
    for _ in range(3):
        s.infer_device(x.data_ptr(), n_cells, y.data_ptr(), n_cells)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    ev0.record(stream)
    for _ in range(reps):
        s.infer_device(x.data_ptr(), n_cells, y.data_ptr(), n_cells)
    ev1.record(stream)
    ev1.synchronize()
    infer_s = ev0.elapsed_time(ev1) / 1000.0 / reps
    tflops = MLP_FLOP_PER_CELL * n_cells / infer_s / 1e12

    # The tick in each mode, from the tick-1000 state of the seed-42 default run
    # (the run's population at the end of the configured 1000 ticks).
    e = marl.Engine(DIMS, p, rng_seed=SEED, seed_count=SEED_COUNT, cell_capacity=1 << 20)
    e.set_stream(stream.cuda_stream)
    e.step(TICK_COMPARE)
    field, cells, light = e.field(), e.cells(), e.light()
    e.close()
    modes = {}
    finals = {}
    for name, mode in (("plain", marl.SURR_OFF), ("gated", marl.SURR_GATED), ("trusted", marl.SURR_TRUSTED)):
        # one cell phase from the identical state, for the error against the plain kernel
        ctx = marl.Context(DIMS, p, cell_capacity=len(cells))
        ctx.upload_field(field)
        ctx.upload_light(light)
        ctx.upload_cells(cells)
        if mode != marl.SURR_OFF:
            marl.ctx_set_surrogate(ctx.h, s, mode, 1e-3)
        ctx.cell_phase()
        finals[name] = ctx.download_cells()["internal"]
        ctx.close()
        # whole ticks through the engine, device time
        eng = marl.Engine(DIMS, p, rng_seed=SEED, field=field, cells=cells, cell_capacity=1 << 20)
        eng.set_stream(stream.cuda_stream)
        h = eng.lib.marl_engine_ctx(eng.h)
        if mode != marl.SURR_OFF:
            marl.ctx_set_surrogate(h, s, mode, 1e-3)
        eng.step(3)
        torch.cuda.synchronize()
        c0 = eng.counters()
        k = 20
        eng.step(k)
        c1 = eng.counters()
        cnt = marl.ctx_surrogate_counters(h) if mode != marl.SURR_OFF else None
        modes[name] = {"ticks_per_s": k / ((c1["device_us"] - c0["device_us"]) / 1e6),
                       "counters": None if cnt is None else {kk: (float(v) if isinstance(v, float) else int(v))
                                                             for kk, v in cnt.items()}}
        eng.close()
    for name in ("gated", "trusted"):
        a, b = finals[name], finals["plain"]
        err = np.abs(a - b).max(1) / np.maximum(np.abs(b).max(1), 1e-6)
        modes[name]["cell_phase_rel_err_max"] = float(err.max())
        modes[name]["cell_phase_cells_within_1e-3"] = float((err <= 1e-3).mean())
    return s, {
        "workload": f"pairs from {seed - 100} seeded 128x128x64 default runs (ticks 21..<=600), "
                    f"{n} rows, last 5% held out; tick comparison from tick {TICK_COMPARE} of the seed-{SEED} "
                    f"run ({len(cells)} cells)",
        "population_note": "the configured ~300k cells at 128x128x64 are not reached by the seeded default run: it "
                           "holds 38k cells at tick 1000 and 57k at tick 1600 (29% occupancy would be 300k); the "
                           "300k-row figure is the inference leg's, on synthetic rows",
        "pairs": n, "capture_s": t_cap, "train_steps": steps, "train_batch": 8192, "train_s": t_train,
        "train_lr_schedule": "2e-3 x 16000, 5e-4 x 16000, 1e-4 x 8000 steps",
        "loss_first": float(losses[0][:20].mean()), "loss_last": float(losses[-1][-100:].mean()),
        "held_out": {"rows": held["rows"], "accepted_frac_1e-3": held["accepted"] / held["rows"],
                     "mean_err": held["mean_err"], "zero_delta_accepted_frac_1e-3": zero_ok},
        "mlp_infer": {"cells": n_cells, "us": infer_s * 1e6, "tflops_algorithmic": tflops,
                      "peak_tflops": peaks_bf16(), "frac": tflops / peaks_bf16(),
                      "flop_per_cell": MLP_FLOP_PER_CELL},
        "tick_modes": modes,
    }


def field_microbench_leg(marl, torch, stream, substeps: int = 100) -> dict:
    """256x256x128 field microbenchmark: 100 diffusion substeps (autotuned
    tile; the last substep also writes species 4 compactly), then the
    Beer-Lambert scan."""
    import workloads

    dims = workloads.MICRO_DIMS
    X, Y, Z = dims
    field, occ = workloads.field_microbench()
    z, y, x = np.nonzero(occ)
    walls = np.zeros(len(x), marl.CELL_DTYPE)  # occupancy only: cells that are never updated here
    walls["pos"] = np.stack([x, y, z], 1).astype(np.uint16)
    p = marl.default_params()
    ctx = marl.Context(dims, p, cell_capacity=len(walls))
    ctx.set_stream(stream.cuda_stream)
    ctx.upload_cells(walls)
    ctx.upload_field(field)
    us_tuned = ctx.autotune(3)
    tile, zc = ctx.get_tile()
    ctx.diffuse(4)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.diffuse(substeps)
    e1.record(stream)
    e1.synchronize()
    t_sub = e0.elapsed_time(e1) / 1000.0 / substeps
    V = X * Y * Z
    peak, src = peaks()
    diff_gbs = BYTES_PER_VOXEL_SUBSTEP * V / t_sub / 1e9
    ctx.light_update()  # warm-up; species 4 comes from the compact copy of the last substep
    reps = 20
    e0.record(stream)
    for _ in range(reps):
        ctx.light_update()
    e1.record(stream)
    e1.synchronize()
    t_light = e0.elapsed_time(e1) / 1000.0 / reps
    ctx.close()
    return {"workload": "256x256x128, 12 species U[0,1), 5% occupied as balls of radius 2-4, deposit factor "
                        "U[0.5,1] through species 7; 100 substeps, then the light scan (absorbance 0.05*U[0,1))",
            "us_per_substep": t_sub * 1e6, "tile": int(tile), "zc": int(zc), "autotune_us": us_tuned,
            "diffusion_gbs_algorithmic": diff_gbs, "diffusion_frac_of_measured_hbm": diff_gbs / peak,
            "bytes_per_voxel_substep": BYTES_PER_VOXEL_SUBSTEP,
            "light_us": t_light * 1e6, "light_gbs_algorithmic": 9 * V / t_light / 1e9,
            "light_frac_of_measured_hbm": 9 * V / t_light / 1e9 / peak, "peak_gbs": peak, "peak_source": src,
            "l2": "the 384 MiB buffers exceed L2"}


def cell_microbench_leg(marl, torch, stream, phases: int = 200) -> dict:
    """1,000,000 cells on 256x256x128: 200 repetitions of the cell loop
    (gather, transport, reactions, effectors, scatter) with no fate edits."""
    import workloads

    dims = workloads.MICRO_DIMS
    field, _ = workloads.field_microbench()
    cells = workloads.cell_microbench()
    touched = workloads.touched_voxels(cells, dims)
    p = marl.default_params()
    ctx = marl.Context(dims, p, cell_capacity=len(cells))
    ctx.set_stream(stream.cuda_stream)
    ctx.upload_field(field)
    ctx.upload_cells(cells)
    ctx.light_update()
    lib = marl.load()
    for _ in range(3):
        marl._check(lib.marl_cell_phase(ctx.h, None), "marl_cell_phase")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(phases):
        marl._check(lib.marl_cell_phase(ctx.h, None), "marl_cell_phase")
    e1.record(stream)
    e1.synchronize()
    t = e0.elapsed_time(e1) / 1000.0 / phases
    ctx.synchronize()
    ctx.close()
    alg = 592 * len(cells) + 96 * touched
    peak, src = peaks()
    return {"workload": "1,000,000 cells at unique random voxels of 256x256x128; 16 reactions with random "
                        "wiring, v_max lognormal(0,1), k_m and k_cat U[0.01,1], light catalysis on 25%; "
                        "8 transporters and 8 effectors; 200 cell-loop phases without fate edits",
            "ms_per_phase": t * 1e3, "cells_per_s": len(cells) / t, "touched_empty_voxels": touched,
            "algorithmic_bytes_per_phase": alg, "gbs_algorithmic": alg / t / 1e9,
            "frac_of_measured_hbm": alg / t / 1e9 / peak, "peak_source": src}


def peaks_bf16() -> float:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"])
    except Exception:
        return 1590.0


# ----------------------------------------------------------------- cases ----
# Single-kernel cases on seeded synthetic inputs, for profiling one kernel in
# isolation (`python bench.py --case ...`).  Each builds a context, uploads the
# state and runs the kernel a few times; under `ncu -k regex:<kernel> -s <n>
# -c 1` that captures one launch with the earlier launches as warm-up.  The
# engine case runs the seed-42 default run: one k_cell_tick launch per tick, so
# `-k regex:k_cell_tick -s <ticks-1> -c 1` captures the last; with
# --device-fate all ticks are enqueued at once.

def case_clustered_cells(marl, dims, frac: float, rng: np.random.Generator) -> np.ndarray:
    """Cells on random balls of radius 2-4 until `frac` of the voxels are covered."""
    X, Y, Z = dims
    occ = np.zeros((Z, Y, X), bool)
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    while occ.sum() < frac * X * Y * Z:
        r = rng.integers(2, 5)
        cx, cy, cz = rng.integers(0, X), rng.integers(0, Y), rng.integers(0, Z)
        occ |= (xx - cx) ** 2 + (yy - cy) ** 2 + (zz - cz) ** 2 <= r * r
    z, y, x = np.nonzero(occ)
    c = np.zeros(len(x), marl.CELL_DTYPE)
    c["pos"] = np.stack([x, y, z], 1)
    return c


def case_random_cells(marl, dims, n: int, rng: np.random.Generator) -> np.ndarray:
    """n cells with random rulesets at unique random voxels."""
    X, Y, Z = dims
    flat = rng.choice(X * Y * Z, size=n, replace=False)
    z, rem = np.divmod(flat, X * Y)
    y, x = np.divmod(rem, X)
    c = np.zeros(n, marl.CELL_DTYPE)
    c["pos"] = np.stack([x, y, z], 1)
    c["internal"] = rng.random((n, 16), dtype=np.float32)
    rx = c["ruleset"]["reactions"]
    rx["substrate"] = rng.integers(0, 16, (n, 16))
    rx["product"] = rng.integers(0, 16, (n, 16))
    rx["catalyst"] = rng.integers(0, 16, (n, 16))
    rx["cofactor"] = 0xFF
    rx["k_m"] = (0.01 + 0.99 * rng.random((n, 16))).astype(np.float32)
    rx["v_max"] = rng.lognormal(0.0, 1.0, (n, 16)).astype(np.float32)
    rx["k_cat"] = (0.01 + 0.99 * rng.random((n, 16))).astype(np.float32)
    tp = c["ruleset"]["transport"]
    tp["uptake_rate"] = rng.random((n, 8), dtype=np.float32)
    tp["secrete_rate"] = rng.random((n, 8), dtype=np.float32)
    tp["ext_species"] = rng.integers(0, 12, (n, 8))
    tp["int_species"] = rng.integers(0, 16, (n, 8))
    c["ruleset"]["fate"]["division_energy"] = 10.0
    return c


def case_mlp(marl, rows: int, reps: int, rng: np.random.Generator) -> int:
    """Surrogate inference on `rows` random standardised feature rows, random weights."""
    import torch

    s = marl.Surrogate(max_pairs=128, batch=128)
    s.set_stream(torch.cuda.current_stream().cuda_stream)  # inputs are torch tensors
    params = np.zeros(marl.SURR_PARAMS, np.float32)
    params[: 256 * 128] = rng.normal(0, 0.1, 256 * 128)
    params[256 * 128 + 256: 256 * 128 + 256 + 65536] = rng.normal(0, 0.06, 65536)
    params[-16 - 4096: -16] = rng.normal(0, 0.06, 4096)
    norm = np.zeros(marl.SURR_NORM, np.float32)
    norm[93:186] = 1.0
    norm[202:218] = 1.0
    s.set_weights(params, norm)
    x = torch.randn(rows, 128, device="cuda").to(torch.bfloat16)
    x[:, 93:] = 0
    y = torch.empty(16, rows, device="cuda")
    torch.cuda.synchronize()
    for _ in range(reps):
        s.infer_device(x.data_ptr(), rows, y.data_ptr(), rows)
    torch.cuda.synchronize()
    print(f"mlp ok: rows={rows} reps={reps} finite={bool(torch.isfinite(y).all())}")
    s.close()
    return 0


def run_case(args) -> int:
    import marl_cuda as marl

    dims = tuple(args.dims)
    X, Y, Z = dims
    rng = np.random.default_rng(1)
    if args.case == "mlp":
        return case_mlp(marl, args.rows, args.reps, rng)
    if args.case == "engine":
        e = marl.Engine(dims, marl.default_params(), rng_seed=42, seed_count=30, cell_capacity=1 << 20)
        if args.device_fate:
            e.set_device_fate(True)
        e.step(args.ticks)
        print(f"engine ok: dims={dims} ticks={args.ticks} stats={e.stats()}")
        return 0
    field = rng.random((Z, Y, X, 12), dtype=np.float32)
    if args.case == "cells":
        cells = case_random_cells(marl, dims, args.cells, rng)
    else:
        cells = case_clustered_cells(marl, dims, 0.05, rng)
    ctx = marl.Context(dims, cell_capacity=max(len(cells), 1))
    ctx.upload_field(field)
    ctx.upload_cells(cells)
    if args.case == "diffusion":
        if args.tile:
            ctx.set_tile(*args.tile)
        else:
            ctx.autotune(3)
        ctx.diffuse(args.substeps)
    elif args.case == "cells":
        ctx.upload_light(rng.random((Z, Y, X), dtype=np.float32))
        for _ in range(args.reps):
            ctx.cell_phase()
    else:
        for _ in range(args.reps):
            ctx.light_update()
    ctx.synchronize()
    print(f"{args.case} ok: dims={dims} cells={len(cells)} tile={ctx.get_tile()}")
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tile", type=int, nargs=2, metavar=("TILE", "ZC"),
                    help="fixed diffusion tile index and z-chunk instead of the autotuner (launch lists, cases)")
    ap.add_argument("--no-roofline", action="store_true", help="skip the separate diffusion timing")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble leg")
    ap.add_argument("--ensemble-ticks", type=int, default=1000, help="ticks of the 64-run ensemble from seeding")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the learned-surrogate leg")
    ap.add_argument("--no-micro", action="store_true", help="skip the field and cell microbenchmarks")
    ap.add_argument("--no-device-fate", action="store_true", help="skip the device-fate engine leg")
    ap.add_argument("--case", choices=["diffusion", "cells", "light", "mlp", "engine"],
                    help="instead of the benchmark, run one kernel on seeded synthetic inputs (for ncu)")
    ap.add_argument("--dims", type=int, nargs=3, default=[128, 128, 64], help="case grid")
    ap.add_argument("--substeps", type=int, default=8, help="case diffusion: substeps")
    ap.add_argument("--cells", type=int, default=90, help="case cells: random cells")
    ap.add_argument("--reps", type=int, default=4, help="case cells/light/mlp: repetitions")
    ap.add_argument("--rows", type=int, default=300_000, help="case mlp: rows per inference")
    ap.add_argument("--ticks", type=int, default=1000, help="case engine: ticks of the seed-42 default run")
    ap.add_argument("--device-fate", action="store_true", help="case engine: fate on the device")
    args = ap.parse_args()
    if args.case:
        return run_case(args)
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import marl_cuda as marl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    # One explicit stream for the engine, the L2 flush and the timing events.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    eng = marl.Engine(DIMS, marl.default_params(), rng_seed=SEED, seed_count=SEED_COUNT, cell_capacity=1 << 20)
    eng.set_stream(stream.cuda_stream)
    if args.tile:
        lib = marl.load()
        marl._check(lib.marl_ctx_set_tile(lib.marl_engine_ctx(eng.h), args.tile[0], args.tile[1]), "set_tile")
    else:
        eng.autotune(5)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    eng.step(args.warmup)
    pop0 = eng.stats()["population"]

    sampler = ClockSampler(torch.cuda.current_device())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    c0 = eng.counters()
    sampler.start()
    wall = 0.0
    h2d = d2h = 0
    for _ in range(args.steps):
        flush.zero_()  # L2 flush between steps (outside the timed spans)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.step(1)
        torch.cuda.synchronize()
        wall += time.perf_counter() - t0
        s = eng.stats()
        h2d += s["h2d_bytes_last_tick"]
        d2h += s["d2h_bytes_last_tick"]
    torch.cuda.synchronize()
    c1 = eng.counters()
    clocks = sampler.stop()
    dev_s = (c1["device_us"] - c0["device_us"]) / 1e6
    launches = c1["kernel_launches"] - c0["kernel_launches"]
    st = eng.stats()
    dev_s, wall = max_over_ranks([dev_s, wall], dist, "cuda")
    if dist:
        dist.barrier()
    value, e2e = replica_rates(args.steps, world, dev_s, wall)

    roof = None
    if rank == 0 and not args.no_roofline:
        roof = diffusion_roofline(marl, torch, eng, stream, tuple(args.tile) if args.tile else None)
    ens = surr = fmicro = cmicro = dfate = None
    if rank == 0 and world == 1 and not args.no_device_fate:
        dfate = device_fate_leg(marl, torch, stream, args.steps, args.warmup, flush)
    if rank == 0 and world == 1 and not args.no_micro:
        fmicro = field_microbench_leg(marl, torch, stream)
        cmicro = cell_microbench_leg(marl, torch, stream)
    trained = None
    if rank == 0 and world == 1 and not args.no_surrogate:
        trained, surr = surrogate_leg(marl, torch, stream)
    if rank == 0 and world == 1 and not args.no_ensemble:
        ens = ensemble_leg(marl, torch, stream, ticks=args.ensemble_ticks, surrogate=trained)
    if trained is not None:
        trained.close()
    if rank == 0:
        base = None if (args.no_cpu_baseline or world > 1) else cpu_baseline()
        line = {
            "metric": METRIC, "value": value, "unit": "ticks/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * dev_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": value / REFERENCE_TICKS_PER_S, "dtype": "f32",
            "data": "synthetic (seeded Winogradsky initial condition of the reference default run)",
            "config": {"workload": WORKLOAD, "grid": list(DIMS), "seed": SEED, "seed_count": SEED_COUNT,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "flushed between steps (256 MiB device write, outside the timed spans)",
                       "population_start": int(pop0), "population_end": int(st["population"]),
                       "divisions": int(st["total_divisions"]), "deaths": int(st["total_deaths"])},
            "roofline": roof,
            "cpu_baseline": base,
            "e2e": {"value": e2e, "unit": "ticks/s", "h2d_bytes_per_step": h2d / args.steps,
                    "d2h_bytes_per_step": d2h / args.steps,
                    "api": "marl_engine_step (C ABI), wall clock per tick"},
            "e2e_device_fate": dfate,
            "clocks": clocks,
            "gpu_launches": int(launches),
            "field_microbench": fmicro,
            "cell_microbench": cmicro,
            "ensemble": ens,
            "surrogate": surr,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
