#!/usr/bin/env python
"""Benchmark of the LSMPS per-step particle hot path on B200.

A step is the reference driver's step without the PPE solve and I/O
(src/app/simulation_driver.cu:346-383): moments -> provision -> PPE assembly
-> pressure correction (pressure = the clamped fluid pressure) -> neighbour
rebuild -> surface labels.  The workload is the splash-heavy dam break:
200 x 50 x 200 = 2,000,000 fluid particles (l0 = 0.0025 m, r_e = 3.1 l0) in
a 1.0 x 0.25 x 0.5 m tank with 3 wall layers, 5% of the fluid lifted into the
10 l0 above the free surface (seeded synthetic input).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload splash|dam_break|hydrostatic|batched|splash_shuffled|virtual_light|ppe_solve]

virtual_light and ppe_solve time one stage outside the step (the
virtual-light diagnostic; the PPE solve with the reference's AMGX settings)
on the splash workload's state after one step.

N > 1 runs under torchrun: every rank runs an independent replica (the path
does not shard; there is no data-path collective) and value = N x particles /
the slowest rank's time.  Rank 0 prints one JSON line.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import __graft_entry__ as graft_entry  # noqa: E402

METRIC = "particles/s per LSMPS step, mixed vs plain FP64 on 1 B200 at stated error; HBM %"
KNOB_NAMES = {0: "moment_occupancy", 1: "ppe_lanes", 2: "gather_lanes"}
WORKLOADS = {
    "splash": ("splash", {}, "splash dam break 200x50x200 (2M fluid, l0=0.0025 m, 5% splash, 3 wall layers)"),
    "dam_break": ("dam_break", {}, "dam break 100x50x100 (500k fluid, l0=0.005 m, jitter 0.05 l0, 3 wall layers)"),
    "hydrostatic": ("hydrostatic", {}, "hydrostatic box 20^3 (8k fluid, l0=0.01 m, 3 wall layers)"),
    "batched": ("batched", {}, "64 independent boxes, fluid counts log-uniform in [8k, 200k] (seed 7), hydrostatic "
                               "or dam-break layout by seeded coin flip, 3 wall layers, l0=0.005 m"),
    # Stages outside the step, on the geometry of the splash workload after one step.
    "splash_shuffled": ("splash_shuffled", {}, "splash dam break 200x50x200 (2M fluid) with the fluid numbered in a "
                                               "seeded random order, stepped before and after lsmps_reorder_fluid"),
    "virtual_light": ("splash", {}, "virtual-light diagnostic on the splash dam break 200x50x200 (2M fluid)"),
    "ppe_solve": ("splash", {}, "PPE solve (GMRES(20), 100 iterations, 1e-6 relative, from zero: the reference's AMGX "
                                "configuration) of the splash dam break 200x50x200 (2M rows)"),
}
STAGE_METRICS = {
    "virtual_light": "particles/s of the virtual-light diagnostic (compute_virtual_light_diagnostics) on 1 B200",
    "ppe_solve": "PPE solves/s (AmgxPpeSolver::solve semantics) on 1 B200",
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOADS), default="splash")
    ap.add_argument("--stage-case", choices=["splash", "dam_break"], default="splash",
                    help="state the virtual_light / ppe_solve workloads run on (dam_break: the 500k case, for "
                         "profiler captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-renumbered", action="store_true",
                    help="skip the extra timing after lsmps_reorder_fluid (fluid renumbered in cell order)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch-shape knobs")
    ap.add_argument("--no-scattered", action="store_true",
                    help="skip the forms on the splash variant with the lifted particles scattered off the lattice "
                         "(ill-conditioned Surface/Splash matrices: the mixed form's FP64 route at full size)")
    ap.add_argument("--knobs", default=None,
                    help="comma-separated launch-shape knob values (moment variant, PPE lanes, gather lanes) to use "
                         "instead of autotuning, e.g. 2,1,1 (what the autotuner picks at 2M)")
    ap.add_argument("--kappa-threshold", type=float, default=None,
                    help="mixed form: condition-estimate threshold of the FP64 route (library default if omitted)")
    ap.add_argument("--precision", choices=["both", "plain", "mixed"], default="both",
                    help="forms to time; the last one timed is the headline (mixed when both)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3][0].isdigit())}


# ---------------------------------------------------------------------------
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, value: float, device) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_traffic(kernel: str, n_fluid: int):
    """DRAM bytes per launch of `kernel` from the committed ncu summary of the
    500k dam break (profiles/), scaled to this workload by fluid-particle
    count (the kernels' traffic grows in proportion); None if not captured."""
    import glob

    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "dram_traffic_*.json"))):
        with open(path) as fh:
            d = json.load(fh)
        k = d.get("kernels", {}).get(kernel)
        if k:
            return (k["dram_bytes_per_fluid_particle"] * n_fluid,
                    f"{os.path.basename(path)}: ncu dram__bytes_read+write at {d['n_fluid']} fluid particles, "
                    f"scaled by fluid count")
    return None, None


def peaks() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    pkg = graft_entry.load_package()
    from importlib import import_module

    import_module("lsmps3d_b200.build").build_all()
    api = import_module("lsmps3d_b200.api")
    roofline = import_module("lsmps3d_b200.roofline")
    device = torch.device(f"cuda:{local}")
    kind, kw, desc = WORKLOADS[args.workload]
    case = pkg.cases.CASES[kind](**kw)
    p = case.params
    stream = torch.cuda.Stream(device)
    with torch.cuda.stream(stream):
        dev = api.device_buffers(case, device=device)
        ctx = api.Context(local)
        if args.kappa_threshold is not None:
            ctx.set_condition_threshold(args.kappa_threshold)
        ctx.reserve(case.n_fluid, case.n_wall, case.n_cells)
        state = dev.step_state(p)

        def reset():
            dev.load_case(case)
            ctx.set_synchronous(True)
            ctx.build_neighbor_lists(dev, p)
            ctx.classify_surface(dev, p)
            ctx.set_synchronous(False)

        def timed_steps(k):
            barrier(world)
            ctx.synchronize()
            torch.cuda.synchronize(device)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            launches0 = ctx.launch_count
            e0.record(stream)
            for _ in range(k):
                ctx.step(dev, p, state)
            e1.record(stream)
            ctx.synchronize()
            torch.cuda.synchronize(device)
            return e0.elapsed_time(e1) / k, ctx.launch_count - launches0

        results = {}
        # (name, precision, condition threshold of the FP64 route); the last
        # form is the headline.  The mixed form is also timed at the 1e6
        # threshold the splash workload names, beside the library default.
        default_kappa = args.kappa_threshold if args.kappa_threshold is not None else 1e4
        forms = [("plain", pkg.abi.PRECISION_PLAIN, default_kappa),
                 ("mixed_kappa1e6", pkg.abi.PRECISION_MIXED, 1e6),
                 ("mixed", pkg.abi.PRECISION_MIXED, default_kappa)]
        if args.precision != "both":
            forms = [f for f in forms if f[0] == args.precision]
        for form, prec, kappa in forms:
            ctx.set_precision(prec)
            ctx.set_condition_threshold(kappa)
            ctx.reserve(case.n_fluid, case.n_wall, case.n_cells)
            reset()
            fallbacks0 = ctx.fp64_fallbacks
            if args.knobs:  # fixed knobs apply from the first step on
                for k, v in enumerate(int(x) for x in args.knobs.split(",")):
                    ctx.set_knob(k, v)
            for _ in range(args.warmup):
                ctx.step(dev, p, state)
            # the project autotuner picks the launch-shape knobs on this state
            # (it runs only stages that are pure functions of the state)
            if args.knobs or args.no_autotune:
                tuned = {k: (ctx.knob(k), 0.0) for k in range(pkg.abi.KNOB_COUNT)}
            else:
                tuned = ctx.autotune(dev, p, repeats=3, state=state)
            ctx.synchronize()
            with ClockSampler(local) as sampler:
                ms, launches = timed_steps(args.steps)
            clocks = sampler.summary()
            ms_max = max_over_ranks(world, ms, device)
            kf = int(dev.fluid_neighbors["offsets"][case.n_fluid].item())
            kw_ = int(dev.wall_neighbors["offsets"][case.n_fluid].item())
            fallbacks = (ctx.fp64_fallbacks - fallbacks0) / max(1, args.warmup + args.steps)
            # per-kernel device time of the same steps (events around each launch)
            ctx.set_profiling(True)
            for _ in range(2):
                ctx.step(dev, p, state)
            prof = ctx.profile_report()
            ctx.set_profiling(False)
            results[form] = dict(ms=ms_max, launches=launches // args.steps, clocks=clocks, kf=kf, kw=kw_, prof=prof,
                                 fallbacks=fallbacks,
                                 autotune={KNOB_NAMES[k]: v for k, (v, _) in tuned.items()})

        # error of the mixed step against the plain FP64 step from the same
        # state, at full size (the parity tests pin the plain form to the FP64
        # oracle)
        error = None
        if "plain" in results and "mixed" in results:
            error = mixed_error(pkg, torch, ctx, dev, case, p, state, reset, default_kappa)

        # The headline form once more after renumbering the fluid in cell
        # order (lsmps_reorder_fluid + rebuild, as a driver would do once after
        # loading its input): the same particles and work, numbered so that
        # neighbours sit close in memory.  Reported beside the as-given value.
        renumbered = None
        if not args.no_renumbered:
            ctx.set_precision(forms[-1][1])
            ctx.set_condition_threshold(forms[-1][2])
            reset()
            ctx.set_synchronous(True)
            ctx.reorder_fluid(dev)
            ctx.build_neighbor_lists(dev, p)
            ctx.classify_surface(dev, p)
            ctx.set_synchronous(False)
            for _ in range(args.warmup):
                ctx.step(dev, p, state)
            ms_r, _ = timed_steps(args.steps)
            ms_r = max_over_ranks(world, ms_r, device)
            ctx.set_profiling(True)
            for _ in range(2):
                ctx.step(dev, p, state)
            prof_r = ctx.profile_report()
            ctx.set_profiling(False)
            renumbered = {"value": world * case.n_fluid / (ms_r * 1e-3), "ms_per_step": ms_r,
                          "kernels": [{"name": nm, "ms_per_step": t / 2, "launches_per_step": c // 2}
                                      for nm, t, c in prof_r],
                          "what": f"{forms[-1][0]} form after lsmps_reorder_fluid renumbered the fluid in cell order "
                                  "once at set-up (same particles and work; the as-given lattice numbering is the "
                                  "headline value)"}

        # end to end through the C ABI with host buffers: the particle state
        # lives in pinned host memory; every step copies it in, steps, and
        # copies the moved fluid state and labels back into the same host
        # buffers, which the next step copies in again.  So each step's
        # inputs are the previous step's outputs, consistent with the
        # neighbour tables and labels that step rebuilt on the device.  The
        # copies overlap the steps where their data dependences allow
        # (host_loop.HostResidentLoop: two device position buffers and the
        # library's step events).
        e2e = None
        if not args.no_e2e:
            host_loop = import_module("lsmps3d_b200.host_loop")
            ctx.set_precision(forms[-1][1])
            ctx.set_condition_threshold(forms[-1][2])
            reset()
            k_e2e = max(1, args.steps)  # the same step count as `value`
            loop = host_loop.HostResidentLoop(ctx, dev, p)
            loop.step()
            loop.sync()
            ctx.synchronize()
            torch.cuda.synchronize(device)
            barrier(world)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(k_e2e):
                loop.step()
            loop.sync()
            e1.record(stream)
            ctx.synchronize()
            torch.cuda.synchronize(device)
            loop.close()
            ms_e2e = max_over_ranks(world, e0.elapsed_time(e1) / k_e2e, device)
            e2e = {"value": world * case.n_fluid / (ms_e2e * 1e-3), "unit": "particles/s",
                   "h2d_bytes_per_step": loop.h2d_bytes, "d2h_bytes_per_step": loop.d2h_bytes,
                   "ms_per_step": ms_e2e, "steps": k_e2e,
                   "copies": "pinned host <-> device every step, overlapped with the steps where their data "
                             "dependences allow (two device position buffers, step events)"}
        # The same forms on the splash variant whose lifted 5% is scattered
        # off the lattice (sparse, ill-conditioned Surface/Splash matrices):
        # the generator's lattice-column splash holds none at 2M, so this is
        # where the mixed form's FP64 route runs at full size.
        scattered = None
        if not args.no_scattered and args.workload == "splash":
            case_s = pkg.cases.CASES["splash_scattered"]()
            p_s = case_s.params
            dev_s = api.device_buffers(case_s, device=device)
            state_s = dev_s.step_state(p_s)

            def reset_s():
                dev_s.load_case(case_s)
                ctx.set_synchronous(True)
                ctx.build_neighbor_lists(dev_s, p_s)
                ctx.classify_surface(dev_s, p_s)
                ctx.set_synchronous(False)

            timing = {}
            for form, prec, kappa in forms:
                ctx.set_precision(prec)
                ctx.set_condition_threshold(kappa)
                reset_s()
                for _ in range(args.warmup):
                    ctx.step(dev_s, p_s, state_s)
                ctx.synchronize()
                f0 = ctx.fp64_fallbacks
                k_s = max(1, min(args.steps, 5))
                barrier(world)
                torch.cuda.synchronize(device)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(k_s):
                    ctx.step(dev_s, p_s, state_s)
                e1.record(stream)
                ctx.synchronize()
                torch.cuda.synchronize(device)
                ms_s = max_over_ranks(world, e0.elapsed_time(e1) / k_s, device)
                timing[form] = {"ms_per_step": ms_s, "value": world * case_s.n_fluid / (ms_s * 1e-3),
                                "fp64_fallbacks_per_step": (ctx.fp64_fallbacks - f0) / k_s}
            err_s = None
            if "plain" in timing and "mixed" in timing:
                err_s = mixed_error(pkg, torch, ctx, dev_s, case_s, p_s, state_s, reset_s, default_kappa)
            scattered = {"workload": "splash dam break 200x50x200 (2M fluid) with the lifted 5% scattered uniformly "
                                     "over the tank floor plan, 0-10 l0 above the free surface (seed 3)",
                         "forms": timing, "error": err_s}
            del dev_s, state_s
        ctx.close()

    head_form = forms[-1][0]
    h = results[head_form]
    peak_s, _ = peaks()
    peak, peak_kind = peaks()
    kb = roofline.kernel_bytes(case.n_fluid, case.n_wall, h["kf"], h["kw"], case.n_cells)
    top = max(h["prof"], key=lambda e: e[1]) if h["prof"] else ("", 0.0, 1)
    total_prof = sum(e[1] for e in h["prof"]) or 1.0
    top_name, top_ms, top_n = top
    avg_ms = top_ms / max(top_n, 1)
    alg = kb.get(top_name)
    achieved = alg / (avg_ms * 1e-3) / 1e9 if alg and avg_ms > 0 else None
    traffic, traffic_source = measured_traffic(top_name, case.n_fluid)
    step_b = roofline.step_bytes(case.n_fluid, case.n_wall, h["kf"], h["kw"], case.n_cells)
    out = {
        "metric": METRIC,
        "value": world * case.n_fluid / (h["ms"] * 1e-3),
        "unit": "particles/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": h["ms"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if head_form == "plain" else "f32+f64 (mixed)",
        "data": "synthetic",
        "config": {
            "workload": desc,
            "n_fluid": case.n_fluid,
            "n_wall": case.n_wall,
            "cells": case.n_cells,
            "csr_fluid_entries": h["kf"],
            "csr_wall_entries": h["kw"],
            "precision": head_form,
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "working set per step > 10 GB, far larger than the 126 MB L2 (no flush needed)",
        },
        "roofline": {
            "bound": "hbm",
            "kernel": top_name,
            "kernel_share_of_step": top_ms / total_prof,
            "achieved": achieved,
            "peak": peak,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
            "unit": "GB/s",
            "frac": achieved / peak if achieved else None,
            "traffic": traffic,
            "traffic_source": traffic_source,
            "algorithmic_bytes": alg,
            "step_bytes_model": step_b,
            "step_hbm_frac": step_b / (h["ms"] * 1e-3) / 1e9 / peak,
        },
        "forms": {
            f: {"value": world * case.n_fluid / (r["ms"] * 1e-3), "ms_per_step": r["ms"],
                "fp64_fallbacks_per_step": r["fallbacks"], "autotune": r["autotune"],
                "step_hbm_frac": roofline.step_bytes(case.n_fluid, case.n_wall, r["kf"], r["kw"], case.n_cells)
                / (r["ms"] * 1e-3) / 1e9 / peak_s,
                "kernels": [{"name": n, "ms_per_step": ms / 2, "launches_per_step": c // 2}
                            for n, ms, c in r["prof"]]}
            for f, r in results.items()},
        "mixed_over_plain": (results["plain"]["ms"] / results["mixed"]["ms"])
        if "plain" in results and "mixed" in results else None,
        "error": error,
        "kernels": [{"name": n, "ms_per_step": ms / 2, "launches_per_step": c // 2} for n, ms, c in h["prof"]],
        "gpu_launches": h["launches"] * args.steps,
        "clocks": h["clocks"],
        "e2e": e2e,
        "renumbered": renumbered,
        "scattered_splash": scattered,
    }
    return out, case


def run_batched(args, world, rank, local):
    """64 independent boxes stepped by one captured CUDA graph: merged (all
    boxes as one particle set; the headline, mixed form) and one step per box
    on 8 worker streams; and the same boxes stepped one after another by
    lsmps_step with no graph; each in both precision forms (the project
    autotuner sets the knobs of each graph)."""
    import torch

    pkg = graft_entry.load_package()
    from importlib import import_module

    import_module("lsmps3d_b200.build").build_all()
    api = import_module("lsmps3d_b200.api")
    partition = import_module("lsmps3d_b200.partition")
    device = torch.device(f"cuda:{local}")
    torch.cuda.set_device(device)
    all_boxes = pkg.cases.batched_boxes()
    # With N GPUs the boxes are split by size over the ranks (no data-path
    # collective); each rank steps its share.
    mine = partition.partition_boxes([c.n_fluid for c in all_boxes], world)[rank]
    boxes = [all_boxes[k] for k in mine]
    setup_stream = torch.cuda.Stream(device)
    n_total = sum(c.n_fluid for c in boxes)
    bufs = []
    with torch.cuda.stream(setup_stream):
        ctx = api.Context(local)
        for case in boxes:
            b = api.device_buffers(case, device=device)
            ctx.build_neighbor_lists(b, case.params)
            ctx.classify_surface(b, case.params)
            bufs.append((b, case.params, b.step_state(case.params)))
        ctx.set_synchronous(False)
        ctx.reserve(max(c.n_fluid for c in boxes), max(c.n_wall for c in boxes), max(c.n_cells for c in boxes))

        def sequential(prec):
            ctx.set_precision(prec)
            for b, p, st in bufs:
                ctx.step(b, p, st)
            ctx.synchronize()
            torch.cuda.synchronize(device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(setup_stream)
            for b, p, st in bufs:
                ctx.step(b, p, st)
            e1.record(setup_stream)
            ctx.synchronize()
            torch.cuda.synchronize(device)
            return e0.elapsed_time(e1)

        seq = {"plain": sequential(pkg.abi.PRECISION_PLAIN), "mixed": sequential(pkg.abi.PRECISION_MIXED)}
        ctx.close()

    def graph(prec, steps, sample, merged=True):
        batch = api.Batch(local, streams=8)
        batch.set_merged(merged)
        for b, p, _ in bufs:
            batch.add(b, p)
        batch.capture(precision=prec, autotune_repeats=2)
        assert batch.merged == merged
        stream = torch.cuda.ExternalStream(batch.stream, device=device)
        for _ in range(args.warmup):
            batch.launch()
        batch.synchronize()
        barrier(world)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(local) if sample else None
        if sampler:
            sampler.__enter__()
        e0.record(stream)
        for _ in range(steps):
            batch.launch()
        e1.record(stream)
        batch.synchronize()
        torch.cuda.synchronize(device)
        if sampler:
            sampler.__exit__(None, None, None)
        batch.close()
        return e0.elapsed_time(e1) / steps, (sampler.summary() if sampler else None)

    plain_ms, _ = graph(pkg.abi.PRECISION_PLAIN, max(1, args.steps // 2), False)
    streams_mixed_ms, _ = graph(pkg.abi.PRECISION_MIXED, max(1, args.steps // 2), False, merged=False)
    streams_plain_ms, _ = graph(pkg.abi.PRECISION_PLAIN, max(1, args.steps // 2), False, merged=False)
    mixed_ms, clocks = graph(pkg.abi.PRECISION_MIXED, args.steps, True)
    # whole job: particles summed over ranks, time the slowest rank's
    n_job, ms = partition.reduce_rank_results(world, n_total, mixed_ms, device)
    value = n_job / (ms * 1e-3)

    def rate(ms_):
        return {"value": n_total / (ms_ * 1e-3), "ms_per_pass": ms_}

    return {
        "metric": METRIC,
        "value": value,
        "unit": "particles/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32+f64 (mixed)",
        "data": "synthetic",
        "config": {"workload": WORKLOADS["batched"][2], "boxes": len(all_boxes), "boxes_rank0": len(boxes),
                   "n_fluid_total": n_job,
                   "n_wall_total": sum(c.n_wall for c in boxes), "graph_streams": 8,
                   "precision": "mixed (headline); every combination below",
                   "parallelism": f"boxes split over {world} GPUs by size" if world > 1 else "single GPU"},
        "graph": {"mixed": rate(mixed_ms), "plain": rate(plain_ms),
                  "what": "merged form: all boxes as one particle set, one launch per stage over every box"},
        "graph_per_box_streams": {"mixed": rate(streams_mixed_ms), "plain": rate(streams_plain_ms),
                                  "what": "one lsmps_step per box on 8 worker streams"},
        "sequential": {"mixed": rate(seq["mixed"]), "plain": rate(seq["plain"]),
                       "what": "the same 64 boxes stepped one after another with lsmps_step, no graph"},
        "graph_over_sequential": {"mixed": seq["mixed"] / mixed_ms, "plain": seq["plain"] / plain_ms},
        "clocks": clocks,
        "e2e": None,
        "gpu_launches": None,
    }


def run_reorder(args, world, rank, local):
    """The splash step on input whose fluid numbering does not follow space,
    then after one lsmps_reorder_fluid (renumbering in cell order) and a
    neighbour rebuild; plain form, default knobs."""
    import torch

    pkg = graft_entry.load_package()
    from importlib import import_module

    import_module("lsmps3d_b200.build").build_all()
    api = import_module("lsmps3d_b200.api")
    device = torch.device(f"cuda:{local}")
    kind, kw, desc = WORKLOADS[args.workload]
    case = pkg.cases.CASES[kind](**kw)
    p = case.params
    stream = torch.cuda.Stream(device)
    out = {}
    with torch.cuda.stream(stream):
        dev = api.device_buffers(case, device=device)
        ctx = api.Context(local)
        ctx.reserve(case.n_fluid, case.n_wall, case.n_cells)
        state = dev.step_state(p)
        ctx.build_neighbor_lists(dev, p)
        ctx.classify_surface(dev, p)
        ctx.set_synchronous(False)

        def timed(k):
            for _ in range(args.warmup):
                ctx.step(dev, p, state)
            ctx.synchronize()
            barrier(world)
            torch.cuda.synchronize(device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            launches0 = ctx.launch_count
            e0.record(stream)
            for _ in range(k):
                ctx.step(dev, p, state)
            e1.record(stream)
            ctx.synchronize()
            torch.cuda.synchronize(device)
            return max_over_ranks(world, e0.elapsed_time(e1) / k, device), ctx.launch_count - launches0

        with ClockSampler(local) as s0:
            ms_shuffled, _ = timed(args.steps)
        ctx.set_synchronous(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.reorder_fluid(dev)
        ctx.build_neighbor_lists(dev, p)
        e1.record(stream)
        torch.cuda.synchronize(device)
        ms_reorder = e0.elapsed_time(e1)
        ctx.set_synchronous(False)
        with ClockSampler(local) as s1:
            ms_sorted, launches = timed(args.steps)
        ctx.close()
    n = case.n_fluid
    return {
        "metric": METRIC,
        "value": world * n / (ms_sorted * 1e-3),
        "unit": "particles/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_sorted,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": desc, "n_fluid": n, "n_wall": case.n_wall, "precision": "plain",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "without_reorder": {"value": world * n / (ms_shuffled * 1e-3), "ms_per_step": ms_shuffled,
                            "clocks": s0.summary()},
        "reorder_and_rebuild_ms": ms_reorder,
        "gpu_launches": launches,
        "clocks": s1.summary(),
        "e2e": None,
    }


def run_stage(args, world, rank, local):
    """A stage outside the benchmark step, on the state one plain step leaves:
    the virtual-light diagnostic (lsmps_virtual_light) or the PPE solve
    (lsmps_solve_ppe on the step's assembled rows, from zero each time)."""
    import torch

    pkg = graft_entry.load_package()
    from importlib import import_module

    import_module("lsmps3d_b200.build").build_all()
    api = import_module("lsmps3d_b200.api")
    roofline = import_module("lsmps3d_b200.roofline")
    device = torch.device(f"cuda:{local}")
    kind, kw, desc = WORKLOADS[args.workload]
    if args.stage_case != "splash":
        kind, kw = args.stage_case, WORKLOADS[args.stage_case][1]
        desc = desc.replace("splash dam break 200x50x200 (2M fluid)", WORKLOADS[args.stage_case][2]).replace(
            "splash dam break 200x50x200 (2M rows)", WORKLOADS[args.stage_case][2])
    case = pkg.cases.CASES[kind](**kw)
    p = case.params
    stream = torch.cuda.Stream(device)
    n = case.n_fluid
    with torch.cuda.stream(stream):
        dev = api.device_buffers(case, device=device)
        ctx = api.Context(local)
        ctx.reserve(case.n_fluid, case.n_wall, case.n_cells)
        state = dev.step_state(p)
        ctx.build_neighbor_lists(dev, p)
        ctx.classify_surface(dev, p)
        ctx.step(dev, p, state)
        kf = int(dev.fluid_neighbors["offsets"][n].item())
        kw_ = int(dev.wall_neighbors["offsets"][n].item())
        nnz = int(dev.ppe["row_offsets"][n].item())
        if args.workload == "virtual_light":
            count = torch.empty(n, dtype=torch.int32, device=device)
            frac = torch.empty(n, dtype=torch.float64, device=device)

            def call():
                ctx.virtual_light(dev, p, count.data_ptr(), frac.data_ptr())
        else:
            x = torch.empty(n, dtype=torch.float64, device=device)
            v = dev.ppe_view()
            opt = pkg.abi.default_solver_options()
            reports = []

            def call():
                reports.append(ctx.solve_csr(v.matrix, v.rhs, x.data_ptr(), opt))
        for _ in range(args.warmup):
            call()
        ctx.synchronize()
        barrier(world)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = ctx.launch_count
        with ClockSampler(local) as sampler:
            e0.record(stream)
            for _ in range(args.steps):
                call()
            e1.record(stream)
            ctx.synchronize()
            torch.cuda.synchronize(device)
        launches = ctx.launch_count - launches0
        ms = max_over_ranks(world, e0.elapsed_time(e1) / args.steps, device)
        ctx.set_profiling(True)
        call()
        prof = ctx.profile_report()
        ctx.set_profiling(False)
        ctx.close()
    peak, peak_kind = peaks()
    if args.workload == "virtual_light":
        kb = roofline.kernel_bytes(n, case.n_wall, kf, kw_, case.n_cells)
        value, unit = world * n / (ms * 1e-3), "particles/s"
        extra = {}
    else:
        kb = roofline.solve_kernel_bytes(n, nnz, restart=opt.restart)
        value, unit = world / (ms * 1e-3), "solves/s"
        r = reports[-1]
        extra = {"solver": {"iterations": r.iterations, "converged": bool(r.converged),
                            "residual_reduction": r.final_residual / r.initial_residual if r.initial_residual else 0.0,
                            "ms_per_iteration": ms / max(r.iterations, 1), "rows": n, "nnz": nnz}}
    top_name, top_ms, top_n = max(prof, key=lambda e: e[1])
    avg_ms = top_ms / max(top_n, 1)
    alg = kb.get(top_name)
    achieved = alg / (avg_ms * 1e-3) / 1e9 if alg else None
    traffic, traffic_source = measured_traffic(top_name, n)
    out = {
        "metric": STAGE_METRICS[args.workload],
        "value": value,
        "unit": unit,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": desc, "n_fluid": n, "n_wall": case.n_wall, "csr_fluid_entries": kf,
                   "csr_wall_entries": kw_, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs larger than the 126 MB L2 (no flush needed)"},
        "roofline": {"bound": "hbm", "kernel": top_name,
                     "kernel_share": top_ms / (sum(e[1] for e in prof) or 1.0), "achieved": achieved, "peak": peak,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else "fallback", "unit": "GB/s", "frac": achieved / peak if achieved else None,
                     "traffic": traffic, "traffic_source": traffic_source, "algorithmic_bytes": alg},
        "kernels": [{"name": k, "ms": t, "launches": c} for k, t, c in prof],
        "gpu_launches": launches,
        "clocks": sampler.summary(),
        "e2e": None,
    }
    out.update(extra)
    return out


def mixed_error(pkg, torch, ctx, dev, case, p, state, reset, default_kappa):
    """Errors of the mixed step against the plain FP64 step from the same
    moving state (the workload's positions and labels with the swirl
    velocity u = 0.1 (sin(x/L), cos(y/L), z/L) m/s, L the fluid extent, so
    that the velocity Laplacian and the PPE divergence are not zero), at the
    library's default condition threshold and at 1e6; plus the statistics
    of the state that decide the FP64 route: neighbour counts, labels and
    the condition number of the moment matrices by label."""
    f = case.fluid
    span = max(float(f[k].max() - f[k].min()) for k in ("x", "y", "z"))

    def moving_state():
        reset()
        dev.fluid["vx"].copy_(0.1 * torch.sin(dev.fluid["x"] / span))
        dev.fluid["vy"].copy_(0.1 * torch.cos(dev.fluid["y"] / span))
        dev.fluid["vz"].copy_(0.1 * dev.fluid["z"] / span)

    def run(prec, kappa):
        ctx.set_precision(prec)
        ctx.set_condition_threshold(kappa)
        moving_state()
        f0 = ctx.fp64_fallbacks
        ctx.step(dev, p, state)
        ctx.synchronize()
        out = {k: v.clone() for k, v in dev.ppe.items() if k in ("values", "rhs", "divergence", "pressure_laplacian")}
        out["row_offsets"] = dev.ppe["row_offsets"].clone()
        for k in ("x", "y", "z", "vx", "vy", "vz", "pressure"):
            out["f_" + k] = dev.fluid[k].clone()
        for k in ("x", "y", "z"):
            out["g_" + k] = dev.pressure_gradient[k].clone()
            out["l_" + k] = dev.velocity_laplacian[k].clone()
        out["fallbacks"] = ctx.fp64_fallbacks - f0
        return out

    # statistics of the state (labels and rows before the step)
    moving_state()
    labels = dev.fluid["surface_type"].clone().long()
    fo = dev.fluid_neighbors["offsets"]
    wo = dev.wall_neighbors["offsets"]
    counts = ((fo[1:] - fo[:-1]) + (wo[1:] - wo[:-1])).long()
    edges = [0, 1, 5, 10, 20, 40, 60, 80, 100, 120, 140, 100000]
    hist = [int(((counts >= lo) & (counts < hi)).sum()) for lo, hi in zip(edges[:-1], edges[1:])]
    ref = run(pkg.abi.PRECISION_PLAIN, default_kappa)
    kappa_stats = {}
    names = {0: "inner", 1: "near_surface", 2: "surface", 3: "splash"}
    for kind, kname in ((0, "velocity"), (1, "pressure")):
        m = dev.moments[kind]
        inv = m["inverse_matrices"].view(-1, 81)
        kap = (m["moment_trace"] + 9.0 * m["regularization_added"]) * inv.pow(2).sum(1).sqrt()
        per = {}
        for lab, lname in names.items():
            sel = labels == lab
            cnt = int(sel.sum())
            if cnt == 0:
                per[lname] = {"count": 0}
                continue
            k_ = kap[sel]
            per[lname] = {"count": cnt, "median": float(k_.median()), "max": float(k_.max()),
                          "above_1e4": int((k_ > 1e4).sum()), "above_1e6": int((k_ > 1e6).sum())}
        kappa_stats[kname] = per
        del inv, kap
    out = {
        "state": "the workload's positions and labels with the swirl velocity u = 0.1 (sin(x/L), cos(y/L), z/L) m/s",
        "reference": "this library's plain FP64 step from the same state (the plain form is held to the FP64 "
                     "oracle by the parity tests)",
        "neighbour_count_histogram": {"edges": edges, "counts": hist, "min": int(counts.min()),
                                      "max": int(counts.max())},
        "labels": {names[k]: int((labels == k).sum()) for k in names},
        "kappa_estimate": "(trace M) ||M^-1||_F of the plain step's inverses (an upper bound of kappa_2 within a "
                          "factor 27)",
        "kappa_by_label": kappa_stats,
        "target": "PPE coefficients <= 1e-5",
        "thresholds": {},
    }
    off = ref["row_offsets"].long()
    n = off.numel() - 1
    nnz = int(off[-1].item())
    lengths = off[1:] - off[:-1]
    row = torch.repeat_interleave(torch.arange(n, device=off.device), lengths)
    a = ref["values"][:nnz].abs()
    amax = torch.zeros(n, dtype=a.dtype, device=a.device).scatter_reduce(0, row, a, "amax")
    floor = 1e-4 * float(a.max())

    def norm_err(mix, keys):
        num = max(float((mix[k] - ref[k]).abs().max()) for k in keys)
        den = max(float(ref[k].abs().max()) for k in keys)
        return num / den if den > 0 else num

    for kappa in (default_kappa, 1e6):
        mix = run(pkg.abi.PRECISION_MIXED, kappa)
        d = (mix["values"][:nnz] - ref["values"][:nnz]).abs()
        dmax = torch.zeros(n, dtype=d.dtype, device=d.device).scatter_reduce(0, row, d, "amax")
        rowwise = float(torch.where(amax > 0, dmax / torch.where(amax > 0, amax, torch.ones_like(amax)), dmax).max())
        per_coef = float((d / torch.clamp(a, min=floor)).max())
        per_coef_2 = float((d / torch.clamp(a, min=100.0 * floor)).max())
        out["thresholds"][f"{kappa:.0e}"] = {
            "fp64_route_matrices": int(mix["fallbacks"]),
            "ppe_coefficients_max_rel_per_coefficient": per_coef,
            "ppe_coefficients_floor": f"|a_ij| below 1e-4 of the largest |a_ij| ({floor:.3e}) counts as that floor",
            "ppe_coefficients_max_rel_per_coefficient_floor_1e-2": per_coef_2,
            "ppe_coefficients_max_rel_rowwise": rowwise,
            "ppe_rhs_rel": norm_err(mix, ["rhs"]),
            "ppe_divergence_rel": norm_err(mix, ["divergence"]),
            "pressure_gradient_rel": norm_err(mix, ["g_x", "g_y", "g_z"]),
            "velocity_laplacian_rel": norm_err(mix, ["l_x", "l_y", "l_z"]),
            "velocity_rel": norm_err(mix, ["f_vx", "f_vy", "f_vz"]),
            "position_rel": norm_err(mix, ["f_x", "f_y", "f_z"]),
        }
        del mix, d, dmax
    ctx.set_precision(pkg.abi.PRECISION_MIXED)
    ctx.set_condition_threshold(default_kappa)
    del row, a, amax
    return out


def cpu_baseline(case_kind: str):
    """The OpenMP oracle step on a bounded sample of the workload: the
    200 x 50 x 50 bottom slab of the same lattice for the splash dam break
    (500k particles), the full case for the smaller workloads."""
    import numpy as np

    pkg = graft_entry.load_package()
    orc_mod = graft_entry.load_oracle()
    orc = orc_mod.Oracle(pkg.abi)
    if case_kind == "splash":
        case = pkg.cases.splash_dam_break(nz=50)
        sample = "one oracle step on the 200x50x50 slab (500k fluid) of the same splash dam-break lattice"
    elif case_kind == "dam_break":
        case = pkg.cases.dam_break(nz=25)
        sample = "one oracle step on the 100x50x25 slab (125k fluid) of the same dam-break lattice"
    else:
        case = pkg.cases.hydrostatic_box()
        sample = "one oracle step on the full 20^3 hydrostatic box"
    b = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells,
                                max_fluid_neighbors=160, max_wall_neighbors=64)
    b.load_case(case)
    orc.build_neighbor_lists(b, case.params)
    orc.classify_surface(b, case.params)
    t0 = time.perf_counter()
    st, _ = orc.step(b, case.params)
    dt = time.perf_counter() - t0
    return {"value": case.n_fluid / dt if st == 0 else None, "unit": "particles/s", "cores": orc.max_threads(),
            "kind": "port", "sample": sample, "seconds": dt}


def run_reference(args, world, rank, local):
    """The reference's own CUDA path (built from its sources into oracle/_ref)
    through its public C++ module API, timed per step with CUDA events."""
    pkg = graft_entry.load_package()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference as ref_mod

    kind, kw, desc = WORKLOADS[args.workload]
    base = {"metric": METRIC, "unit": "particles/s", "impl": "reference", "higher_is_better": True}
    if kind == "batched":
        return dict(impl="reference", unavailable="the reference steps one box per process; it has no batched form")
    if args.workload == "ppe_solve":
        return dict(impl="reference", unavailable="the reference solves the PPE with AMGX, a third-party library that "
                                                  "is not installed here; its build without AMGX has no solve")
    if not ref_mod.available():
        return dict(impl="reference", unavailable="oracle/_ref/libref_lsmps.so was not built (needs the reference sources)")
    case = pkg.cases.CASES[kind](**kw)
    b = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells,
                                fluid_capacity=1, wall_capacity=1)
    b.load_case(case)
    ref = ref_mod.ReferencePath(pkg.abi, case, b)
    ref.rebuild()
    if args.workload == "virtual_light":
        base["metric"] = STAGE_METRICS["virtual_light"]
        ref.steps(1)  # the same state as our arm: one step after the first rebuild
        if args.warmup:
            ref.virtual_light_steps(args.warmup)
        with ClockSampler(local) as sampler:
            ms = ref.virtual_light_steps(args.steps)
    else:
        if args.warmup:
            ref.steps(args.warmup)
        with ClockSampler(local) as sampler:
            ms = ref.steps(args.steps)
    clocks = sampler.summary()
    ref.close()
    mean_ms = sum(ms) / len(ms)
    value = case.n_fluid / (mean_ms * 1e-3)
    base.update({
        "value": value,
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": mean_ms,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": desc, "n_fluid": case.n_fluid, "n_wall": case.n_wall, "cells": case.n_cells,
                   "precision": "plain (reference real = double)", "parallelism": "single GPU"},
        "cpu_baseline": {"value": value, "unit": "particles/s", "cores": 1, "kind": "reference",
                         "sample": "the reference's CUDA path (oracle/_ref, built from its sources for sm_100a) on "
                                   "the full workload; one host thread drives it"},
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clocks,
        "per_step_ms": ms,
    })
    return base


def main():
    args = parse_args()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, world, rank, local)), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    if args.workload in STAGE_METRICS or args.workload == "splash_shuffled":
        out = (run_stage if args.workload in STAGE_METRICS else run_reorder)(args, world, rank, local)
        if rank == 0:
            print(json.dumps(out), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    if args.workload == "batched":
        out = run_batched(args, world, rank, local)
        if rank == 0:
            print(json.dumps(out), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    out, case = run_ours(args, world, rank, local)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(WORKLOADS[args.workload][0])
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
