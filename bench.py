#!/usr/bin/env python3
"""Benchmark of the B200 dycore: cell-steps/s of the order-9 WENO SSPRK3
dynamical core on the neutral boundary-layer workload (256x256x128, dx=10 m,
tracers water_vapor + TKE), one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value: K SSPRK3 steps of the resident FP32 state, timed with CUDA events
  on the dycore's stream between a barrier and a device synchronize on both
  sides, max over ranks; the state (>= 0.9 GB) is larger than L2.
* e2e: the reference-facing call (pu_dycore_time_step, dt_phys = 10 dycore
  steps as the reference's drivers use, abl_neutral.cpp:25) with the coupler
  arrays in pinned host memory: host->device copy, conversion, 10 SSPRK3
  steps, conversion back and device->host copy inside every timed call.
* roofline: the x/y flux kernel (the larger share of the step), its
  algorithmic bytes per launch over its CUDA-event duration in the timed
  region; traffic from the committed ncu capture (profiles/).
* cpu_baseline: the reference's own dycore code (oracle/_ref, built from the
  reference's headers with a single-rank shim) on all host cores, on a
  bounded sample of the same workload.
* learned: the learned-weight form on the same state and timed region,
  after harvesting 2^21 stencils from it and training the network on the GPU
  (3000 Adam steps, batch 16384); kernel times and the fallback fraction.
* physics: the modules the boundary-layer driver runs beside the dycore
  every dt_phys (geostrophic forcing, sponge, surface fluxes, LES closure;
  FP64 as the reference) on device coupler arrays of the same workload.
* Multi-GPU: the dycore is not domain-decomposed here; N ranks run N
  independent replicas (ensemble members) with no collective in the data
  path (weak scaling).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "source": "fallback"}
WORKLOAD = dict(nx=256, ny=256, nz=128, dx=10.0)
DYN_CYCLE = 10
LEARNED_THRESHOLD = 0.5


def decomposed_tiles(case, world, steps, warmup, grid=(2, 2)):
    """The same workload as a grid of tiles of one process on this GPU
    (pu_dycore_group_*: per stage a pack of the 5-cell halo slabs, device
    copies between the tiles, the x/y kernel reading them): the cost of the
    decomposed path without the interconnect."""
    import torch
    from porturb_b200 import decomp
    grp = decomp.TileGroup(case, *grid, precision="f32")
    grp.init_case(perturbed=False)
    for h, c in zip(grp.handles, grp.cases):
        rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in c.coupler_arrays(perturbed=True)]
        h.load_state(rd, u, v, w, T, [np.ascontiguousarray(x) for x in trc])
    dt = grp.handles[0].compute_time_step()
    grp.advance(dt, warmup)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    grp.advance(dt, steps)
    ev1.record()
    torch.cuda.synchronize()
    ms = reduce_max(ev0.elapsed_time(ev1), world)
    grp.close()
    return {"tiles": "%dx%d" % grid, "value": aggregate_value(case.ncells, steps, ms / 1e3, world),
            "unit": "cell-steps/s", "ms_per_step": ms / steps,
            "note": "tiles of one process on the legacy default stream: halo slabs packed and copied on the device "
                    "every stage, no interconnect"}


def physics_modules(case, stream, world, reps=10):
    """The modules the boundary-layer driver runs beside the dycore every
    dt_phys (geostrophic forcing, sponge, surface fluxes, LES closure, time
    averager) on
    device coupler arrays of the same workload: CUDA-event time per call and,
    for the LES kernel (the out-of-place form, no copy-back), algorithmic
    HBM bytes over its time."""
    import torch
    from porturb_b200.physics import Physics
    ph = Physics.from_case(case, stream=stream.cuda_stream, device=torch.cuda.current_device())
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=True)]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    A = [dev(x) for x in (rd, u, v, w, T)]
    At = [dev(trc[t]) for t in range(trc.shape[0])]
    B = [torch.empty_like(x) for x in A]
    Bt = [torch.empty_like(x) for x in At]
    dt = 0.1
    N = case.ncells
    nd = sum(1 for t in case.tracers if t.diffuse and t.name != "TKE")
    out = {}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        ph.les_to(tuple(A) + (At,), tuple(B) + (Bt,), dt)
    ph.synchronize()
    les_ms = []
    for _ in range(reps):
        ph.les_to(tuple(A) + (At,), tuple(B) + (Bt,), dt)
        les_ms.append(ph.last_les_ms())
    les_ms = reduce_max(float(np.median(les_ms)), world)
    # read rho_d, u, v, w, T, TKE, diffused tracers and the immersed proportion;
    # write u, v, w, T, TKE, diffused tracers (FP64)
    les_bytes = 8.0 * N * ((7 + nd) + (5 + nd))
    out["les_kernel_ms"] = les_ms
    out["les_gbs"] = les_bytes / (les_ms / 1e3) / 1e9
    calls = (("les", (dt,)), ("sponge", (dt, 100 * dt, 300.0 / case.zlen)),
             ("geostrophic", (dt, 43.29, 10.0, 0.0)), ("surface_fluxes", (dt,)))
    for name, args in calls:
        getattr(ph, name)(*A, At, *args)
        ph.synchronize()
        ev0.record(stream)
        for _ in range(reps):
            getattr(ph, name)(*A, At, *args)
        ev1.record(stream)
        torch.cuda.synchronize()
        out[name + "_ms"] = reduce_max(ev0.elapsed_time(ev1) / reps, world)
    # The time averager: reads u, v, w, TKE, reads and writes the 13 averages.
    avgs = [torch.zeros_like(A[1]) for _ in range(13)]
    etime = ph.time_average(*A, At, avgs, 0.0, 0.0, dt)
    ph.synchronize()
    ev0.record(stream)
    for r in range(reps):
        etime = ph.time_average(*A, At, avgs, etime, dt * (r + 1), dt)
    ev1.record(stream)
    torch.cuda.synchronize()
    out["time_averager_ms"] = reduce_max(ev0.elapsed_time(ev1) / reps, world)
    out["time_averager_gbs"] = 8.0 * N * (4 + 2 * 13) / (out["time_averager_ms"] / 1e3) / 1e9
    out["dtype"] = "f64"
    out["note"] = ("les_ms includes the copy-back of the in-place call; les_kernel_ms is the fused kernel alone; "
                   "FP64 pow/sqrt/division bound, not HBM bound")
    ph.close()
    return out


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        d["source"] = "measured"
        return d
    return dict(PEAKS_FALLBACK)


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_case(seed=0):
    from porturb_b200 import cases
    return cases.abl_neutral(nx=WORKLOAD["nx"], ny=WORKLOAD["ny"], nz=WORKLOAD["nz"], dx=WORKLOAD["dx"], seed=seed)


def workload_name():
    w = WORKLOAD
    return "abl_neutral %dx%dx%d dx=%gm, water_vapor+TKE tracers, WENO order 9, SSPRK3" % (
        w["nx"], w["ny"], w["nz"], w["dx"])


def cpu_sample_case():
    """The bounded CPU sample: the same boundary-layer configuration on a
    64x64 column block of the full 128 levels (same spacing and profile)."""
    from porturb_b200 import cases
    return cases.abl_neutral(nx=64, ny=64, nz=WORKLOAD["nz"], dx=WORKLOAD["dx"], seed=0)


def cpu_reference_rate(steps=1, warmup=1):
    """Cell-steps/s of the reference's own dycore code on the host cores
    (oracle/_ref); falls back to this project's REF restatement if the
    reference library was not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    kind = "reference" if pyoracle.have_ref() else "ref"
    case = cpu_sample_case()
    d = pyoracle.Dycore(case, kind)
    d.init_case()
    d.load_coupler(list(case.coupler_arrays(perturbed=True)))
    dt = d.compute_time_step()
    for _ in range(warmup):
        d.advance(dt, 1)
    t0 = time.perf_counter()
    d.advance(dt, steps)
    el = time.perf_counter() - t0
    import ctypes
    lib = pyoracle._lib(pyoracle.ORACLE_SO, "orc_")
    threads = int(lib.orc_num_threads())
    return {"value": case.ncells * steps / el, "unit": "cell-steps/s", "cores": threads,
            "kind": "reference" if kind == "reference" else "port",
            "sample": "%d SSPRK3 step(s) of abl_neutral on a %dx%dx%d block (same dx and profile), "
                      "after %d warm-up step(s), %.1f s" % (steps, case.nx, case.ny, case.nz, warmup, el)}


def setup_dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_max(x, world, device="cuda"):
    """Max of a per-rank scalar over all ranks (the timing rule: the job is as
    slow as its slowest rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_value(cells_per_rank, steps, seconds_max, world):
    """Whole-job throughput: every rank advanced its own replica of the
    workload, so the job processed world*cells*steps cell-steps in the time of
    the slowest rank."""
    return world * cells_per_rank * steps / seconds_max


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    base = cpu_reference_rate(steps=max(1, args.steps // 10), warmup=1)
    line = {"impl": "reference", "metric": "cell-steps/s", "value": base["value"], "unit": "cell-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64-state/f32-stencil", "data": "synthetic",
            "config": {"workload": workload_name(), "sample": base["sample"]},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-calls", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-physics", action="store_true")
    ap.add_argument("--no-decomposed", action="store_true")
    args = ap.parse_args()
    world, rank, local = setup_dist()
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return

    import torch
    import torch.distributed as dist
    from porturb_b200 import Dycore, build
    build.build()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    case = build_case(seed=rank)
    stream = torch.cuda.Stream(device=local)
    g = Dycore.from_case(case, precision="f32", device=local, stream=stream.cuda_stream)
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=False)]
    g.init(rd, u, v, w, T, list(trc), None)
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=True)]
    g.load_state(rd, u, v, w, T, list(trc))
    dt = g.compute_time_step()
    N = case.ncells
    S = 5 + len(case.tracers)

    # Warm-up, then the timed region.
    for _ in range(args.warmup):
        g.advance(dt, 1)
    g.synchronize()
    clocks = ClockSampler(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    launches0 = g.kernel_launches()
    ev0.record(stream)
    for _ in range(args.steps):
        g.advance(dt, 1)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = g.kernel_launches() - launches0
    # Per-kernel CUDA events on the launching stream, in a second pass of the
    # same number of steps: an event pair around every launch costs ~1.7 % of
    # the step, so the headline region above runs without them.
    g.profile(True)
    for _ in range(args.steps):
        g.advance(dt, 1)
    prof = g.profile_read()
    g.profile(False)
    clk = clocks.stop()
    barrier(world)
    g.synchronize()
    ms = reduce_max(ev0.elapsed_time(ev1), world)
    value = aggregate_value(N, args.steps, ms / 1e3, world)

    # e2e through the C-ABI with pinned host coupler arrays.
    shp = (case.nz, case.ny, case.nx)
    pinned = [torch.empty(shp, dtype=torch.float64).pin_memory() for _ in range(5)]
    ptrc = [torch.empty(shp, dtype=torch.float64).pin_memory() for _ in range(len(case.tracers))]
    g.store_state(*pinned, ptrc)
    dt_phys = DYN_CYCLE * dt
    g.time_step(*pinned, ptrc, dt_phys)   # warm-up call
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ncyc = 0
    for _ in range(args.e2e_calls):
        ncyc += g.time_step(*pinned, ptrc, dt_phys)
    torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t0, world)
    e2e_value = aggregate_value(N, ncyc, e2e_s, world)
    bytes_io = (5 + len(case.tracers)) * N * 8

    # Learned-weight form: network trained on stencils harvested from this
    # run's own state (GPU training kernels), then the same timed region.
    physics = None if args.no_physics else physics_modules(case, stream, world)
    decomposed = None if args.no_decomposed else decomposed_tiles(case, world, min(args.steps, 10), args.warmup)

    learned = None
    if not args.no_learned:
        g.learned_harvest(1 << 21, seed=1 + rank)
        tstats = g.learned_train(3000, batch=16384, lr=2e-3, seed=3)
        g.set_weno_mode("learned")
        g.learned_set_threshold(LEARNED_THRESHOLD)
        g.advance(dt, 1)
        g.learned_counts()
        barrier(world)
        torch.cuda.synchronize()
        g.profile(True)
        ev0.record(stream)
        for _ in range(args.steps):
            g.advance(dt, 1)
        ev1.record(stream)
        torch.cuda.synchronize()
        lprof = g.profile_read()
        g.profile(False)
        barrier(world)
        g.synchronize()
        nl, nf = g.learned_counts()
        g.set_weno_mode("plain")
        ms_l = reduce_max(ev0.elapsed_time(ev1), world)
        learned = {"value": aggregate_value(N, args.steps, ms_l / 1e3, world), "unit": "cell-steps/s",
                   "ms_per_step": ms_l / args.steps, "dtype": "f32 stencils, bf16 network (fp32 accumulate)",
                   "threshold": LEARNED_THRESHOLD, "fallback_frac": nf / max(1, nl + nf),
                   "kernel_ms": {"k_xy": lprof["xy"][0] / max(lprof["xy"][1], 1),
                                 "k_z": lprof["z"][0] / max(lprof["z"][1], 1)},
                   "training": {"samples": tstats["samples"], "steps": tstats["steps"], "batch": 16384,
                                "loss_first": tstats["loss_first"], "loss_last": tstats["loss_last"],
                                "ms": tstats["ms"]}}

    if rank == 0:
        peaks = measured_peaks()
        hbm_peak = peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
        xy_ms, xy_n = prof["xy"]
        z_ms, z_n = prof["z"]
        # Algorithmic bytes: 32*S B per cell-step (8 passes over the S-field
        # FP32 state).  The x/y kernel owns 1 of the 8 passes per stage
        # (reading the stage input), i.e. 4*S B per cell per launch.
        alg_xy = 4.0 * S * N
        xy_avg_s = xy_ms / 1e3 / max(xy_n, 1)
        achieved = alg_xy / xy_avg_s / 1e9
        traffic, tinfo = None, {}
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            with open(tpath) as f:
                tinfo = json.load(f)
            traffic = tinfo.get("k_xy_bytes_per_launch")
        cpu = None
        if not args.no_cpu_baseline:
            try:
                cpu = cpu_reference_rate(steps=1, warmup=1)
            except Exception as e:  # the baseline is a report, not the product
                cpu = {"error": str(e)}
        line = {
            "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": workload_name(), "cells": N, "prognostics": S, "weno": "plain",
                       "l2": "state and stage buffers (%.2f GB) exceed L2" % (4 * S * N * 4 / 1e9),
                       "parallelism": "replicas" if world > 1 else "single"},
            "hbm_gbs_step": 32.0 * S * N * args.steps / (ms / 1e3) / 1e9,
            "roofline": {"kernel": "k_xy (x/y WENO + Riemann + divergence)", "bound": "hbm",
                         "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                         "traffic": traffic, "peak_source": peaks.get("source"),
                         "note": "FP32-FMA-pipe bound (compute_roofline); the HBM fraction is reported from algorithmic bytes"},
            "compute_roofline": {"kernel": "k_xy", "bound": "fp32 fma pipe",
                                 "fma_pipe_frac": tinfo.get("k_xy_fma_pipe_frac"),
                                 "issue_frac": tinfo.get("k_xy_issue_frac"),
                                 "k_z_fma_pipe_frac": tinfo.get("k_z_fma_pipe_frac"),
                                 "k_z_issue_frac": tinfo.get("k_z_issue_frac"),
                                 "source": tinfo.get("source")},
            "kernel_ms": {"k_xy": xy_ms / max(xy_n, 1), "k_z": z_ms / max(z_n, 1),
                          "share_xy": xy_ms / max(xy_ms + z_ms, 1e-12),
                          "timing": "CUDA events around each launch on its stream, in a second pass of the same "
                                    "steps right after the headline region"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": bytes_io,
                    "d2h_bytes_per_step": bytes_io, "calls": args.e2e_calls, "dycore_steps_per_call": ncyc // max(1, args.e2e_calls)},
            "gpu_launches": launches,
            "clocks": clk,
            "learned": learned,
            "physics": physics,
            "decomposed": decomposed,
        }
        print(json.dumps(line), flush=True)
    g.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
