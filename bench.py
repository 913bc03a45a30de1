#!/usr/bin/env python3
"""Benchmark of the B200 dycore: cell-steps/s of the order-9 WENO SSPRK3
dynamical core on the large urban canopy (1024x1024x256 cells at 1 m,
seeded cuboid buildings as a binary immersed mask, one water-vapour tracer;
268 M cells), plain FP32 beside the learned-weight form, each with its L2 and
Linf error per prognostic against the FP64 build of the same kernels after
the same steps from the same state.  One JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value: K SSPRK3 steps of the resident FP32 state in one advance call, timed
  with CUDA events on the dycore's stream between a barrier and a device
  synchronize on both sides, max over ranks; the state (6.4 GB per buffer) is
  far larger than L2.
* errors: after the W+K steps, the conserved variables of the plain and the
  learned runs against the FP64 build's (same initial state, same dt),
  relative to the FP64 field's departure from the hydrostatic background.
* e2e: the reference-facing call (pu_dycore_time_step, dt_phys = 10 dycore
  steps as the reference's drivers use, abl_neutral.cpp:25) with the coupler
  arrays in pinned host memory: host->device copy, conversion, 10 SSPRK3
  steps, conversion back and device->host copy inside every timed call (the
  library overlaps the copies with the steps chunk by chunk).
* roofline: the x/y flux kernel (the larger share of the step), its
  algorithmic bytes per launch over its CUDA-event duration; traffic from the
  committed ncu capture (profiles/traffic.json).
* cpu_baseline / --impl reference: the reference's own dycore code
  (oracle/_ref, built from the reference's headers with a single-rank shim)
  on all host cores, on a 64x64x256 window of the same domain; beside it the
  FP64 oracle's rate on that window.
* learned: the learned-weight form on the same initial state, after
  harvesting 2^24 stencils from the plain run and training the network on the
  GPU (Adam, batch 65536); kernel times and the fallback fraction.
* abl: the neutral boundary layer (256x256x128, dx = 10 m, water_vapor + TKE)
  as an extra object: the plain dycore rate, the physics modules its driver
  runs beside the dycore (FP64), the driver's whole step with the TKE LES
  closure (driver_chain), and the same grid as 2x2 tiles of one GPU.
* Multi-GPU: N ranks run N independent replicas (ensemble members: the same
  city, each rank its own noise seed) with no collective in the data path
  (weak scaling).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import platform
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "source": "fallback"}
WORKLOAD = dict(nx=1024, ny=1024, nz=256, dx=1.0)      # the large urban canopy
CPU_WINDOW = (0, 0, 64, 64)                            # columns of the CPU sample
ABL = dict(nx=256, ny=256, nz=128, dx=10.0)            # the boundary layer (extra object)
DYN_CYCLE = 10
LEARNED_THRESHOLD = 0.5
LEARN_SAMPLES = 1 << 24
LEARN_BATCH = 65536
LEARN_STEPS = 3000
LEARN_LR = 2e-3


def workload_name():
    w = WORKLOAD
    return ("urban_canopy %dx%dx%d dx=%gm: seeded cuboid buildings (40 m lots, footprints 20-32 m, heights "
            "10-60 m, 70%% occupancy) as a binary immersed mask, water_vapor tracer, WENO order 9, SSPRK3"
            % (w["nx"], w["ny"], w["nz"], w["dx"]))


def build_case(seed=0, window=None):
    """The workload; replicas (ensemble members) share the city (layout seed 1)
    and differ in their theta noise (seed = rank)."""
    from porturb_b200 import cases
    return cases.urban_canopy(nx=WORKLOAD["nx"], ny=WORKLOAD["ny"], nz=WORKLOAD["nz"], dx=WORKLOAD["dx"],
                              seed=seed, window=window, layout_seed=1)


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
        sm, mx, pw, reasons = [], None, [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
                pw.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "power_w_median": float(np.median(pw)) if pw else None}


def cpu_info():
    model = platform.processor() or ""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "logical_cpus": os.cpu_count()}


def cpu_f64_rate(case, steps=2, warmup=1):
    """Cell-steps/s of the FP64 oracle (the same algorithm with FP64
    arithmetic throughout) on the host cores, on the same window."""
    import pyoracle
    d = pyoracle.Dycore(case, "f64")
    d.init_case()
    d.load_coupler(list(case.coupler_arrays(perturbed=True)))
    dt = d.compute_time_step()
    for _ in range(warmup):
        d.advance(dt, 1)
    t0 = time.perf_counter()
    d.advance(dt, steps)
    el = time.perf_counter() - t0
    return {"value": case.ncells * steps / el, "unit": "cell-steps/s", "ms_per_step": el * 1e3 / steps, "kind": "port",
            "sample": "%d step(s) after %d warm-up step(s), the same window" % (steps, warmup)}


def cpu_reference_rate(steps=3, warmup=1, f64=False):
    """Cell-steps/s of the reference's own dycore code on the host cores
    (oracle/_ref; this project's REF restatement if the reference library was
    not built), on a window of the benchmark domain; with f64, also the FP64
    oracle's rate there."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    kind = "reference" if pyoracle.have_ref() else "ref"
    case = build_case(seed=0, window=CPU_WINDOW)
    d = pyoracle.Dycore(case, kind)
    t0 = time.perf_counter()
    d.init_case()
    init_s = time.perf_counter() - t0
    d.load_coupler(list(case.coupler_arrays(perturbed=True)))
    dt = d.compute_time_step()
    for _ in range(warmup):
        d.advance(dt, 1)
    t0 = time.perf_counter()
    d.advance(dt, steps)
    el = time.perf_counter() - t0
    lib = pyoracle._lib(pyoracle.ORACLE_SO, "orc_")
    threads = int(lib.orc_num_threads())
    out = {"value": case.ncells * steps / el, "unit": "cell-steps/s", "cores": threads,
           "kind": "reference" if kind == "reference" else "port",
           "sample": "%d SSPRK3 step(s) after %d warm-up step(s) on the %dx%dx%d window (columns %d..%d x %d..%d) "
                     "of the %dx%dx%d urban canopy, periodic laterally, %.1f s timed (init %.1f s untimed)"
                     % (steps, warmup, case.nx, case.ny, case.nz, CPU_WINDOW[0], CPU_WINDOW[0] + case.nx - 1,
                        CPU_WINDOW[1], CPU_WINDOW[1] + case.ny - 1, WORKLOAD["nx"], WORKLOAD["ny"], WORKLOAD["nz"],
                        el, init_s),
           "threads": threads, "ms_per_step": el * 1e3 / steps}
    out.update(cpu_info())
    if f64:
        out["f64_oracle"] = cpu_f64_rate(case)
    return out


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
    steps = max(3, min(args.steps, 5))
    base = cpu_reference_rate(steps=steps, warmup=1)
    line = {"impl": "reference", "metric": "cell-steps/s", "value": base["value"], "unit": "cell-steps/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": 1,
            "ms_per_step": base["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64-state/f32-stencil", "data": "synthetic",
            "config": {"workload": workload_name(), "sample": base["sample"]},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU pieces
# ---------------------------------------------------------------------------
def timed_steps(g, dt, steps, stream, world):
    """K SSPRK3 steps in one advance call (the enforcement that starts every
    step, dynamics_rk.h:301, runs in the previous step's last stage kernel;
    a separate pass only before the first), CUDA events on the dycore's
    stream, max over ranks."""
    import torch
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    ev0.record(stream)
    g.advance(dt, steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    return reduce_max(ev0.elapsed_time(ev1), world)


def kernel_pass(g, dt, steps):
    """Per-kernel CUDA events on the launching stream, in a pass of its own:
    an event pair around every launch costs ~2 % of the step, so the timed
    regions run without them."""
    g.profile(True)
    g.advance(dt, steps)
    prof = g.profile_read()
    g.profile(False)
    return {"k_xy": prof["xy"][0] / max(prof["xy"][1], 1), "k_z": prof["z"][0] / max(prof["z"][1], 1),
            "share_xy": prof["xy"][0] / max(prof["xy"][0] + prof["z"][0], 1e-12),
            "launches_xy": prof["xy"][1], "launches_z": prof["z"][1]}


def abl_extras(stream, world, steps, warmup, rank, no_physics, no_decomposed):
    """The neutral boundary layer (256x256x128, dx = 10 m): plain dycore rate,
    the physics modules beside it and the 2x2-tile form."""
    import torch
    from porturb_b200 import Dycore, cases
    case = cases.abl_neutral(nx=ABL["nx"], ny=ABL["ny"], nz=ABL["nz"], dx=ABL["dx"], seed=rank)
    g = Dycore.from_case(case, precision="f32", device=torch.cuda.current_device(), stream=stream.cuda_stream)
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=False)]
    g.init(rd, u, v, w, T, list(trc), None)
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=True)]
    g.load_state(rd, u, v, w, T, list(trc))
    dt = g.compute_time_step()
    for _ in range(warmup):
        g.advance(dt, 1)
    ms = timed_steps(g, dt, steps, stream, world)
    kern = kernel_pass(g, dt, steps)
    g.close()
    out = {"workload": "abl_neutral %dx%dx%d dx=%gm, water_vapor+TKE tracers" % (ABL["nx"], ABL["ny"], ABL["nz"],
                                                                                    ABL["dx"]),
           "value": aggregate_value(case.ncells, steps, ms / 1e3, world), "unit": "cell-steps/s",
           "ms_per_step": ms / steps, "kernel_ms": kern}
    if not no_physics:
        out["physics"] = physics_modules(case, stream, world)
        out["driver_chain"] = driver_chain(world, rank)
    if not no_decomposed:
        out["decomposed"] = decomposed_tiles(case, world, min(steps, 10), warmup)
    return out


def driver_chain(world, rank, calls=5):
    """The boundary-layer driver's whole step (abl_neutral.cpp:93-108) on
    device coupler arrays of the same workload, through the module API:
    geostrophic forcing, the dycore's time_step of dt_phys = 10 dycore steps,
    sponge, surface fluxes, the TKE LES closure and the time averager; CUDA
    events over `calls` driver steps after one, cell-steps/s of the dycore
    steps inside them, the TKE LES closure's cost included."""
    import types
    from porturb_b200 import cases
    from porturb_b200.run_case import run_driver
    case = cases.abl_neutral(nx=ABL["nx"], ny=ABL["ny"], nz=ABL["nz"], dx=ABL["dx"], seed=rank)
    a = types.SimpleNamespace(case="abl_neutral", nx=ABL["nx"], ny=ABL["ny"], nz=ABL["nz"], steps=calls,
                              precision="f32")
    out = run_driver(case, a)
    out["ms_per_call"] = reduce_max(out["ms_per_call"], world)
    out["cell_steps_per_s"] = world * case.ncells * out["dycore_steps_per_call"] / (out["ms_per_call"] / 1e3)
    return out


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
    averager) on device coupler arrays: CUDA-event time per call and, for the
    LES kernel (the out-of-place form, no copy-back), algorithmic HBM bytes
    over its time."""
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-calls", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-f64", action="store_true")
    ap.add_argument("--no-abl", action="store_true")
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
    from porturb_b200.run_case import _snapshot as snapshot, field_errors
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    t_setup = time.perf_counter()
    case = build_case(seed=rank)
    stream = torch.cuda.Stream(device=local)
    N = case.ncells
    S = 5 + len(case.tracers)
    shape = (case.nz, case.ny, case.nx)
    base = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=False)]
    pert = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=True)]
    prop = np.ascontiguousarray(case.immersed_proportion)

    g = Dycore.from_case(case, precision="f32", device=local, stream=stream.cuda_stream)
    g.init(*base[:5], list(base[5]), prop)
    g.load_state(*pert[:5], list(pert[5]))
    dt = g.compute_time_step()
    setup_s = time.perf_counter() - t_setup

    # Warm-up, then the timed region (the headline).
    for _ in range(args.warmup):
        g.advance(dt, 1)
    g.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    launches0 = g.kernel_launches()
    ms = timed_steps(g, dt, args.steps, stream, world)
    launches = g.kernel_launches() - launches0
    clk = clocks.stop()
    value = aggregate_value(N, args.steps, ms / 1e3, world)
    P = None if args.no_f64 else snapshot(g, S, shape)   # after W+K steps
    kern = kernel_pass(g, dt, args.steps)

    # e2e through the C-ABI with pinned host coupler arrays.
    pinned = [torch.empty(shape, dtype=torch.float64, pin_memory=True) for _ in range(5)]
    ptrc = [torch.empty(shape, dtype=torch.float64, pin_memory=True) for _ in range(len(case.tracers))]
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
    bytes_io = S * N * 8
    steps_per_call = ncyc // max(1, args.e2e_calls)
    del pinned, ptrc

    # Learned-weight form: stencils harvested from the plain run's state, the
    # network trained on the GPU, then the same initial state and steps.
    learned, L = None, None
    if not args.no_learned:
        g.learned_harvest(LEARN_SAMPLES, seed=1 + rank)
        tstats = g.learned_train(LEARN_STEPS, batch=LEARN_BATCH, lr=LEARN_LR, seed=3)
        g.load_state(*pert[:5], list(pert[5]))
        g.set_weno_mode("learned")
        g.learned_set_threshold(LEARNED_THRESHOLD)
        for _ in range(args.warmup):
            g.advance(dt, 1)
        g.learned_counts()
        ms_l = timed_steps(g, dt, args.steps, stream, world)
        nl, nf = g.learned_counts()
        if not args.no_f64:
            L = snapshot(g, S, shape)
        lkern = kernel_pass(g, dt, min(args.steps, 3))
        g.set_weno_mode("plain")
        learned = {"value": aggregate_value(N, args.steps, ms_l / 1e3, world), "unit": "cell-steps/s",
                   "ms_per_step": ms_l / args.steps, "dtype": "f32 stencils, bf16 network (fp32 accumulate)",
                   "threshold": LEARNED_THRESHOLD, "fallback_frac": nf / max(1, nl + nf),
                   "kernel_ms": {"k_xy": lkern["k_xy"], "k_z": lkern["k_z"]},
                   "training": {"samples": tstats["samples"], "steps": tstats["steps"], "batch": LEARN_BATCH,
                                "loss_first": tstats["loss_first"], "loss_last": tstats["loss_last"],
                                "ms": tstats["ms"]}}
    g.close()
    del g
    torch.cuda.synchronize()

    # FP64 build of the same kernels, same initial state and steps.
    f64 = None
    if not args.no_f64:
        h = Dycore.from_case(case, precision="f64", device=local, stream=stream.cuda_stream)
        h.init(*base[:5], list(base[5]), prop)
        h.load_state(*pert[:5], list(pert[5]))
        for _ in range(args.warmup):
            h.advance(dt, 1)
        ms_64 = timed_steps(h, dt, args.steps, stream, world)
        D = snapshot(h, S, shape)
        cells, _ = h.get_hydrostasis()
        h.close()
        del h
        f64 = {"value": aggregate_value(N, args.steps, ms_64 / 1e3, world), "unit": "cell-steps/s",
               "ms_per_step": ms_64 / args.steps, "dtype": "f64",
               "errors_after_steps": args.warmup + args.steps,
               "error_norm": "L2 and Linf of (X - FP64) over the FP64 field's departure from the hydrostatic "
                             "background (rho_h, 0, 0, 0, rho_h*theta_h, 0), per prognostic",
               "plain_vs_f64": field_errors(P, D, cells, case.nz)}
        if L is not None:
            f64["learned_vs_f64"] = field_errors(L, D, cells, case.nz)
        del D, P, L
        torch.cuda.empty_cache()

    abl = None if args.no_abl else abl_extras(stream, world, min(args.steps, 20), args.warmup, rank, args.no_physics,
                                              args.no_decomposed)

    if rank == 0:
        peaks = measured_peaks()
        hbm_peak = peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
        # Algorithmic bytes: 32*S B per cell-step (8 passes over the S-field
        # FP32 state) + 1 B of immersed flags per stage.  The x/y kernel owns
        # the read of the stage input and its flags, (4*S + 1) B per cell per
        # launch.
        alg_xy = (4.0 * S + 1.0) * N
        achieved = alg_xy / (kern["k_xy"] / 1e3) / 1e9
        tinfo = {}
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            with open(tpath) as f:
                tinfo = json.load(f).get("urban_canopy_1m", {})
        traffic = tinfo.get("k_xy_bytes_per_cell")
        traffic = traffic * N if traffic is not None else None
        cpu = None
        if not args.no_cpu_baseline:
            try:
                cpu = cpu_reference_rate(steps=3, warmup=1, f64=True)
            except Exception as e:  # the baseline is a report, not the product
                cpu = {"error": str(e)}
        line = {
            "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator; no dataset)",
            "config": {"workload": workload_name(), "cells": N, "prognostics": S, "weno": "plain",
                       "immersed_cells_frac": float(prop.mean()),
                       "l2": "state and stage buffers (%.1f GB) exceed L2" % (4 * S * N * 4 / 1e9),
                       "parallelism": "replicas" if world > 1 else "single", "setup_s": setup_s},
            "hbm_gbs_step": (32.0 * S + 3.0) * N * args.steps / (ms / 1e3) / 1e9,
            "roofline": {"kernel": "k_xy (x/y WENO + Riemann + divergence, immersed)", "bound": "hbm",
                         "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                         "traffic": traffic, "peak_source": peaks.get("source"),
                         "algorithmic_bytes_per_launch": alg_xy,
                         "traffic_source": tinfo.get("source"),
                         "note": "FP32-FMA-pipe bound (compute_roofline); the HBM fraction is reported from "
                                 "algorithmic bytes"},
            "compute_roofline": {"kernel": "k_xy", "bound": "fp32 fma pipe",
                                 "fma_pipe_frac": tinfo.get("k_xy_fma_pipe_frac"),
                                 "issue_frac": tinfo.get("k_xy_issue_frac"),
                                 "k_z_fma_pipe_frac": tinfo.get("k_z_fma_pipe_frac"),
                                 "k_z_issue_frac": tinfo.get("k_z_issue_frac"),
                                 "source": tinfo.get("source")},
            "kernel_ms": dict(kern, timing="CUDA events around each launch on its stream, in a pass of the same "
                                           "number of steps right after the headline region"),
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "cell-steps/s",
                    "h2d_bytes_per_step": bytes_io / max(1, steps_per_call),
                    "d2h_bytes_per_step": bytes_io / max(1, steps_per_call),
                    "h2d_bytes_per_call": bytes_io, "d2h_bytes_per_call": bytes_io,
                    "calls": args.e2e_calls, "dycore_steps_per_call": steps_per_call,
                    "note": "pu_dycore_time_step on pinned host coupler arrays; each call copies the S FP64 "
                            "arrays in and out once and runs dycore_steps_per_call SSPRK3 steps"},
            "gpu_launches": launches,
            "clocks": clk,
            "learned": learned,
            "f64": f64,
            "abl": abl,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
