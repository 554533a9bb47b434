#!/usr/bin/env python
"""Benchmark of the B200 backend: throughput of the per-RK-stage RHS + update of the Cartesian
solver in Mcell-steps/s (1 cell-step = one interior cell advanced one full RK3 step).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload bl|channel|sbli] [--size NXxNYxNZ]

Default workload (--workload bl): the Mach 2 spatially developing turbulent boundary layer of the
benchmark suite at its size, 1024x256x192, FP64: box 100 x 12 x 8 inflow thicknesses, BL grid
(wall-resolved tanh-law part plus geometric stretching), recycling-rescaling inflow, zeroth-order
extrapolation with characteristic non-reflecting outflow and top, isothermal wall at the recovery
temperature, periodic z, power-law viscosity, hybrid 6th-order central / WENO5 with Ducros
threshold 0.05, CFL 0.8.  Seeded synthetic initial field: 1/7 power-law mean velocity,
Crocco-Busemann temperature, +-5 % uniform random velocity noise (no dataset exists).
--workload channel is the supersonic channel at 512x256x256 (Mach_b 1.5, Re_b 3000, Poiseuille +
+-10 % noise); --workload sbli the Mach 2.28 shock / boundary-layer interaction at 1024x256x128.

The b200 arm prints one JSON line with: device-timed throughput (value, CUDA events on the
context's stream, max over ranks), the end-to-end throughput through the C ABI with pinned host
buffers (e2e), the roofline of the dominant kernel from live per-kernel CUDA events, the CPU
oracle timed on the host cores (cpu_baseline), the SM clocks sampled during the timed region, the
mixed-precision form on the three workloads, the batched form (48 channel boxes) and the served
form (a Poisson stream of solves).  The headline is timed from step 4 of the synthetic start, a
transient in which most faces take the WENO branch (weno_face_fraction_xyz); "developed" repeats
the measurement from step 300, when the hybrid scheme runs mostly central; "full_run" times the
configuration's whole run (--run-steps, 500, after the warm-up) in event-bracketed segments, the
headline's and the developed window's steps included.  With --gpus N > 1 each rank advances an independent replica
(the path has no exchange step).  --impl reference times the CPU restatement of the reference's
CPU backend (oracle/) on the host.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for p in (ROOT / "streams-2_b200", ROOT / "oracle"):
    sys.path.insert(0, str(p))

# Algorithmic (compulsory) bytes per interior cell of one launch of each kernel: the fields the
# kernel must read and write once; stencil re-reads of neighbours are excluded.
ALG_BYTES_PER_CELL = {
    "k_aux": 40 + 56,                          # read w (5), write rho,u,v,w,H,T,mu
    "k_euler_x": 6 * 8 + 8 + 40,               # read rho,u,v,w,H,T + sensor, write fl (5)
    "k_visc": 5 * 8 + 32 + 32 + 8,             # read u,v,w,T,mu + fl(2:5), write fl(2:5) + div/3
    "k_euler_y": 6 * 8 + 8 + 40 + 40,          # + read-modify-write fl
    "k_euler_z": 7 * 8 + 8 + 8 + 40 + 40 + 32,  # + div/3, fl_prev(1:2), w(1:2)
    "k_update": 40 + 40 + 40 + 8 + 40,         # read w, fl_prev, fl_new, u; write w
    "k_dt": 8 + 5 * 8,
}
# Passes per time step of the kernels above (one per Runge-Kutta stage; dt once per step).
PASSES_PER_STEP = {"k_aux": 3, "k_euler_x": 3, "k_visc": 3, "k_euler_y": 3, "k_euler_z": 3, "k_update": 3, "k_dt": 1}
# Compulsory traffic of a whole RK3 step per cell (state read/written once per stage, RK register).
STEP_BYTES_PER_CELL = 440
# FP64 roofline of the flux passes: operations per WENO face and per central face counted
# through the oracle's face-flux code (profiles/fp64_flops.json, written by
# oracle/count_flops.py), plus the divergence (10 per cell), times the faces of the direction
FLUX_DIR = {"k_euler_x": 0, "k_euler_y": 1, "k_euler_z": 2}
# nominal FP64 rate of a B200: 148 SMs x 64 FMA lanes x 2 flops x 1.965 GHz
NOMINAL_FP64_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12


def flux_flops(kernel, nx, ny, nz, weno_fraction, scheme="weno5_central6"):
    f = ROOT / "profiles" / "fp64_flops.json"
    if kernel not in FLUX_DIR or not f.exists():
        return None
    d = json.loads(f.read_text())
    sc = d["schemes"][scheme]
    dr = FLUX_DIR[kernel]
    faces = nx * ny * nz * ((nx, ny, nz)[dr] + 1) / (nx, ny, nz)[dr]
    fw = weno_fraction[dr]
    per_face = fw * sc["weno_face"]["flops"] + (1 - fw) * sc["central_face"]["flops"]
    return faces * per_face + nx * ny * nz * d["divergence_per_cell_per_direction"]


def fp64_peak(torch):
    """Measured FP64 rate of this GPU: cuBLAS DGEMM (torch.matmul, float64, 8192^3), best of 5
    by CUDA events; the nominal rate is reported beside it."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = None
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def parse_size(s):
    a = [int(v) for v in s.lower().split("x")]
    assert len(a) == 3
    return a


def peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.out.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def channel_case_ini(nx, ny, nz, steps, **kw):
    from streams_b200.cases import channel_ini
    return channel_ini(nx, ny, nz, num_iter=steps, print_control=max(1, steps), **kw)


# Boundary-layer workload: Mach 2 spatially developing turbulent boundary layer, box 100 x 12 x 8
# inflow thicknesses, BL grid, recycling-rescaling inflow, non-reflecting outflow and top,
# isothermal wall at the recovery temperature, periodic z; the SBLI variant adds an impinging
# shock of 8-degree deflection at Mach 2.28 on the top boundary.
SBLI_KW = dict(mach=2.28, shock_angle=32.6)


def bl_case_ini(nx, ny, nz, steps, **kw):
    from streams_b200.cases import bl_ini
    return bl_ini(nx, ny, nz, num_iter=steps, print_control=max(1, steps), **kw)


def case_ini(workload, nx, ny, nz, steps):
    if workload == "channel":
        return channel_case_ini(nx, ny, nz, steps)
    if workload == "sbli":
        return bl_case_ini(nx, ny, nz, steps, **SBLI_KW)
    return bl_case_ini(nx, ny, nz, steps)


DEFAULT_SIZE = {"bl": "1024x256x192", "channel": "512x256x256", "sbli": "1024x256x128"}


def run_batched(torch, precision, steps, warmup, tune_cache, shared=1):
    """The batched form: 48 channel boxes of uneven grids and flow parameters (seeded mix),
    autotuned launch shapes, one CUDA graph per 10 steps of all boxes: with shared launches (one
    launch per kernel kind and stage over the box table of all 48 boxes; shared=2: the boxes in
    two such groups on parallel graph branches) or, shared=0, one graph branch per box.  Device time from CUDA events recorded on every box's stream (start on
    the first box, max over the ends)."""
    from streams_b200 import Batch, Case, Solver
    from streams_b200.cases import batch_mix
    from streams_b200.tune import autotune
    boxes = batch_mix()
    solvers, cells = [], 0
    with tempfile.TemporaryDirectory() as d:
        for i, b in enumerate(boxes):
            kw = dict(b)
            nx, ny, nz = kw.pop("nx"), kw.pop("ny"), kw.pop("nz")
            bd = os.path.join(d, f"b{i}")
            os.makedirs(bd)
            case = Case(bd, channel_case_ini(nx, ny, nz, steps, **kw))
            t = autotune(case, precision=precision, cache=tune_cache)
            sv = Solver.from_case(case, precision=precision)
            sv.set_tuning(*t)
            sv.init_run()
            solvers.append(sv)
            cells += nx * ny * nz
    batch = Batch(solvers, steps_per_graph=10)
    batch.set_shared_launches(shared)
    groups = batch.groups()
    batch.advance(1 + warmup)
    batch.synchronize()
    streams = [torch.cuda.ExternalStream(sv.stream_handle) for sv in solvers]
    e0 = torch.cuda.Event(enable_timing=True)
    ends = [torch.cuda.Event(enable_timing=True) for _ in solvers]
    torch.cuda.synchronize()
    l0 = sum(sv.launches for sv in solvers)
    e0.record(streams[0])
    batch.advance(steps)
    for e, st in zip(ends, streams):
        e.record(st)
    batch.synchronize()
    ms = max(e0.elapsed_time(e) for e in ends)
    replays, per = batch.stats()
    launches = sum(sv.launches for sv in solvers) - l0
    batch.close()
    for sv in solvers:
        sv.close()
    return {"value": cells * steps / (ms / 1e3) / 1e6, "unit": "Mcell-steps/s", "boxes": len(boxes),
            "cells": cells, "steps": steps, "ms": ms, "graph_replays": replays, "launches_per_replay": per,
            "gpu_launches": launches, "shared_launches": shared, "groups": groups[0], "boxes_in_groups": groups[1]}


def run_serving(torch, duration_s, step_scale, single_rate, tune_cache):
    """The served form: a Poisson stream of channel solves (grids log-uniform between 48^3 and
    384x192x128 cells, Mach 0.5-2.5, FP64 or mixed), arrivals over duration_s seconds at a rate
    that saturates the GPU (from the single-box throughput), step counts 200-2000 scaled by
    step_scale so the run stays short; HBM budget 150 GB (or what is free)."""
    import numpy as np
    from streams_b200.cases import serve_mix
    from streams_b200.serve import Server
    lo, hi = max(2, int(200 * step_scale)), max(3, int(2000 * step_scale))
    mean_cells = (384 * 192 * 128 - 48 ** 3) / np.log((384 * 192 * 128) / 48 ** 3)
    # offered load: 1.25x what one large box sustains, from the drawn requests' own work
    rate = 1.25 * single_rate * 1e6 / (mean_cells * (lo + hi) / 2)
    reqs = serve_mix(int(rate * duration_s * 2) + 8, 1.0, steps=(lo, hi))
    work, k = 0.0, 0
    while k < len(reqs) and work < 1.25 * single_rate * 1e6 * duration_s:
        work += reqs[k]["nx"] * reqs[k]["ny"] * reqs[k]["nz"] * reqs[k]["nsteps"]
        k += 1
    reqs = reqs[:k]
    scale = duration_s / reqs[-1]["arrival"]
    for r in reqs:
        r["arrival"] *= scale
    rate = len(reqs) / duration_s
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(150e9, free - 8e9))
    srv = Server(budget_bytes=budget, tick_steps=10, tune_cache=tune_cache)
    out = srv.run(reqs)
    return {"requests": len(reqs), "completed": out["completed"], "rejected": len(out["rejected"]),
            "rate_per_s": rate, "arrival_window_s": duration_s, "steps_range": [lo, hi],
            "p50_s": out["p50_s"], "p99_s": out["p99_s"], "mean_s": out["mean_s"],
            "mcell_steps_per_s": out["mcell_steps_per_s"], "mcell_steps_per_busy_s": out["mcell_steps_per_busy_s"],
            "max_resident": out["max_resident"], "ticks": out["ticks"], "budget_gb": budget / 1e9,
            "offered_mcell_steps_per_s": work / duration_s / 1e6, "loop_admit_wait_s": out["admit_wait_s"],
            "loop_iterations": out["loop_iterations"], "cohort_ticks": out["cohort_ticks"],
            "max_cohort": out["max_cohort"],
            "loop": "admission (tuning, context, first step, first tick) on 2 admission threads; the resident "
                    "solves of a class take their next 10-step tick together (a cohort: shared launches over their "
                    "box table) once all of them are seen done, a solve without a class on its own"}


def cpu_oracle_rate(workload, nx, ny, nz, nsteps, budget_s=20.0):
    """Oracle (restated CPU backend) throughput on a slab of the workload: all host threads."""
    from oracle_py import Oracle
    ini = case_ini(workload, nx, ny, nz, nsteps)
    with tempfile.TemporaryDirectory() as d:
        o = Oracle(d, ini)
        o.init_run()
        o.step()  # warm-up step (first-touch of the arrays)
        t0 = time.perf_counter()
        n = 0
        while n < nsteps:
            o.step()
            n += 1
            if time.perf_counter() - t0 > budget_s:
                break
        dt = time.perf_counter() - t0
    return nx * ny * nz * n / dt / 1e6, n, dt


def sample_dims(nx, ny, nz, target_cells=2_200_000):
    """Slab of the workload with the same x-y plane and fewer z planes (at least 8)."""
    kz = max(8, min(nz, target_cells // (nx * ny)))
    return nx, ny, kz


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    nx, ny, nz = parse_size(args.size)
    sx, sy, sz = sample_dims(nx, ny, nz)
    from oracle_py import Oracle
    threads = os.environ.get("ORACLE_THREADS") or str(os.cpu_count() or 1)
    ini = case_ini(args.workload, sx, sy, sz, args.steps)
    with tempfile.TemporaryDirectory() as d:
        o = Oracle(d, ini)
        o.init_run()
        for _ in range(args.warmup):
            o.step()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            o.step()
        dt = time.perf_counter() - t0
    value = sx * sy * sz * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": "Mcell-steps/s", "value": value, "unit": "Mcell-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.workload, nx, ny, nz),
        "cpu_baseline": {"value": value, "unit": "Mcell-steps/s", "cores": int(threads), "kind": "port",
                         "sample": f"{sx}x{sy}x{sz} slab of the {nx}x{ny}x{nz} {args.workload}, "
                                   f"{args.steps} RK3 steps"},
        "e2e": {"value": value, "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's Fortran/MPI CPU backend cannot be built on this image (no Fortran compiler, "
                "no MPI); this arm times the C++ restatement of that backend (oracle/), pinned to the "
                "reference's golden row",
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(workload, nx, ny, nz):
    if workload == "channel":
        desc = (f"supersonic channel {nx}x{ny}x{nz} FP64, hybrid central-6/WENO5 (Ducros 0.05), "
                "Mach_b 1.5, Re_b 3000, power-law mu, CFL 0.8")
    elif workload == "sbli":
        desc = (f"Mach 2.28 shock / boundary-layer interaction {nx}x{ny}x{nz} FP64, 8-degree impinging shock, "
                "recycling inflow, NR outflow, hybrid central-6/WENO5 (Ducros 0.05), CFL 0.8")
    else:
        desc = (f"Mach 2 spatially developing boundary layer {nx}x{ny}x{nz} FP64, box 100x12x8 delta, "
                "recycling-rescaling inflow, NR outflow and top, isothermal wall at T_recovery, "
                "hybrid central-6/WENO5 (Ducros 0.05), power-law mu, CFL 0.8")
    return {"workload": desc, "grid": [nx, ny, nz], "cells": nx * ny * nz, "precision": "fp64",
            "l2_policy": "inputs larger than L2 (state ~12 x 8 B per cell)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="bl", choices=["bl", "channel", "sbli"])
    ap.add_argument("--size", default=None, help="NXxNYxNZ (default: the workload's benchmark size)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision measurement")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-form measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-form measurement")
    ap.add_argument("--no-developed", action="store_true",
                    help="skip the second measurement on the developed flow")
    ap.add_argument("--run-steps", type=int, default=500,
                    help="length of the configuration's whole run, timed after the warm-up (full_run)")
    ap.add_argument("--developed-at", type=int, default=300,
                    help="step from which the developed-flow measurement is timed")
    ap.add_argument("--batched-steps", type=int, default=200)
    ap.add_argument("--serve-seconds", type=float, default=30.0)
    ap.add_argument("--serve-step-scale", type=float, default=0.1)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.size is None:
        args.size = DEFAULT_SIZE[args.workload]
    if args.impl == "reference":
        return run_reference(args)

    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from streams_b200 import Case, Solver

    nx, ny, nz = parse_size(args.size)
    ncell = nx * ny * nz
    with tempfile.TemporaryDirectory() as d:
        case = Case(d, case_ini(args.workload, nx, ny, nz, args.steps))
    info = case.info()
    s = Solver.from_case(case)
    s.init_run()
    stream = torch.cuda.ExternalStream(s.stream_handle)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # warm-up
    s.advance(args.warmup, 1, 0, 0)
    s.synchronize()
    icyc = args.warmup
    weno_timed = [round(x, 4) for x in s.count_weno()]  # fraction of WENO faces entering the timed steps

    # timed region: device-resident state, CUDA events on the context's stream
    barrier()
    l0 = s.launches
    weno_before = s.count_weno()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        s.advance(args.steps, 1, icyc, 0)
        ev1.record(stream)
        s.synchronize()
        barrier()
    icyc += args.steps
    launches = s.launches - l0
    weno_after = s.count_weno()
    weno_mean = [(a_ + b_) / 2 for a_, b_ in zip(weno_before, weno_after)]
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = ncell * args.steps * world / (ms / 1e3) / 1e6

    # per-kernel device time: the timed steps again, with the event profiler on, in a fresh solver
    # of the same case (the run is deterministic, so it replays the timed region exactly)
    sp = Solver.from_case(case)
    sp.init_run()
    sp.advance(args.warmup, 1, 0, 0)
    sp.profile(-1)
    sp.profile(1)
    sp.advance(args.steps, 1, args.warmup, 0)
    sp.synchronize()
    sp.profile(0)
    prof = sp.profile_report()
    sp.close()
    total_prof = sum(v[0] for v in prof.values())
    dom = max((k for k in prof if k in ALG_BYTES_PER_CELL), key=lambda k: prof[k][0])
    # time of one pass (both forms of the y and z passes are launched; one leaves at once)
    dom_ms = prof[dom][0] / (PASSES_PER_STEP[dom] * args.steps)
    dom_bytes = ALG_BYTES_PER_CELL[dom] * ncell
    peak, peak_kind = peaks()
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "dram_traffic.json"
    if tf.exists():
        t = json.loads(tf.read_text()).get(dom)
        if t:
            traffic = t["bytes_per_cell"] * ncell
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                "alg_bytes_per_cell": ALG_BYTES_PER_CELL[dom], "launch_ms": dom_ms,
                "share": prof[dom][0] / total_prof}
    # the flux passes are FP64-bound: their counted operations against the measured DGEMM rate
    roofline_fp64 = None
    dflops = flux_flops(dom, nx, ny, nz, weno_mean)
    if dflops is not None:
        pk = fp64_peak(torch)
        ach = dflops / (dom_ms / 1e3) / 1e12
        step_flux = sum(flux_flops(k, nx, ny, nz, weno_mean) for k in FLUX_DIR)
        step_ms_flux = sum(prof[k][0] for k in FLUX_DIR if k in prof) / args.steps
        roofline_fp64 = {"bound": "fp64", "kernel": dom, "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                         "frac": ach / pk, "peak_kind": "measured (cuBLAS DGEMM 8192^3, float64)",
                         "nominal_peak": NOMINAL_FP64_TFLOPS, "frac_of_nominal": ach / NOMINAL_FP64_TFLOPS,
                         "flops_per_launch": dflops, "weno_face_fraction_xyz": [round(x, 4) for x in weno_mean],
                         "flops_source": "profiles/fp64_flops.json (oracle/count_flops.py)",
                         "three_flux_passes": {"tflops": step_flux * 3 / (step_ms_flux / 1e3) / 1e12,
                                               "ms_per_step": step_ms_flux}}
        roofline["binding"] = "fp64 (see roofline_fp64): the flux passes do ~10 FP64 operations per byte"
    step_gbs = STEP_BYTES_PER_CELL * ncell * args.steps / (ms / 1e3) / 1e9
    step_roofline = {"bytes_per_cell_step": STEP_BYTES_PER_CELL, "achieved": step_gbs, "peak": peak,
                     "frac": step_gbs / peak, "unit": "GB/s", "peak_kind": peak_kind}
    kernels = {k: {"ms_per_step": v[0] / args.steps, "ms_per_launch": v[0] / v[1], "launches": v[1],
                   "share": v[0] / total_prof}
               for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}

    # the configuration's whole run (run_steps steps after the warm-up) and, inside it, the same
    # measurement on the developed flow: the synthetic start is a strong transient in which the
    # Ducros sensor sends most faces to WENO; after a few hundred steps the hybrid scheme runs
    # mostly central, as a production run does (fraction of WENO faces reported).  The run is
    # timed in segments, each bracketed by events on the context's stream with nothing else
    # inside, and the segments are summed with the timed region above.
    developed = None
    full_run = None
    if not args.no_developed and args.developed_at > icyc:
        def timed_advance(n):
            nonlocal icyc
            a0_, a1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            barrier()
            a0_.record(stream)
            s.advance(n, 1, icyc, 0)
            a1_.record(stream)
            s.synchronize()
            barrier()
            icyc += n
            return max_over_ranks(a0_.elapsed_time(a1_))

        seg_ms = [ms, timed_advance(args.developed_at - icyc)]
        weno_dev = [round(x, 4) for x in s.count_weno()]
        dms = timed_advance(args.steps)
        seg_ms.append(dms)
        run_end = max(args.warmup + args.run_steps, icyc)
        if run_end > icyc:
            seg_ms.append(timed_advance(run_end - icyc))
        run_n = icyc - args.warmup
        full_run = {"value": ncell * run_n * world / (sum(seg_ms) / 1e3) / 1e6, "unit": "Mcell-steps/s",
                    "ms_per_step": sum(seg_ms) / run_n, "steps": run_n, "from_step": args.warmup,
                    "weno_face_fraction_xyz_at_end": [round(x, 4) for x in s.count_weno()]}
        # per-kernel device time of the steps that follow (the developed regime)
        s.profile(-1)
        s.profile(1)
        s.advance(args.steps, 1, icyc, 0)
        s.synchronize()
        s.profile(0)
        icyc += args.steps
        dprof = s.profile_report()
        developed = {"value": ncell * args.steps * world / (dms / 1e3) / 1e6, "unit": "Mcell-steps/s",
                     "ms_per_step": dms / args.steps, "timed_from_step": args.developed_at,
                     "weno_face_fraction_xyz": weno_dev,
                     "kernels_ms_per_step": {k: round(v[0] / args.steps, 3)
                                             for k, v in sorted(dprof.items(), key=lambda kv: -kv[1][0])},
                     "kernels_from_step": icyc - args.steps}

    # end to end through the C ABI with pinned host buffers: upload the field, run, read the
    # progress scalars after every step (the step's metric), download the final field
    nbytes = 5 * (nx + 6) * (ny + 6) * (nz + 6) * 8
    hin = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
    hout = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
    hin.numpy()[:] = case.field().reshape(-1)
    s2 = Solver(case.params(0), case.grid(), keepalive=case)
    st2 = torch.cuda.ExternalStream(s2.stream_handle)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    t0 = time.perf_counter()
    e0.record(st2)
    s2.copy_from_host_ptr(hin.data_ptr())
    s2.init_run()
    for n in range(args.steps):
        s2.advance(1, 1, n, 0)
        s2.scalars()
    s2.copy_to_host_ptr(hout.data_ptr())
    e1.record(st2)
    s2.synchronize()
    wall = time.perf_counter() - t0
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_val = ncell * args.steps * world / (e2e_ms / 1e3) / 1e6
    s2.close()

    # mixed form (FP32 fluxes, FP64 state): throughput on the headline workload and on the two
    # mixed-precision workloads (the channel at 512x256x256, the shock / boundary-layer interaction at
    # 1024x256x128), each with its error against the FP64 form after 100 steps of a smaller case
    def device_rate(cs, precision, kernel_table=None):
        sv = Solver.from_case(cs, precision=precision)
        sv.init_run()
        sv.advance(args.warmup, 1, 0, 0)
        st_ = torch.cuda.ExternalStream(sv.stream_handle)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        a0.record(st_)
        sv.advance(args.steps, 1, args.warmup, 0)
        a1.record(st_)
        sv.synchronize()
        t_ms = max_over_ranks(a0.elapsed_time(a1))
        n_ = cs.shape[0] * cs.shape[1] * cs.shape[2]
        sv.close()
        if kernel_table is not None:
            # per-kernel device time of the same steps replayed with the event profiler
            sp_ = Solver.from_case(cs, precision=precision)
            sp_.init_run()
            sp_.advance(args.warmup, 1, 0, 0)
            sp_.profile(-1)
            sp_.profile(1)
            sp_.advance(args.steps, 1, args.warmup, 0)
            sp_.synchronize()
            sp_.profile(0)
            rep = sp_.profile_report()
            sp_.close()
            kernel_table.update({k: round(v[0] / args.steps, 3)
                                 for k, v in sorted(rep.items(), key=lambda kv: -kv[1][0])})
        return n_ * args.steps * world / (t_ms / 1e3) / 1e6, t_ms

    def mixed_error(wl, dims):
        with tempfile.TemporaryDirectory() as d:
            c0 = Case(d, case_ini(wl, *dims, 100))
        fields = []
        for prec in (0, 1):
            sv = Solver.from_case(c0, precision=prec)
            sv.init_run()
            sv.advance(100, 1, 0, 0)
            fields.append(sv.copy_to_field()[:, 3:-3, 3:-3, 3:-3])
            sv.close()
        return [float(np.linalg.norm(fields[1][m] - fields[0][m]) / np.linalg.norm(fields[0][m])) for m in range(5)]

    small = {"bl": (128, 64, 32), "channel": (128, 96, 64), "sbli": (128, 64, 32)}
    mixed = None
    if not args.no_mixed:
        mkern = {}
        mval, mms = device_rate(case, 1, mkern)
        errs = mixed_error(args.workload, small[args.workload])
        mixed = {"value": mval, "unit": "Mcell-steps/s", "ms_per_step": mms / args.steps, "speedup_vs_fp64": mval / value,
                 "rel_l2_vs_fp64_100_steps": errs, "error_case": "x".join(map(str, small[args.workload])),
                 "max_rel_l2": max(errs), "kernels_ms_per_step": mkern,
                 "precision": "FP32 flux/viscous arithmetic, FP64 state, RK register, T recovery, sensor, dt, "
                              "reductions"}
        # the long-run check of the mean flow (5000 steps of the channel at 512x256x256 and the
        # shock interaction at 1024x256x128 in both precisions, statistics post-processed as
        # tools/postpro does): too long for this run, measured by streams_b200.mean_profile_check
        mp = ROOT / "profiles" / "mixed_mean_profile_5000.json"
        if mp.exists():
            mixed["mean_profile_err_5000"] = {
                k: {"max_rel_diff": v["max_rel_diff_mixed_vs_fp64"], "stat_samples": v["stat_samples"],
                    "source": "profiles/mixed_mean_profile_5000.json"}
                for k, v in json.loads(mp.read_text()).items()}
        for wl in ("channel", "sbli"):
            if wl == args.workload:
                continue
            dims = parse_size(DEFAULT_SIZE[wl])
            with tempfile.TemporaryDirectory() as d:
                cw = Case(d, case_ini(wl, *dims, args.steps))
            f64, _ = device_rate(cw, 0)
            f32, _ = device_rate(cw, 1)
            e = mixed_error(wl, small[wl])
            mixed[f"{wl}_{DEFAULT_SIZE[wl]}"] = {
                "fp64": f64, "mixed": f32, "speedup_vs_fp64": f32 / f64, "rel_l2_vs_fp64_100_steps": e,
                "error_case": "x".join(map(str, small[wl])), "max_rel_l2": max(e)}
            del cw

    # batched and served forms (rank 0 of a replica run measures them on its own GPU)
    tune_cache = {}
    batched = None
    if not args.no_batched:
        batched = {"fp64": run_batched(torch, 0, args.batched_steps, args.warmup, tune_cache),
                   "mixed": run_batched(torch, 1, args.batched_steps, args.warmup, tune_cache)}
        # the same boxes in two groups on parallel branches, and with a graph branch per box
        for name, shared in (("two_groups", 2), ("separate_branches", 0)):
            for k, prec in (("fp64", 0), ("mixed", 1)):
                o = run_batched(torch, prec, args.batched_steps, args.warmup, tune_cache, shared=shared)
                batched[k][name] = {q: o[q] for q in ("value", "ms", "launches_per_replay", "groups")}
        batched["fp64"]["vs_single_box"] = batched["fp64"]["value"] / value
        if mixed:
            batched["mixed"]["vs_single_box"] = batched["mixed"]["value"] / mixed["value"]
        batched["workload"] = ("48 channel boxes, grids from {64,96,128}x{64,96}x{32,64,96}, Mach U[0.3,2], "
                               "Re_b U[2000,6000], seeded; one CUDA graph per 10 steps of all boxes, shared launches over "
                               "the box table (one launch per kernel kind and stage)")
    serving = None
    if not args.no_serve:
        serving = run_serving(torch, args.serve_seconds, args.serve_step_scale, value, tune_cache)
        serving["vs_single_box"] = (serving["mcell_steps_per_s"] or 0.0) / value

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            sx, sy, sz = sample_dims(nx, ny, nz)
            rate, nst, sec = cpu_oracle_rate(args.workload, sx, sy, sz, 5)
            cpu = {"value": rate, "unit": "Mcell-steps/s", "cores": int(os.environ.get("ORACLE_THREADS") or
                                                                       (os.cpu_count() or 1)),
                   "kind": "port", "sample": f"{sx}x{sy}x{sz} slab of the {nx}x{ny}x{nz} {args.workload}, "
                                             f"{nst} RK3 steps in {sec:.1f} s"}
        except Exception as e:  # the baseline is reported, not required
            cpu = {"value": None, "unit": "Mcell-steps/s", "cores": 0, "kind": "port", "sample": f"failed: {e}"}

    res = s.compute_residual()
    sc = s.scalars()
    if rank == 0:
        line = {
            "metric": "Mcell-steps/s", "value": value, "unit": "Mcell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.workload, nx, ny, nz),
            "e2e": {"value": e2e_val, "unit": "Mcell-steps/s", "h2d_bytes_per_step": nbytes / args.steps,
                    "d2h_bytes_per_step": (nbytes + 56 * args.steps) / args.steps, "wall_s": wall,
                    "what": "copy_from_field (pinned) + init_run + K x (rk step + scalar read) + copy_to_field"},
            "roofline": roofline, "roofline_fp64": roofline_fp64, "step_roofline": step_roofline, "kernels": kernels,
            "gpu_launches": launches, "clocks": clk.summary(), "cpu_baseline": cpu, "mixed": mixed,
            "batched": batched, "serving": serving,
            "weno_face_fraction_xyz": weno_timed, "developed": developed, "full_run": full_run,
            "state": {"dt": sc["dt"], "rhobulk": sc["rhobulk"], "ubulk": sc["ubulk"], "tbulk": sc["tbulk"],
                      "residual_rhou": res["residual_rhou"], "nan": res["nan"]},
            "u0": info["u0"],
        }
        print(json.dumps(line), flush=True)
    s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
