"""Serving form: a request loop over resident solves with continuous batching.

Requests (channel solves of any size, Mach number, step count and precision) arrive over time.
Each is prepared on the host as it arrives (input parsing, grid, initial field: worker
threads, so that set-up overlaps the GPU work), then admitted in arrival order as soon as its
device footprint fits the HBM budget next to the solves already resident.  A resident solve
keeps its fields in HBM from admission to completion.  The loop advances all resident solves
together in ticks: every resident solve replays its own CUDA graph of a tick's steps (a one-box
``Batch``, captured once when the solve joins) on its own stream, so the solves' stages overlap on
the GPU and a change of the resident set rebuilds nothing (one graph over all resident solves had
to be captured again whenever a solve joined or left, which at a hundred resident solves cost more
host time than the tick's GPU work).  Solves are admitted while a tick runs (their first step
overlaps it), join the next tick, and leave, freeing their memory, at the end of the tick in which
they complete.  Completion latency is
measured from a request's arrival to the end of the tick that completes it.

A solve's arithmetic does not depend on what else is resident: with the same launch tuning its
result is bit-identical alone and in any mix.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import tempfile
import time
from dataclasses import dataclass, field

import numpy as np

from . import Batch, Case, Solver, lib
from .cases import bl_ini, channel_ini


@dataclass
class Solve:
    rid: int
    arrival: float
    nsteps: int
    precision: int
    case: Case
    footprint: int
    cells: int
    solver: Solver | None = None
    batch: Batch | None = None      # the solve's own tick graph
    remaining: int = 0
    admitted: float = 0.0
    finished: float = 0.0
    tuning: tuple | None = None
    result: dict = field(default_factory=dict)


def footprint_of(case: Case, precision: int) -> int:
    import ctypes as C
    p = case.params(precision)
    return int(lib.streams_b200_footprint_bytes(C.byref(p)))


def prepare(req: dict, workdir: str) -> Case:
    """Host set-up of one request (runs in a worker thread; the C++ set-up releases the GIL)."""
    kw = {k: v for k, v in req.items() if k not in ("rid", "arrival", "nsteps", "precision", "kind")}
    d = os.path.join(workdir, f"req{req['rid']}")
    os.makedirs(d, exist_ok=True)
    if req.get("kind", "channel") == "sbli":
        return Case(d, bl_ini(num_iter=req["nsteps"], **kw))
    return Case(d, channel_ini(num_iter=req["nsteps"], **kw))


class Server:
    """Continuous-batching solve server on one GPU.

    budget_bytes  device memory the resident solves may hold together
    tick_steps    steps of every resident solve per tick (fewer when a solve completes sooner)
    tune          autotune each new (grid, precision) class before its first admission
    keep_fields   download each completed solve's conserved field into Solve.result["w"]
    """

    def __init__(self, budget_bytes: int, tick_steps: int = 10, tune: bool = True, keep_fields: bool = False,
                 prep_threads: int = 4, tune_cache: dict | None = None):
        self.budget = int(budget_bytes)
        self.tick_steps = int(tick_steps)
        self.tune = tune
        self.keep_fields = keep_fields
        self.prep_threads = prep_threads
        self.tune_cache = {} if tune_cache is None else tune_cache
        self.log: list[tuple] = []

    def run(self, requests: list[dict], time_scale: float = 1.0) -> dict:
        """Serve `requests` (dicts with rid, arrival [s], nsteps, precision and channel
        parameters) with arrivals replayed in real time (scaled by time_scale); returns the
        per-request records and the latency / throughput summary."""
        from .tune import autotune
        reqs = sorted(requests, key=lambda r: r["arrival"])
        workdir = tempfile.mkdtemp(prefix="streams_b200_serve_")
        pool = cf.ThreadPoolExecutor(max_workers=self.prep_threads)
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        futures: dict[int, cf.Future] = {}
        waiting: list[Solve] = []      # prepared, not admitted (arrival order)
        active: list[Solve] = []
        done: list[Solve] = []
        rejected: list[int] = []
        used = 0
        nxt = 0
        busy = 0.0
        host = {"admit_s": 0.0, "batch_build_s": 0.0}
        try:
            while nxt < len(reqs) or futures or waiting or active:
                # arrivals: start host set-up of every request whose arrival time has come
                while nxt < len(reqs) and reqs[nxt]["arrival"] * time_scale <= now():
                    r = reqs[nxt]
                    futures[r["rid"]] = pool.submit(prepare, r, workdir)
                    nxt += 1
                # prepared requests join the admission queue in arrival order
                for r in reqs:
                    f = futures.get(r["rid"])
                    if f is not None and f.done():
                        case = f.result()
                        del futures[r["rid"]]
                        nx, ny, nz, _ = case.shape
                        s = Solve(r["rid"], r["arrival"] * time_scale, r["nsteps"], r["precision"], case,
                                  footprint_of(case, r["precision"]), nx * ny * nz)
                        if s.footprint > self.budget:
                            rejected.append(s.rid)
                        else:
                            waiting.append(s)
                waiting.sort(key=lambda s: s.arrival)
                # issue one tick of every resident solve, each through its own graph (asynchronous)
                n = 0
                if active:
                    n = tick_length([s.remaining for s in active], self.tick_steps)
                    ta = now()
                    for s in active:
                        if s.batch is None:
                            tc = now()
                            s.batch = Batch([s.solver], steps_per_graph=self.tick_steps, dt_every=1)
                            host["batch_build_s"] += now() - tc
                        s.batch.advance(n)
                # admission by footprint, first come first served, while the tick runs; the
                # solves admitted now take their first step on their own streams and join the
                # next tick (memory of solves finishing in this tick is released after it)
                tadm = now()
                joining = []
                for _ in range(admit_fifo([w.footprint for w in waiting], used, self.budget)):
                    s = waiting.pop(0)
                    if self.tune:
                        s.tuning = autotune(s.case, precision=s.precision, cache=self.tune_cache)
                    s.solver = Solver.from_case(s.case, precision=s.precision)
                    if s.tuning:
                        s.solver.set_tuning(*s.tuning)
                    s.solver.init_run()
                    # the first step runs alone, so that the solve's graph only holds steady steps
                    s.solver.advance(1)
                    s.remaining = s.nsteps - 1
                    s.admitted = now()
                    used += s.footprint
                    joining.append(s)
                host["admit_s"] += now() - tadm
                if n:
                    for s in active:
                        s.batch.synchronize()
                    tb = now()
                    busy += tb - ta
                    self.log.append((ta, tb, len(active), n))
                    still = []
                    for s in active:
                        s.remaining -= n
                        if s.remaining > 0:
                            still.append(s)
                        else:
                            used -= self._finish(s, tb, done)
                    active = still
                # a one-step solve is complete after its first step
                for s in joining:
                    if s.remaining <= 0:
                        s.solver.synchronize()
                        used -= self._finish(s, now(), done)
                    else:
                        active.append(s)
                if not active and not joining:
                    # idle until the next arrival or finished set-up
                    if futures:
                        cf.wait(list(futures.values()), timeout=0.05, return_when=cf.FIRST_COMPLETED)
                    elif nxt < len(reqs):
                        time.sleep(max(0.0, min(0.05, reqs[nxt]["arrival"] * time_scale - now())))
        finally:
            for s in active:
                if s.batch is not None:
                    s.batch.close()
                if s.solver is not None:
                    s.solver.close()
            pool.shutdown(wait=True)
        out = summarize(done, rejected, busy, self.log)
        out.update(host)
        return out


    def _finish(self, s: Solve, t: float, done: list) -> int:
        """Record a completed solve, release its device memory; returns the bytes freed."""
        s.finished = t
        s.result["scalars"] = s.solver.scalars()
        if self.keep_fields:
            s.result["w"] = s.solver.copy_to_field()
        if s.batch is not None:
            s.batch.close()
            s.batch = None
        s.solver.close()
        s.solver = None
        done.append(s)
        return s.footprint


def admit_fifo(footprints: list[int], used: int, budget: int) -> int:
    """How many requests at the head of the queue (arrival order) are admitted now: strictly
    first come first served, so a large request is never overtaken by later small ones."""
    n = 0
    for f in footprints:
        if used + f > budget:
            break
        used += f
        n += 1
    return n


def tick_length(remaining: list[int], tick_steps: int) -> int:
    """Steps of the next tick: tick_steps, or fewer so that no resident solve overshoots."""
    return max(1, min([tick_steps] + list(remaining)))


def summarize(done: list[Solve], rejected: list[int], busy: float, log: list) -> dict:
    lat = np.array([s.finished - s.arrival for s in done]) if done else np.zeros(0)
    cell_steps = float(sum(s.cells * s.nsteps for s in done))
    span = (max(s.finished for s in done) - min(s.arrival for s in done)) if done else 0.0
    return {
        "completed": len(done),
        "rejected": rejected,
        "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
        "p99_s": float(np.percentile(lat, 99)) if lat.size else None,
        "mean_s": float(lat.mean()) if lat.size else None,
        "mcell_steps_per_s": cell_steps / span / 1e6 if span > 0 else None,
        "mcell_steps_per_busy_s": cell_steps / busy / 1e6 if busy > 0 else None,
        "span_s": span,
        "ticks": len(log),
        "max_resident": max((x[2] for x in log), default=0),
        "solves": {s.rid: s for s in done},
    }
