"""Serving form: a request loop over resident solves with continuous batching.

Requests (channel and shock-interaction solves of any size, Mach number, step count and
precision) arrive over time.  Each is prepared on the host as it arrives (input parsing, grid,
initial field: worker threads, so that set-up overlaps the GPU work), then admitted in arrival
order as soon as its device footprint fits the HBM budget next to the solves already resident;
its device set-up runs on an admission thread, off the loop.  A resident solve keeps its fields in
HBM from admission to completion and advances in ticks.  Resident solves of one class (the same
stage kernels: precision, scheme, channel forcing; Solver.batch_class) advance together: when the
class's previous tick is seen complete, its solves take their next tick as one cohort, a
``Batch`` over them whose stages run as shared launches (one launch per kernel kind and stage for
all of them, over a table of the solves' boxes), captured once per cohort membership.  A solve of
a class of its own, or of none (shock interactions: stored ghosts, non-reflecting faces), replays
its own CUDA graph of a tick's steps (a one-box ``Batch``) as soon as its stream reports the
previous tick complete.  Cohorts and lone solves overlap on the GPU.  A solve leaves, freeing its
memory, when its last tick is seen complete; completion latency is measured from the request's
arrival to then.

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
    cls: int | None = None          # class for shared launches (None: always alone)
    remaining: int = 0
    admitted: float = 0.0
    finished: float = 0.0
    tuning: tuple | None = None
    inflight: int = 0               # steps issued on the solve's stream and not yet seen complete
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
    tick_steps    steps a resident solve is given at a time (fewer when it completes sooner)
    tune          autotune each new (grid, precision) class before its first admission
    keep_fields   download each completed solve's conserved field into Solve.result["w"]
    shared        advance the resident solves of a class as one cohort with shared launches
                  (False: every solve on its own tick graph)

    The loop thread only decides and polls.  Host set-up runs on the preparation threads; an
    admitted solve's device set-up (tuning of a new class, context creation and upload,
    run() preamble, first step, capture of its tick graph and its first tick) runs on an
    admission thread.  A class's cohort (or a lone solve) is given its next tick as soon as its
    previous one has completed (non-blocking queries of the solves' streams), so no class waits
    for another, and a finishing solve releases its memory (stream-ordered, no device-wide
    synchronisation) the moment it is seen complete.
    """

    def __init__(self, budget_bytes: int, tick_steps: int = 10, tune: bool = True, keep_fields: bool = False,
                 prep_threads: int = 4, tune_cache: dict | None = None, admit_threads: int = 2,
                 shared: bool = True):
        self.budget = int(budget_bytes)
        self.shared = shared
        self._cohorts: dict[int, tuple[tuple[int, ...], Batch]] = {}  # class -> (members, batch)
        self.tick_steps = int(tick_steps)
        self.tune = tune
        self.keep_fields = keep_fields
        self.prep_threads = prep_threads
        self.admit_threads = admit_threads
        self.tune_cache = {} if tune_cache is None else tune_cache
        self.log: list[tuple] = []

    def _admit(self, s: Solve) -> Solve:
        """Device set-up of an admitted solve (admission thread): the solve is resident when this
        returns, with its first step and first tick issued on its own stream."""
        from .tune import autotune
        if self.tune:
            s.tuning = autotune(s.case, precision=s.precision, cache=self.tune_cache)
        s.solver = Solver.from_case(s.case, precision=s.precision)
        if s.tuning:
            s.solver.set_tuning(*s.tuning)
        s.solver.init_run()
        s.cls = s.solver.batch_class() if self.shared else None
        # the first step runs alone, so that the solve's graph only holds steady steps
        s.solver.advance(1)
        s.remaining = s.nsteps - 1
        s.inflight = 0
        if s.remaining > 0:
            s.batch = Batch([s.solver], steps_per_graph=self.tick_steps, dt_every=1)
            n = min(self.tick_steps, s.remaining)
            s.batch.advance(n)
            s.inflight = n
        return s

    def run(self, requests: list[dict], time_scale: float = 1.0) -> dict:
        """Serve `requests` (dicts with rid, arrival [s], nsteps, precision and channel
        parameters) with arrivals replayed in real time (scaled by time_scale); returns the
        per-request records and the latency / throughput summary."""
        reqs = sorted(requests, key=lambda r: r["arrival"])
        workdir = tempfile.mkdtemp(prefix="streams_b200_serve_")
        pool = cf.ThreadPoolExecutor(max_workers=self.prep_threads)
        admit_pool = cf.ThreadPoolExecutor(max_workers=self.admit_threads)
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        futures: dict[int, cf.Future] = {}
        admitting: dict[int, cf.Future] = {}
        waiting: list[Solve] = []      # prepared, not admitted (arrival order)
        active: list[Solve] = []
        done: list[Solve] = []
        rejected: list[int] = []
        used = 0
        nxt = 0
        busy = 0.0
        last = None  # start of the current interval with resident solves
        host = {"admit_wait_s": 0.0, "loop_iterations": 0, "cohort_ticks": 0, "max_cohort": 0}
        try:
            while nxt < len(reqs) or futures or waiting or admitting or active:
                host["loop_iterations"] += 1
                progressed = False
                # arrivals: start host set-up of every request whose arrival time has come
                while nxt < len(reqs) and reqs[nxt]["arrival"] * time_scale <= now():
                    r = reqs[nxt]
                    futures[r["rid"]] = pool.submit(prepare, r, workdir)
                    nxt += 1
                # prepared requests join the admission queue in arrival order
                for rid in [rid for rid, f in futures.items() if f.done()]:
                    r = next(q for q in reqs if q["rid"] == rid)
                    case = futures.pop(rid).result()
                    nx, ny, nz, _ = case.shape
                    sv = Solve(r["rid"], r["arrival"] * time_scale, r["nsteps"], r["precision"], case,
                               footprint_of(case, r["precision"]), nx * ny * nz)
                    if sv.footprint > self.budget:
                        rejected.append(sv.rid)
                    else:
                        waiting.append(sv)
                    progressed = True
                waiting.sort(key=lambda q: q.arrival)
                # admission by footprint, first come first served: the memory is reserved now,
                # the device set-up runs on an admission thread
                for _ in range(admit_fifo([q.footprint for q in waiting], used, self.budget)):
                    sv = waiting.pop(0)
                    used += sv.footprint
                    admitting[sv.rid] = admit_pool.submit(self._admit, sv)
                    progressed = True
                for rid in [rid for rid, f in admitting.items() if f.done()]:
                    sv = admitting.pop(rid).result()
                    sv.admitted = now()
                    active.append(sv)
                    progressed = True
                if active and last is None:
                    last = now()
                # every resident solve whose tick has completed gets its next one, or leaves; the
                # solves of a class move together, once all of them are seen complete
                still = []
                classes: dict[int, list[Solve]] = {}
                for sv in active:
                    if sv.cls is not None:
                        classes.setdefault(sv.cls, []).append(sv)
                        continue
                    if sv.inflight and sv.solver.busy():
                        still.append(sv)
                        continue
                    sv.remaining -= sv.inflight
                    sv.inflight = 0
                    progressed = True
                    if sv.remaining <= 0:
                        used -= self._finish(sv, now(), done)
                        continue
                    n = tick_length([sv.remaining], self.tick_steps)
                    sv.batch.advance(n)
                    sv.inflight = n
                    still.append(sv)
                for cls, members in classes.items():
                    if any(sv.inflight and sv.solver.busy() for sv in members):
                        still.extend(members)
                        continue
                    progressed = True
                    live = []
                    for sv in members:
                        sv.remaining -= sv.inflight
                        sv.inflight = 0
                        if sv.remaining > 0:
                            live.append(sv)
                    if len(live) != len(members):
                        self._drop_cohort(cls)  # before its finished solves' contexts go
                        for sv in members:
                            if sv.remaining <= 0:
                                used -= self._finish(sv, now(), done)
                    if not live:
                        continue
                    n = tick_length([sv.remaining for sv in live], self.tick_steps)
                    if len(live) == 1:
                        live[0].batch.advance(n)
                    else:
                        self._cohort(cls, live).advance(n)
                        host["cohort_ticks"] += 1
                        host["max_cohort"] = max(host["max_cohort"], len(live))
                    for sv in live:
                        sv.inflight = n
                    still.extend(live)
                if len(still) != len(active) or progressed:
                    self.log.append((now(), len(still)))
                active = still
                if not active and last is not None:
                    busy += now() - last
                    last = None
                if not progressed:
                    if admitting and not active:
                        tw = now()
                        cf.wait(list(admitting.values()), timeout=0.05, return_when=cf.FIRST_COMPLETED)
                        host["admit_wait_s"] += now() - tw
                    elif futures and not active:
                        cf.wait(list(futures.values()), timeout=0.05, return_when=cf.FIRST_COMPLETED)
                    elif not active and nxt < len(reqs):
                        time.sleep(max(0.0, min(0.05, reqs[nxt]["arrival"] * time_scale - now())))
                    else:
                        time.sleep(0.0002)
            if last is not None:
                busy += now() - last
        finally:
            for f in admitting.values():
                sv = f.result()
                active.append(sv)
            for cls in list(self._cohorts):
                self._drop_cohort(cls)
            for sv in active:
                if sv.batch is not None:
                    sv.batch.close()
                if sv.solver is not None:
                    sv.solver.close()
            admit_pool.shutdown(wait=True)
            pool.shutdown(wait=True)
        out = summarize(done, rejected, busy, self.log)
        out.update(host)
        return out

    def _cohort(self, cls: int, live: list[Solve]) -> Batch:
        """The class's cohort batch over exactly the solves `live` (rebuilt when they change)."""
        key = tuple(sv.rid for sv in live)
        cur = self._cohorts.get(cls)
        if cur is not None and cur[0] == key:
            return cur[1]
        self._drop_cohort(cls)
        b = Batch([sv.solver for sv in live], steps_per_graph=self.tick_steps, dt_every=1)
        self._cohorts[cls] = (key, b)
        return b

    def _drop_cohort(self, cls: int) -> None:
        cur = self._cohorts.pop(cls, None)
        if cur is not None:
            cur[1].close()

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
        "max_resident": max((x[1] for x in log), default=0),
        "solves": {s.rid: s for s in done},
    }
