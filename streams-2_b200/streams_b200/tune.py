"""Autotuner of the flux passes' launch shape.

The y and z flux passes march along grid lines; each line is cut into segments so that about
``march_threads`` threads run, every segment at least ``march_minseg`` cells long (the pencil
tile of the march).  The best cut depends on the box's shape and precision: short segments
give more threads for small boxes, long ones re-load fewer halo points.  ``autotune`` times
each candidate on a scratch copy of the box (its own context, so the solve being tuned is not
advanced) with the library's CUDA-event profiler and keeps the fastest; results are cached
per (grid, precision, scheme).  A tuning changes only the thread partition: boxes with equal
tunings give bit-identical results, different tunings differ in the summation order of the
bulk-forcing block partials.  Boxes of one tuning class (sizes within a factor sqrt(2) of the
same powers of two) share a tuning.
"""
from __future__ import annotations

import math

from . import Solver

# march_threads x march_minseg candidates (148 SMs x 256 .. 2048 threads; segments 8 .. 32)
CANDIDATES = [(t, m) for t in (37888, 75776, 151552, 303104) for m in (8, 16, 32)]
DEFAULT = (151552, 16)

_cache: dict[tuple, tuple[int, int]] = {}


def key_of(params) -> tuple:
    """Tuning class of a box: grid sizes rounded to the nearest power of two (the launch shape
    depends on the line counts and lengths, not on their exact values), precision and scheme."""
    b = lambda n: int(round(math.log2(max(n, 1))))
    return (b(params.nx), b(params.ny), b(params.nz), params.precision, params.ep_order, params.weno_scheme,
            params.nkeep, params.weno_version)


def march_time_ms(solver: Solver, steps: int) -> float:
    """Device time of the y and z flux passes over `steps` steps (CUDA events)."""
    solver.profile(-1)
    solver.profile(1)
    solver.advance(steps)
    solver.synchronize()
    rep = solver.profile_report()
    solver.profile(0)
    return sum(rep.get(k, (0.0, 0))[0] for k in ("k_euler_y", "k_euler_z"))


def autotune(case, precision: int = 0, steps: int = 2, candidates=CANDIDATES,
             cache: dict | None = None) -> tuple[int, int]:
    """Best (march_threads, march_minseg) for boxes like `case` at `precision`; cached."""
    cache = _cache if cache is None else cache
    k = key_of(case.params(precision))
    if k in cache:
        return cache[k]
    scratch = Solver.from_case(case, precision=precision)
    try:
        scratch.init_run()
        scratch.advance(1)  # warm-up: the steady step sequence
        best, best_ms = DEFAULT, float("inf")
        for cand in candidates:
            scratch.set_tuning(*cand)
            scratch.advance(1)
            ms = march_time_ms(scratch, steps)
            if ms < best_ms:
                best, best_ms = cand, ms
    finally:
        scratch.close()
    cache[k] = best
    return best


def tune_solver(solver: Solver, case, cache: dict | None = None) -> tuple[int, int]:
    """Tune `solver` (built from `case`) through a scratch twin, and apply the result."""
    t = autotune(case, precision=solver.params.precision, cache=cache)
    solver.set_tuning(*t)
    return t
