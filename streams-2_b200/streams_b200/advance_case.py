"""Advance one synthetic case on the device: the driver of the profiling commands.

    PYTHONPATH=streams-2_b200 python -m streams_b200.advance_case --workload bl --size 256x128x96 \\
        --steps 300 --then 2 [--precision 1] [--weno-split 0.55]

Builds the case's input file (``streams_b200.cases``), runs ``init_run``, advances ``--steps``
steps, prints the WENO face fractions (``count_weno``), then advances ``--then`` more steps and
synchronises.  Under ``ncu -s <launches> -c <n>`` the captured launches are those of the
``--then`` steps; the workloads are the benchmark's (channel, boundary layer, shock interaction).
"""
from __future__ import annotations

import argparse
import sys
import tempfile


def build_ini(workload: str, nx: int, ny: int, nz: int) -> str:
    from streams_b200.cases import bl_ini, channel_ini
    if workload == "channel":
        return channel_ini(nx, ny, nz)
    if workload == "sbli":
        return bl_ini(nx, ny, nz, mach=2.28, shock_angle=32.6)
    if workload == "bl":
        return bl_ini(nx, ny, nz)
    raise ValueError(f"unknown workload {workload!r} (channel, bl, sbli)")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="bl", choices=["channel", "bl", "sbli"])
    ap.add_argument("--size", default="256x128x96", help="nx x ny x nz")
    ap.add_argument("--steps", type=int, default=0, help="steps before the WENO face count")
    ap.add_argument("--then", type=int, default=2, help="steps after it (the profiled ones)")
    ap.add_argument("--precision", type=int, default=0, help="0 FP64, 1 mixed")
    ap.add_argument("--weno-split", type=float, default=None,
                    help="WENO split threshold (0 off); the default is the library's choice")
    a = ap.parse_args(argv)
    from streams_b200 import Case, Solver
    nx, ny, nz = (int(v) for v in a.size.lower().split("x"))
    with tempfile.TemporaryDirectory() as d:
        case = Case(d, build_ini(a.workload, nx, ny, nz))
        s = Solver.from_case(case, precision=a.precision)
        if a.weno_split is not None:
            s.set_weno_split(a.weno_split)
        s.init_run()
        if a.steps:
            s.advance(a.steps)
        frac = s.count_weno()
        print(f"{a.workload} {nx}x{ny}x{nz} precision {a.precision}: WENO face fraction x/y/z after "
              f"{a.steps} steps = " + " / ".join(f"{v:.3f}" for v in frac), flush=True)
        if a.then:
            s.advance(a.then)
        s.synchronize()
    return 0


if __name__ == "__main__":
    sys.exit(main())
