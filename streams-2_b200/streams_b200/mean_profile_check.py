"""Mean-profile agreement of the mixed form with the FP64 form over a long run.

    PYTHONPATH=streams-2_b200 python -m streams_b200.mean_profile_check --workload channel \\
        --size 512x256x256 --steps 5000 --dtstat-steps 10 --out profiles/mixed_mean_profile_5000.json

A thresholded hybrid scheme evaluated in FP32 switches some faces between the central and the
WENO flux differently from FP64 after a few steps, so the two fields decorrelate like two
turbulent realisations; what must agree is the mean flow.  Both precisions run the same case for
--steps steps from the same seeded field, sampling the running statistics (compute_stats, the
reference's 70 z- and time-averaged quantities) every --dtstat-steps steps, post-process them as
tools/postpro does (channel: stats1d profiles; boundary layer / shock interaction: stats2d skin
friction), and report the largest relative difference of each mean quantity, normalised by the
quantity's largest magnitude over the profile:
  channel    u/u0 (Favre), T/t0 (Favre), u'u'/tau_w and u_tau, over the half channel
  bl / sbli  cf(x) over all stations, the Favre u/u0 and T of the station in the middle of the
             box
"""
from __future__ import annotations

import argparse
import json
import re
import sys
import tempfile
import time
from pathlib import Path


def _ini(workload: str, nx: int, ny: int, nz: int, steps: int) -> str:
    from .cases import bl_ini, channel_ini
    if workload == "channel":
        return channel_ini(nx, ny, nz, num_iter=steps, print_control=max(1, steps))
    if workload == "sbli":
        return bl_ini(nx, ny, nz, mach=2.28, shock_angle=32.6, num_iter=steps, print_control=max(1, steps))
    return bl_ini(nx, ny, nz, num_iter=steps, print_control=max(1, steps))


def _with_dtstat(ini: str, dtstat: float) -> str:
    return re.sub(r"(?m)^dtstat\s*=.*$", f"dtstat = {dtstat!r}", ini)


def run_precision(workload, dims, steps, dtstat_steps, precision, workdir):
    """One run with statistics; returns the post-processed result and the run's clocks."""
    import numpy as np
    from . import Case, Solver, postpro
    nx, ny, nz = dims
    ini = _ini(workload, nx, ny, nz, steps)
    # the sampling interval in time units: dtstat_steps steps of the first step's dt
    probe = Case(workdir, ini)
    s = Solver.from_case(probe, precision=precision)
    s.init_run()
    dt0 = s.compute_dt()
    s.close()
    d = Path(workdir) / f"p{precision}"
    d.mkdir(parents=True, exist_ok=True)
    case = Case(d, _with_dtstat(ini, dtstat_steps * dt0 * 0.999))
    t0 = time.perf_counter()
    res = case.run_stats(steps, precision=precision)
    wall = time.perf_counter() - t0
    case.write_state_stats(res["w"], steps, float(res["row"][2]), res["w_stat"], None, res["itav"],
                           res["time_from_last_stat"], d)
    out = postpro.main(d, ixstat=[nx // 2] if workload != "channel" else None)
    out["samples"] = res["itav"]
    out["wall_s"] = wall
    out["x"] = np.loadtxt(d / "x.dat")[3:3 + nx] if workload != "channel" else None
    return out


def compare(workload, a, b, recyc_x=None):
    import numpy as np

    def rel(p, q):
        return float(np.max(np.abs(p - q)) / max(np.max(np.abs(q)), 1e-300))

    if workload == "channel":
        pa, pb = a["profile"], b["profile"]
        return {"u_favre": rel(pa[:, 2], pb[:, 2]), "t_favre": rel(pa[:, 3], pb[:, 3]),
                "uu_reynolds_stress": rel(pa[:, 20], pb[:, 20]),
                "u_tau": abs(a["info"]["utau"] - b["info"]["utau"]) / abs(b["info"]["utau"])}
    ca, cb = a["cf"], b["cf"]
    sel = np.ones(ca.shape[0], dtype=bool) if recyc_x is None else a["x"] > recyc_x
    out = {"cf": rel(ca[sel, 13], cb[sel, 13])}
    sa, sb = a.get("profiles", {}), b.get("profiles", {})
    for k in sa:
        out[f"station_{k}_u_favre"] = rel(sa[k][:, 2], sb[k][:, 2])
        out[f"station_{k}_t_favre"] = rel(sa[k][:, 4], sb[k][:, 4])
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="channel", choices=["channel", "bl", "sbli"])
    ap.add_argument("--size", default="512x256x256")
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--dtstat-steps", type=int, default=10)
    ap.add_argument("--out", default=None, help="JSON file to merge the result into")
    a = ap.parse_args(argv)
    dims = tuple(int(v) for v in a.size.lower().split("x"))
    with tempfile.TemporaryDirectory() as d:
        r64 = run_precision(a.workload, dims, a.steps, a.dtstat_steps, 0, d)
        r32 = run_precision(a.workload, dims, a.steps, a.dtstat_steps, 1, d)
    err = compare(a.workload, r32, r64)
    res = {"workload": a.workload, "size": a.size, "steps": a.steps, "stat_samples": r64["samples"],
           "max_rel_diff_mixed_vs_fp64": err, "wall_s": {"fp64": r64["wall_s"], "mixed": r32["wall_s"]},
           "command": "PYTHONPATH=streams-2_b200 python -m streams_b200.mean_profile_check " + " ".join(
               sys.argv[1:] if argv is None else argv)}
    print(json.dumps(res), flush=True)
    if a.out:
        p = Path(a.out)
        allres = json.loads(p.read_text()) if p.exists() else {}
        allres[f"{a.workload}_{a.size}"] = res
        p.write_text(json.dumps(allres, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
