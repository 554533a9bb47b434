"""Running statistics on the GPU against the oracle: compute_stats (70 z-averaged quantities,
code/src/singleideal/singleideal.F90:2003-2179) and compute_stats_3d (14 point quantities,
:2513-2543), sampled after steps and averaged in time, on the channel (periodic x and z whose
ghost layers the kernel rebuilds as the bcswap of stage 3 left them, staggered walls, force_var
temperature) and on the boundary layer (recycling inflow, extrapolated outflow and top with the
non-reflecting correction, node-based wall, periodic z).

Bound (FP64): per statistic, max |device - oracle| over the (i, j) plane <= 1e-11 of the
statistic's largest magnitude after 3 samples.  Mixed form (FP32 aux temperature and viscosity,
FP32 fluxes): <= 1e-4 for the statistics that do not difference the velocity (1-21, 25-42,
66-70) after one step.
"""
import numpy as np
import pytest

from conftest import channel_ini, requires_gpu
from test_oracle_stats import stat_err

pytestmark = [pytest.mark.gpu, requires_gpu]


def bl(**kw):
    from streams_b200.cases import bl_ini
    base = dict(nx=48, ny=40, nz=16)
    base.update(kw)
    return bl_ini(**base)


CASES = {
    "channel": lambda: channel_ini(nx=32, ny=24, nz=16),
    "channel_no_force_var": lambda: channel_ini(nx=32, ny=24, nz=16, theta_wall=-2.0),
    "channel_order4": lambda: channel_ini(nx=32, ny=24, nz=16, ep_order=4, weno_scheme=2),
    "bl": lambda: bl(),
    "sbli": lambda: bl(mach=2.28, shock_angle=32.6, lx=60.0),
}


def sampled_pair(tmp_path, ini, nsamples, precision=0, three_d=True):
    from oracle_py import Oracle
    from streams_b200 import Case, Solver
    case = Case(tmp_path, ini)
    o = Oracle(tmp_path, ini)
    s = Solver.from_case(case, precision=precision)
    o.init_run()
    s.init_run()
    for itav in range(nsamples):
        o.run(1)
        s.advance(1)
        o.compute_stats(itav)
        s.compute_stats(itav)
        if three_d:
            o.compute_stats_3d(itav)
            s.compute_stats_3d(itav)
    return o, s


@pytest.mark.parametrize("name", sorted(CASES))
def test_stats_match_oracle(name, tmp_path):
    o, s = sampled_pair(tmp_path, CASES[name](), 3)
    for which in (0, 1, 2):
        err = stat_err(s.stats(which), o.stats(which))
        assert err.max() <= 1e-11, (name, which, int(err.argmax()) + 1, float(err.max()))


def test_stats_after_a_download_equal_stats_before(tmp_path):
    """A download between the step and the sample (manage_output writes fields before it samples)
    leaves the sampled state alone: same statistics bit for bit."""
    from streams_b200 import Case, Solver
    ini = CASES["channel"]()
    out = []
    for download in (False, True):
        s = Solver.from_case(Case(tmp_path, ini))
        s.init_run()
        s.advance(2)
        if download:
            s.copy_to_field()
        s.compute_stats(0)
        s.compute_stats_3d(0)
        out.append((s.stats(0), s.stats(2)))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_stats_need_a_completed_step(tmp_path):
    from streams_b200 import BackendError, Case, Solver
    s = Solver.from_case(Case(tmp_path, CASES["channel"]()))
    s.init_run()
    with pytest.raises(BackendError, match="rk_sync"):
        s.compute_stats(0)
    s.advance(1)
    s.compute_dt()  # the next step has started: the sampled state is gone
    with pytest.raises(BackendError, match="rk_sync"):
        s.compute_stats(0)


def test_mixed_stats(tmp_path):
    o, s = sampled_pair(tmp_path, CASES["channel"](), 1, precision=1, three_d=False)
    err = stat_err(s.stats(0), o.stats(0))
    direct = [l - 1 for l in list(range(1, 22)) + list(range(25, 43)) + list(range(66, 71))]
    assert err[direct].max() <= 1e-4, (direct[int(np.argmax(err[direct]))] + 1, float(err[direct].max()))


def test_run_case_samples_as_manage_output(tmp_path):
    """The host run loop samples with the reference's clock (time_from_last_stat += dt, a sample
    when it reaches dtstat): with dtstat below every dt each step is a sample, equal to sampling
    by hand; the end-of-run files (rst.bin, stat.bin, stat3d.bin, field_info0.dat) resume the
    averaging with restart_type = 2."""
    import re
    from streams_b200 import Case, Solver
    ini = CASES["channel"]().replace("dtstat = 50.", "dtstat = 1e-12\nenable_stat_3d = 1")
    case = Case(tmp_path, ini)
    a = tmp_path / "a"
    a.mkdir()
    case.write_restart(a)  # grid files and the input of the restart
    r = case.run_stats(nsteps=3, output_dir=a)
    assert r["itav"] == 3 and r["time_from_last_stat"] == 0.0
    s = Solver.from_case(Case(tmp_path, ini))
    s.init_run()
    for itav in range(3):
        s.advance(1)
        s.compute_stats(itav)
        s.compute_stats_3d(itav)
    assert np.array_equal(r["w_stat"], s.stats(0))
    assert np.array_equal(r["w_stat_3d"], s.stats(2))
    # resume from the end-of-run files: two more samples continue the average of the first three
    text = re.sub(r"restart_type\s*=\s*\d", "restart_type = 2", (a / "singleideal.ini").read_text())
    back = Case(a, text)
    info = back.stats_info()
    assert info["itav"] == 3 and info["enable_stat_3d"] == 1
    assert np.array_equal(back.restart_stats(0), r["w_stat"])
    assert np.array_equal(back.field()[:, 3:-3, 3:-3, 3:-3], r["w"][:, 3:-3, 3:-3, 3:-3])
    r2 = back.run_stats(nsteps=2)
    assert r2["itav"] == 5
    t = Solver.from_case(back)
    t.set_stats(0, back.restart_stats(0))
    t.set_stats(2, back.restart_stats(2))
    t.init_run()
    for itav in range(3, 5):
        t.advance(1)
        t.compute_stats(itav)
        t.compute_stats_3d(itav)
    assert np.array_equal(r2["w_stat"], t.stats(0))
    assert np.array_equal(r2["w_stat_3d"], t.stats(2))
