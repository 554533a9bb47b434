"""Thermally perfect gas (calorically_perfect = 0, cp(T) polynomial) on the GPU against the
oracle: Newton temperature recovery in the aux pass, the walls and the energy shift, the Newton
Roe-averaged temperature and gamma(T) of the characteristic and component-wise WENO fluxes,
cp(T) in the viscous terms, gamma(T) in the time step, the non-reflecting boundaries and the
statistics.

Bounds as for the calorically perfect gas (FP64): relative L2 of every conserved variable
<= 1e-12 after one step and <= 1e-11 after 20 steps; statistics <= 1e-11 of each statistic's
largest magnitude.  A constant polynomial equal to the calorically perfect gas reproduces that
gas's device run to 1e-12.
"""
import numpy as np
import pytest

from conftest import requires_gpu
from test_oracle_stats import stat_err

pytestmark = [pytest.mark.gpu, requires_gpu]


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def channel(**kw):
    from streams_b200.cases import SYNTHETIC_CP_POLY, channel_ini
    base = dict(nx=32, ny=24, nz=16, cp_poly=SYNTHETIC_CP_POLY, mach=2.5)
    base.update(kw)
    return channel_ini(**base)


def bl(**kw):
    from streams_b200.cases import SYNTHETIC_CP_POLY, bl_ini
    base = dict(nx=48, ny=40, nz=16, cp_poly=SYNTHETIC_CP_POLY)
    base.update(kw)
    return bl_ini(**base)


CASES = {
    "channel_hybrid": lambda: channel(),
    "channel_full_weno": lambda: channel(sensor=-1.0),
    "channel_rusanov": lambda: channel(sensor=-1.0, flux_splitting=1),
    "channel_nonconservative": lambda: channel(conservative_viscous=0),
    "bl": lambda: bl(),
    "sbli": lambda: bl(mach=2.28, shock_angle=32.6, lx=60.0),
}


def pair(tmp_path, ini, nsteps):
    from oracle_py import Oracle
    from streams_b200 import Case, Solver
    case = Case(tmp_path, ini)
    o = Oracle(tmp_path, ini)
    s = Solver.from_case(case)
    o.init_run()
    s.init_run()
    o.run(nsteps)
    s.advance(nsteps)
    return o, s


def field_errors(o, s):
    g = o.ng
    wo, wg = o.w(), s.copy_to_field()
    inner = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))
    return [rel_l2(wg[inner][m], wo[inner][m]) for m in range(5)]


@pytest.mark.parametrize("name", sorted(CASES))
def test_one_step(name, tmp_path):
    o, s = pair(tmp_path, CASES[name](), 1)
    errs = field_errors(o, s)
    assert max(errs) <= 1e-12, (name, errs)


@pytest.mark.parametrize("name", ["channel_hybrid", "bl"])
def test_twenty_steps(name, tmp_path):
    o, s = pair(tmp_path, CASES[name](), 20)
    errs = field_errors(o, s)
    assert max(errs) <= 1e-11, (name, errs)
    so, sg = o.scalars(), s.scalars()
    assert sg["dt"] == pytest.approx(so["dt"], rel=1e-11)


@pytest.mark.parametrize("name", ["channel_hybrid", "bl"])
def test_statistics(name, tmp_path):
    from oracle_py import Oracle
    from streams_b200 import Case, Solver
    ini = CASES[name]()
    o = Oracle(tmp_path, ini)
    s = Solver.from_case(Case(tmp_path, ini))
    o.init_run()
    s.init_run()
    for itav in range(2):
        o.run(1)
        s.advance(1)
        o.compute_stats(itav)
        s.compute_stats(itav)
    err = stat_err(s.stats(0), o.stats(0))
    assert err.max() <= 1e-11, (int(err.argmax()) + 1, float(err.max()))


def test_constant_polynomial_matches_the_calorically_perfect_gas(tmp_path):
    from streams_b200 import Case, Solver
    from streams_b200.cases import channel_ini
    out = []
    for poly in (None, (-2, 2, (0.0, 0.0, 3.5, 0.0, 0.0, 0.0))):
        s = Solver.from_case(Case(tmp_path, channel_ini(nx=32, ny=24, nz=16, cp_poly=poly, sensor=-1.0)))
        s.init_run()
        s.advance(5)
        out.append(s.copy_to_field())
    errs = [rel_l2(out[1][m], out[0][m]) for m in range(5)]
    assert max(errs) <= 1e-12, errs
