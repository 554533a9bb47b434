"""The boundary-layer boundary set on the GPU against the oracle: recycling-rescaling inflow
(z-shifted recycling plane, spanwise means, inner/outer rescaling, random plane drawn from the
continued glibc sequence every stage), zeroth-order extrapolation with the characteristic
non-reflecting correction at the outflow and top, the node-based isothermal wall, and the
impinging oblique shock at the top (shock / boundary-layer interaction).

Bounds as for the channel: relative L2 of every conserved variable <= 1e-12 after one step and
<= 1e-11 after 100 steps (FP64), including the stored inflow ghost planes.
"""
import numpy as np
import pytest

from conftest import requires_gpu

pytestmark = [pytest.mark.gpu, requires_gpu]


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bl(**kw):
    from streams_b200.cases import bl_ini
    base = dict(nx=48, ny=40, nz=16)
    base.update(kw)
    return bl_ini(**base)


def pair(tmp_path, ini, nsteps, precision=0):
    from oracle_py import Oracle
    from streams_b200 import Case, Solver
    case = Case(tmp_path, ini)
    o = Oracle(tmp_path, ini)
    s = Solver.from_case(case, precision=precision)
    o.init_run()
    s.init_run()
    o.run(nsteps)
    s.advance(nsteps)
    return o, s


def compare(o, s, tol):
    g = o.ng
    wo, wg = o.w(), s.copy_to_field()
    inner = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))
    errs = [rel_l2(wg[inner][m], wo[inner][m]) for m in range(5)]
    assert max(errs) <= tol, errs
    # the recycled inflow ghosts (i = 1-ng .. 0) and the extrapolated outflow ghosts
    for sl in (slice(0, g), slice(-g, None)):
        a, b = wg[:, g:-g, g:-g, sl], wo[:, g:-g, g:-g, sl]
        assert rel_l2(a, b) <= tol, rel_l2(a, b)
    return errs


SBLI = dict(mach=2.28, shock_angle=32.6, lx=60.0)  # an 8-degree deflection at Mach 2.28


@pytest.mark.parametrize("kw", [dict(), dict(nr_outflow=2, nr_top=3), dict(nr_outflow=6, nr_top=1),
                                dict(sensor=-1.0), dict(conservative_viscous=0), SBLI, dict(flux_splitting=1)],
                         ids=["nr1", "nr2_nr3", "nr6", "full_weno", "nonconservative", "sbli", "rusanov"])
def test_bl_one_step(kw, tmp_path):
    o, s = pair(tmp_path, bl(**kw), 1)
    compare(o, s, 1e-12)
    so, sg = o.scalars(), s.scalars()
    assert abs(sg["dt"] - so["dt"]) <= 1e-12 * so["dt"]


@pytest.mark.parametrize("kw", [dict(), SBLI], ids=["bl", "sbli"])
def test_bl_hundred_steps(kw, tmp_path):
    o, s = pair(tmp_path, bl(**kw), 100)
    compare(o, s, 1e-11)


def test_bl_wall_node_is_at_rest(tmp_path):
    from streams_b200 import Case, Solver
    s = Solver.from_case(Case(tmp_path, bl()))
    s.init_run()
    s.advance(3)
    w = s.copy_to_field()
    g = 3
    assert np.all(w[1:4, g:-g, g, g:-g] == 0.0)  # u, v, w at j = 1


def test_bl_batch_equals_alone(tmp_path):
    """The random inflow plane is drawn on the device, so a graph replay draws new numbers."""
    from streams_b200 import Batch, Case, Solver
    ini = bl()
    a = Solver.from_case(Case(tmp_path, ini))
    a.init_run()
    a.advance(12)
    b = Solver.from_case(Case(tmp_path, ini))
    b.init_run()
    bt = Batch([b], steps_per_graph=5)
    bt.advance(12)
    bt.synchronize()
    assert bt.stats()[0] == 2
    assert np.array_equal(a.copy_to_field(), b.copy_to_field())


def test_bl_mixed_central_100_steps(tmp_path):
    """Mixed form on the boundary layer, central scheme everywhere: <= 1e-5 relative L2."""
    o, s = pair(tmp_path, bl(sensor=1.01), 100, precision=1)
    g = o.ng
    wo, wg = o.w()[:, g:-g, g:-g, g:-g], s.copy_to_field()[:, g:-g, g:-g, g:-g]
    errs = [rel_l2(wg[m], wo[m]) for m in range(5)]
    assert max(errs) <= 1e-5, errs


@pytest.mark.parametrize("kw", [dict(), SBLI], ids=["bl", "sbli"])
def test_bl_hundred_steps_256x64x32(kw, tmp_path):
    """The boundary layer and the shock interaction at 256x64x32 (recycling station, NR outflow
    and top, node wall, shock), 100 steps within 1e-11."""
    o, s = pair(tmp_path, bl(nx=256, ny=64, nz=32, **kw), 100)
    compare(o, s, 1e-11)


def test_bl_inflow_draws_continue_the_setup_sequence(tmp_path):
    """The random inflow plane continues the crandom sequence after the set-up's draws (seed and
    draw count passed at create, as the Fortran object passes them): a context created with the
    set-up's count equals the oracle; one told that the set-up drew nothing draws other numbers."""
    from streams_b200 import Case, Solver
    ini = bl()
    case = Case(tmp_path, ini)
    o, s = pair(tmp_path, ini, 3)
    compare(o, s, 1e-12)
    p = case.params()
    assert p.rng_draws > 0 and p.rng_seed == 1
    p.rng_draws = 0
    s0 = Solver(p, case.grid(), keepalive=case)
    s0.copy_from_field(case.field())
    s0.init_run()
    s0.advance(3)
    g = o.ng
    a, b = s0.copy_to_field()[:, g:-g, g:-g, :g], s.copy_to_field()[:, g:-g, g:-g, :g]
    assert rel_l2(a, b) > 1e-6  # the inflow ghosts carry other random numbers


@pytest.mark.parametrize("example", ["supersonic_bl", "supersonic_sbli"])
def test_reference_example_inputs_ten_steps(example, tmp_path):
    """The reference's own boundary-layer and shock-interaction inputs (examples/supersonic_bl,
    supersonic_sbli: init_bl with hasan_meanprofile and the synthetic streaks, Sutherland
    viscosity, recycling inflow, NR outflow and top, impinging shock) with the grid reduced to
    256x64x32: 10 steps on the device against the oracle within 1e-12."""
    from conftest import ROOT
    ini = (ROOT / "tests" / "golden" / f"{example}.ini").read_text()
    o, s = pair(tmp_path, ini, 10)
    compare(o, s, 1e-12)
    so, sg = o.scalars(), s.scalars()
    assert abs(sg["dt"] - so["dt"]) <= 1e-12 * so["dt"]
