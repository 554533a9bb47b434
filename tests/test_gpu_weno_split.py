"""WENO faces computed apart (per-direction face lists, the face kernel and the face buffer read
by the hybrid passes) and WENO faces computed inside the hybrid passes, each against the oracle
and against each other, selected with streams_b200_set_weno_split (1: always apart, 0: always
inside).

Bounds (FP64, relative L2 of every conserved variable, interior points): <= 1e-12 after one
step and <= 1e-11 after 20 steps in either form, as for the hybrid scheme alone; the two forms
within 1e-13 of each other (the same arithmetic, which the compiler may contract differently in
the two kernels).  Mixed form: both forms <= 2e-6 against the oracle over the 10 steps before
any sensor crossing, and within 1e-6 of each other.
"""
import numpy as np
import pytest

from conftest import requires_gpu

pytestmark = [pytest.mark.gpu, requires_gpu]


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def case(name):
    from streams_b200.cases import SYNTHETIC_CP_POLY, bl_ini, channel_ini
    return {
        "channel": lambda: channel_ini(nx=32, ny=24, nz=16),
        "channel_weno_z": lambda: channel_ini(nx=32, ny=24, nz=16, weno_version=1, mach=2.5),
        "channel_order4_weno2": lambda: channel_ini(nx=24, ny=16, nz=12, ep_order=4, weno_scheme=2),
        "channel_order6_weno2": lambda: channel_ini(nx=24, ny=24, nz=16, weno_scheme=2),
        "channel_thermally_perfect": lambda: channel_ini(nx=32, ny=24, nz=16, cp_poly=SYNTHETIC_CP_POLY, mach=2.5),
        "bl": lambda: bl_ini(nx=48, ny=40, nz=16),
        "sbli": lambda: bl_ini(nx=48, ny=40, nz=16, mach=2.28, shock_angle=32.6, lx=60.0),
        "bl_rusanov": lambda: bl_ini(nx=48, ny=40, nz=16, flux_splitting=1),
        "bl_nonconservative": lambda: bl_ini(nx=48, ny=40, nz=16, conservative_viscous=0),
    }[name]()


def interior(o, w):
    g = o.ng
    return w[:, g:-g, g:-g, g:-g]


def run(tmp_path, ini, nsteps, frac, precision=0):
    from streams_b200 import Case, Solver
    s = Solver.from_case(Case(tmp_path, ini), precision=precision)
    s.set_weno_split(frac)
    assert s.get_weno_split() == frac
    s.init_run()
    s.advance(nsteps)
    return s.copy_to_field()


def oracle(tmp_path, ini, nsteps):
    from oracle_py import Oracle
    o = Oracle(tmp_path, ini)
    o.init_run()
    o.run(nsteps)
    return o


@pytest.mark.parametrize("name,nsteps,tol", [
    ("channel", 1, 1e-12), ("channel", 20, 1e-11), ("channel_weno_z", 20, 1e-11),
    ("channel_order4_weno2", 20, 1e-11), ("channel_order6_weno2", 20, 1e-11),
    ("channel_thermally_perfect", 20, 1e-11), ("bl", 1, 1e-12), ("bl", 20, 1e-11), ("sbli", 20, 1e-11),
    ("bl_rusanov", 20, 1e-11), ("bl_nonconservative", 20, 1e-11)])
def test_both_forms_match_the_oracle(name, nsteps, tol, tmp_path):
    ini = case(name)
    o = oracle(tmp_path, ini, nsteps)
    wo = interior(o, o.w())
    out = {}
    for frac in (0.0, 1.0):
        w = interior(o, run(tmp_path, ini, nsteps, frac))
        errs = [rel_l2(w[m], wo[m]) for m in range(5)]
        assert max(errs) <= tol, (frac, errs)
        out[frac] = w
    diff = [rel_l2(out[1.0][m], out[0.0][m]) for m in range(5)]
    assert max(diff) <= 1e-13, diff


def test_mixed_forms_agree(tmp_path):
    from streams_b200.cases import channel_ini
    ini = channel_ini(nx=32, ny=24, nz=16)
    o = oracle(tmp_path, ini, 10)
    wo = interior(o, o.w())
    out = {}
    for frac in (0.0, 1.0):
        w = interior(o, run(tmp_path, ini, 10, frac, precision=1))
        errs = [rel_l2(w[m], wo[m]) for m in range(5)]
        assert max(errs) <= 2e-6, (frac, errs)
        out[frac] = w
    diff = [rel_l2(out[1.0][m], out[0.0][m]) for m in range(5)]
    assert max(diff) <= 1e-6, diff


def test_the_default_threshold_and_its_limits(tmp_path):
    """On by default (0.55) from 2^21 cells, off (0) below; turning it on allocates the buffers."""
    from streams_b200 import BackendError, Case, Solver
    from streams_b200.cases import channel_ini
    big = Solver.from_case(Case(tmp_path, channel_ini(nx=128, ny=128, nz=128)))
    assert big.get_weno_split() == 0.55
    big.close()
    s = Solver.from_case(Case(tmp_path, channel_ini(nx=16, ny=12, nz=8)))
    assert s.get_weno_split() == 0.0
    for bad in (-0.1, 1.5, float("nan")):
        with pytest.raises(BackendError, match="max_fraction"):
            s.set_weno_split(bad)
    s.set_weno_split(0.3)
    assert s.get_weno_split() == 0.3


@pytest.mark.parametrize("frac", [1.0, 0.55])
def test_batch_with_the_split_equals_alone(frac, tmp_path):
    """The lists, samples and face kernels replayed from the batch graph (with a change of the
    fraction between replays, which recaptures it) give the bits of the box advanced alone."""
    from streams_b200 import Batch, Case, Solver
    from streams_b200.cases import bl_ini, channel_ini
    ini = bl_ini(nx=48, ny=40, nz=16, mach=2.28, shock_angle=32.6, lx=60.0)
    ch = channel_ini(nx=32, ny=24, nz=16)
    alone = []
    for case_ini in (ini, ch):
        a = Solver.from_case(Case(tmp_path, case_ini))
        a.set_weno_split(frac)
        a.init_run()
        a.advance(6)
        a.set_weno_split(0.3)
        a.advance(6)
        alone.append(a.copy_to_field())
    boxes = []
    for case_ini in (ini, ch):
        b = Solver.from_case(Case(tmp_path, case_ini))
        b.set_weno_split(frac)
        b.init_run()
        boxes.append(b)
    bt = Batch(boxes, steps_per_graph=5)
    bt.advance(6)
    for b in boxes:
        b.set_weno_split(0.3)
    bt.advance(6)
    bt.synchronize()
    for a, b in zip(alone, boxes):
        assert np.array_equal(a, b.copy_to_field())
