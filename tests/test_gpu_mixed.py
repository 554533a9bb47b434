"""The mixed-precision form (FP32 flux and viscous arithmetic; FP64 state, RK register,
temperature recovery, Ducros sensor, time step and reductions) against the FP64 oracle.

Stated tolerances (relative L2 per conserved variable, interior points):
  * one fixed scheme everywhere (central only, or WENO only): <= 1e-5 after 100 steps for
    rho, rho*u, rho*E and the central rho*v, rho*w; <= 2e-5 for the WENO-only rho*v, rho*w
    (the transverse momenta are perturbation-sized, so their relative error is the largest);
    bulk rho_b, u_b, T_b within 1e-6 relative, wall shear within 1e-5.
  * the hybrid scheme: <= 2e-6 while no point's sensor has crossed the threshold differently
    from the FP64 run (10 steps here).  A crossing switches one face between the central and
    the WENO flux, an O(1) local change, so after 100 steps the hybrid fields only agree to
    <= 1e-3 (rho, rho*u, rho*E) and <= 2e-2 (rho*v, rho*w); bulk quantities within 1e-4.
"""
import numpy as np
import pytest

from conftest import channel_ini, requires_gpu

pytestmark = [pytest.mark.gpu, requires_gpu]


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run_gpu(tmp_path, ini, nsteps, precision):
    from streams_b200 import Case, Solver
    case = Case(tmp_path, ini)
    s = Solver.from_case(case, precision=precision)
    s.init_run()
    s.advance(nsteps)
    return s


def errors_vs_oracle(tmp_path, ini, nsteps):
    from oracle_py import Oracle
    o = Oracle(tmp_path, ini)
    o.init_run()
    o.run(nsteps)
    s = run_gpu(tmp_path, ini, nsteps, precision=1)
    g = o.ng
    wo = o.w()[:, g:-g, g:-g, g:-g]
    wm = s.copy_to_field()[:, g:-g, g:-g, g:-g]
    errs = [rel_l2(wm[m], wo[m]) for m in range(5)]
    so, sm = o.scalars(), s.scalars()
    bulk = {k: abs(sm[k] - so[k]) / abs(so[k]) for k in ("dt", "time", "rhobulk", "ubulk", "tbulk")}
    return errs, bulk, o, s


FIXED = [
    ("central", dict(nx=32, ny=24, nz=16, sensor=1.01), [1e-5] * 5),
    ("weno", dict(nx=24, ny=16, nz=12, sensor=-1.0), [1e-5, 1e-5, 2e-5, 2e-5, 1e-5]),
    ("central_sutherland_cold_wall", dict(nx=24, ny=20, nz=12, sensor=1.01, visc_model=2, theta_wall=-2.5,
                                          mach=0.5), [1e-5] * 5),
    ("central_nonconservative_viscous", dict(nx=32, ny=24, nz=16, sensor=1.01, conservative_viscous=0),
     [1e-5] * 5),
]


@pytest.mark.parametrize("name,kw,tol", FIXED, ids=[f[0] for f in FIXED])
def test_mixed_fixed_scheme_100_steps(name, kw, tol, tmp_path):
    errs, bulk, o, s = errors_vs_oracle(tmp_path, channel_ini(**kw), 100)
    assert all(e <= t for e, t in zip(errs, tol)), (errs, tol)
    for k in ("rhobulk", "ubulk", "tbulk"):
        assert bulk[k] <= 1e-6, (k, bulk)
    a, b = o.wallprop(), s.wallprop()
    for m in range(a.shape[0]):
        assert rel_l2(b[m], a[m]) <= 1e-5, m


def test_mixed_hybrid_before_threshold_crossings(tmp_path):
    errs, bulk, _, _ = errors_vs_oracle(tmp_path, channel_ini(nx=32, ny=24, nz=16), 10)
    assert max(errs) <= 2e-6, errs
    for k in ("rhobulk", "ubulk", "tbulk"):
        assert bulk[k] <= 1e-6, (k, bulk)


def test_mixed_hybrid_100_steps(tmp_path):
    errs, bulk, _, _ = errors_vs_oracle(tmp_path, channel_ini(nx=32, ny=24, nz=16), 100)
    assert max(errs[0], errs[1], errs[4]) <= 1e-3, errs
    assert max(errs[2], errs[3]) <= 2e-2, errs
    for k in ("rhobulk", "ubulk", "tbulk"):
        assert bulk[k] <= 1e-4, (k, bulk)


def test_mixed_is_deterministic_and_differs_from_fp64(tmp_path):
    ini = channel_ini(nx=24, ny=16, nz=12)
    a = run_gpu(tmp_path, ini, 3, 1).copy_to_field()
    b = run_gpu(tmp_path, ini, 3, 1).copy_to_field()
    c = run_gpu(tmp_path, ini, 3, 0).copy_to_field()
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)  # the FP32 path really runs


def test_mixed_aux_is_fp32_and_sensor_fp64(tmp_path):
    ini = channel_ini(nx=24, ny=16, nz=12)
    s = run_gpu(tmp_path, ini, 1, 1)
    aux = s.debug_fetch(0)
    x = aux[1][3:-3, 3:-3, 3:-3].ravel()
    assert np.array_equal(x.astype(np.float32).astype(np.float64), x)
    # the sensor is computed in FP64 from the FP64 state: it matches the FP64 form's initial sensor
    a = run_gpu(tmp_path, ini, 0, 0).debug_fetch(2)
    b = run_gpu(tmp_path, ini, 0, 1).debug_fetch(2)
    assert rel_l2(b, a) <= 1e-14
