"""Parity of the CUDA path (through the C ABI) with the CPU oracle on the same seeded inputs.

FP64 form: relative L2 of every conserved variable <= 1e-11 after 100 steps (the north-star
bound) and <= 1e-12 after one step; bulk quantities (dt, dpdx, rho_b, u_b, T_b) to 1e-11.
"""
import numpy as np
import pytest

from conftest import channel_ini, requires_gpu

pytestmark = [pytest.mark.gpu, requires_gpu]


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def interior(w, ng):
    return w[:, ng:-ng, ng:-ng, ng:-ng]


def run_pair(tmp_path, ini, nsteps):
    from oracle_py import Oracle
    from streams_b200 import Case, Solver
    case = Case(tmp_path, ini)
    o = Oracle(tmp_path, ini)
    s = Solver.from_case(case)
    o.init_run()
    s.init_run()
    o.run(nsteps)
    s.advance(nsteps, 1, 0, 0)
    return o, s


CASES = {
    # the benchmark channel's physics at a small size: power law, M_b 1.5, T_b held (force_var),
    # hybrid central/WENO with the Ducros threshold 0.05, near-wall order reduction
    "hybrid": dict(nx=32, ny=24, nz=16),
    "full_weno": dict(nx=24, ny=16, nz=12, sensor=-1.0),
    "full_central_sutherland": dict(nx=24, ny=20, nz=12, sensor=1.01, visc_model=2, theta_wall=-2.5,
                                    mach=0.5),
    "weno_z": dict(nx=24, ny=16, nz=12, sensor=-1.0, weno_version=1),
    "keep_enthalpy": dict(nx=24, ny=16, nz=12, nkeep=-1),
    "keep_n2": dict(nx=24, ny=16, nz=12, nkeep=2, sensor=1.01),
    "order4_weno2": dict(nx=24, ny=16, nz=12, ep_order=4, weno_scheme=2),
    "ragged": dict(nx=37, ny=13, nz=11),
    "no_order_reduction": dict(nx=24, ny=16, nz=12, correct_bound_ord=0),
    # conservative_viscous = 0: visflx_nosensor + visflx_div at visc_order, stage-3 sensor from them
    "nonconservative_viscous": dict(nx=32, ny=24, nz=16, conservative_viscous=0),
    "nonconservative_viscous_order4": dict(nx=24, ny=20, nz=16, conservative_viscous=0, ep_order=4,
                                           weno_scheme=2),
    # flux_splitting = 1: component-wise (Rusanov) WENO instead of the characteristic one
    "rusanov": dict(nx=32, ny=24, nz=16, flux_splitting=1),
    "rusanov_full_weno": dict(nx=24, ny=16, nz=12, sensor=-1.0, flux_splitting=1),
    # seventh-order WENO with the eighth-order central flux (ng = 4)
    "weno7_central8": dict(nx=32, ny=24, nz=16, weno_scheme=4, ep_order=8),
    "weno7_full": dict(nx=24, ny=16, nz=12, weno_scheme=4, ep_order=8, sensor=-1.0),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_one_step(name, tmp_path):
    o, s = run_pair(tmp_path, channel_ini(**CASES[name]), 1)
    ng = o.ng
    wo, wg = interior(o.w(), ng), interior(s.copy_to_field(), ng)
    for m in range(5):
        assert rel_l2(wg[m], wo[m]) <= 1e-12, (name, m, rel_l2(wg[m], wo[m]))
    so, sg = o.scalars(), s.scalars()
    for k in ("dt", "time", "dpdx", "rhobulk", "ubulk", "tbulk"):
        assert abs(sg[k] - so[k]) <= 1e-11 * max(abs(so[k]), 1e-30), (name, k, sg[k], so[k])


@pytest.mark.parametrize("name", ["hybrid", "full_weno", "full_central_sutherland", "nonconservative_viscous",
                                  "rusanov", "weno7_central8"])
def test_hundred_steps(name, tmp_path):
    o, s = run_pair(tmp_path, channel_ini(**CASES[name]), 100)
    ng = o.ng
    wo, wg = interior(o.w(), ng), interior(s.copy_to_field(), ng)
    errs = [rel_l2(wg[m], wo[m]) for m in range(5)]
    assert max(errs) <= 1e-11, (name, errs)
    so, sg = o.scalars(), s.scalars()
    for k in ("dt", "time", "rhobulk", "ubulk", "tbulk"):
        assert abs(sg[k] - so[k]) <= 1e-11 * max(abs(so[k]), 1e-30), (name, k, sg[k], so[k])


def test_residual_and_extrema(tmp_path):
    o, s = run_pair(tmp_path, channel_ini(nx=24, ny=16, nz=12), 3)
    ro, rg = o.residual(), s.compute_residual()
    for k in ro:
        assert abs(rg[k] - ro[k]) <= 1e-11 * max(abs(ro[k]), 1e-30), (k, rg[k], ro[k])
    assert not rg["nan"]


def test_wall_shear_matches(tmp_path):
    o, s = run_pair(tmp_path, channel_ini(nx=24, ny=16, nz=12), 2)
    a, b = o.wallprop(), s.wallprop()
    assert rel_l2(b, a) <= 1e-11


def test_golden_row_on_device(golden, tmp_path):
    """The reference's subsonic_channel golden row reproduced by the CUDA path."""
    from streams_b200 import Case
    case = Case(tmp_path, golden["ini"])
    row, _ = case.run(10)
    exp = np.array(golden["row"])
    assert row[0] == exp[0]
    tol = 1e-12 + 6e-11 * np.abs(exp[1:])
    assert np.all(np.abs(row[1:] - exp[1:]) <= tol), list(zip(row[1:], exp[1:]))


def test_deterministic_rerun(tmp_path):
    from streams_b200 import Case, Solver
    ini = channel_ini(nx=24, ny=16, nz=12)
    out = []
    for _ in range(2):
        case = Case(tmp_path, ini)
        s = Solver.from_case(case)
        s.init_run()
        s.advance(5)
        out.append(s.copy_to_field())
    assert np.array_equal(out[0], out[1])


def test_conservation_of_mass(tmp_path):
    """With the bulk forcing the mass is held: sum(rho * dy) stays at its initial value."""
    from streams_b200 import Case, Solver
    ini = channel_ini(nx=24, ny=16, nz=12)
    case = Case(tmp_path, ini)
    s = Solver.from_case(case)
    w0 = s.copy_to_field()
    s.init_run()
    s.advance(20)
    w1 = s.copy_to_field()
    ng = 3
    g = case.grid()
    ny = case.shape[1]
    dy = np.diff(np.ctypeslib.as_array(g.yn, shape=(ny + 1,)))
    # force_rhs removes the dy-weighted bulk mass source each stage (volchan = sum(dy) nx nz)
    m0 = (interior(w0, ng)[0] * dy[None, :, None]).sum()
    m1 = (interior(w1, ng)[0] * dy[None, :, None]).sum()
    assert abs(m1 - m0) <= 1e-12 * abs(m0)


def face_mask(nx, ny, nz, ng):
    """Interior and face-ghost points of a ghosted array (halo edges and corners excluded)."""
    k, j, i = np.meshgrid(np.arange(nz + 2 * ng), np.arange(ny + 2 * ng), np.arange(nx + 2 * ng), indexing="ij")
    out = ((i < ng) | (i >= nx + ng)).astype(int) + ((j < ng) | (j >= ny + ng)) + ((k < ng) | (k >= nz + ng))
    return out <= 1


def test_aux_sensor_after_init_and_rhs_after_one_step(tmp_path):
    """Stage-level parity: primitive fields and initial sensor after run()'s preamble, and the
    right-hand side of the last stage after one step."""
    from oracle_py import Oracle
    from streams_b200 import Case, Solver
    ini = channel_ini(nx=24, ny=16, nz=12)
    case = Case(tmp_path, ini)
    o = Oracle(tmp_path, ini)
    s = Solver.from_case(case)
    o.init_run()
    s.init_run()
    ng = 3
    mask = face_mask(24, 16, 12, ng)
    ag, ao = s.debug_fetch(0), o.waux()
    for m in range(7):
        assert rel_l2(ag[m][mask], ao[m][mask]) <= 1e-14, ("aux", m, rel_l2(ag[m][mask], ao[m][mask]))
    sg = s.debug_fetch(2)
    so = ao[7][ng:-ng, ng:-ng, ng:-ng]
    assert rel_l2(sg, so) <= 1e-12
    o.run(1)
    s.advance(1)
    fg, fo = s.debug_fetch(1), o.fl()
    for m in range(5):
        assert rel_l2(fg[m], fo[m]) <= 1e-12, ("fl", m, rel_l2(fg[m], fo[m]))


def test_restart_from_device_state(tmp_path):
    """A solve written out after 6 steps (rst.bin, field_info0.dat) resumes on the device and in
    the oracle from the same files; the two continuations agree."""
    from oracle_py import Oracle
    from streams_b200 import Case, Solver
    (tmp_path / "a").mkdir()
    (tmp_path / "r").mkdir()
    ini = channel_ini(nx=24, ny=16, nz=12)
    case = Case(tmp_path / "a", ini)
    s = Solver.from_case(case)
    s.init_run()
    s.advance(6)
    case.write_state(s.copy_to_field(), 6, s.scalars()["time"], tmp_path / "r")
    back = Case(tmp_path / "r")
    assert back.info()["icyc0"] == 6
    s2 = Solver.from_case(back)
    s2.set_time(back.info()["time0"])
    s2.init_run()
    s2.advance(4, 1, 6, 6)
    o = Oracle(tmp_path / "r")
    o.init_run()
    o.run(4)
    ng = o.ng
    wo, wg = interior(o.w(), ng), interior(s2.copy_to_field(), ng)
    for m in range(5):
        assert rel_l2(wg[m], wo[m]) <= 1e-12, (m, rel_l2(wg[m], wo[m]))
    assert abs(s2.scalars()["time"] - o.scalars()["time"]) <= 1e-12 * o.scalars()["time"]


def test_channel_128x96x64_hundred_steps(tmp_path):
    """The plain FP64 channel workload itself: 128x96x64, tanh 1.5 stretching, bulk Mach 1.5,
    bulk Re 3000, power law 0.76, Ducros threshold 0.05, CFL 0.8, +-10 % seeded noise (seed 1),
    T_b held by force_var; 100 steps.  Every conserved variable within 1e-11 relative L2 of the
    oracle, the bulk values and dpdx within 1e-11, the wall shear within 1e-11, and the bulk
    temperature held at its target by the device's force_var."""
    ini = channel_ini(nx=128, ny=96, nz=64, mach=1.5, re_bulk=3000.0, vt_exp=0.76, sensor=0.05, cfl=0.8,
                      seed=1, y_stretch=1.5, amp=0.1, theta_wall=0.0)
    o, s = run_pair(tmp_path, ini, 100)
    ng = o.ng
    wo, wg = interior(o.w(), ng), interior(s.copy_to_field(), ng)
    errs = [rel_l2(wg[m], wo[m]) for m in range(5)]
    assert max(errs) <= 1e-11, errs
    so, sg = o.scalars(), s.scalars()
    for k in ("dt", "time", "dpdx", "rhobulk", "ubulk", "tbulk"):
        assert abs(sg[k] - so[k]) <= 1e-11 * max(abs(so[k]), 1e-30), (k, sg[k], so[k])
    assert rel_l2(s.wallprop(), o.wallprop()) <= 1e-11
    # force_var on the device: sum(rho u T dy) / (volchan rho_b u_b) at the target
    from streams_b200 import Case
    case = Case(tmp_path, ini)
    p = case.params()
    dy = np.diff(np.ctypeslib.as_array(case.grid().yn, shape=(p.ny + 1,)))
    rho, ru, rv, rw, re = wg
    tt = p.t0 + (re / rho - 0.5 * ((ru / rho) ** 2 + (rv / rho) ** 2 + (rw / rho) ** 2) - p.cv_last * p.t0) / p.cv0
    tb = (ru * tt * dy[None, :, None]).sum() / p.volchan / sg["rhobulk"] / sg["ubulk"]
    assert abs(tb - p.t_bulk_target) <= 1e-12 * p.t_bulk_target, (tb, p.t_bulk_target)
