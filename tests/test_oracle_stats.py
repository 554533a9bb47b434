"""Running statistics on the CPU: the oracle's compute_stats / compute_stats_3d
(code/src/singleideal/singleideal.F90:2003-2179, 2513-2543) against an independent numpy
restatement, the state they sample (the ghost layers and temperatures a step leaves behind, which
the device kernel rebuilds), the time average, and the stat.bin / stat3d.bin restart files."""
import numpy as np
import pytest

from conftest import channel_ini

NV = 70


def bl_ini(**kw):
    from streams_b200.cases import bl_ini as build
    return build(**kw)


def numpy_stats(o, case):
    """compute_stats of one sample from the oracle's w (ghosts included) and w_aux(6), w_aux(7):
    the 70 quantities z-averaged, as (ny, nx, 70)."""
    g = case.grid()
    p = case.params()
    nx, ny, nz, ng = o.nx, o.ny, o.nz, o.ng
    lmax = p.ep_order // 2
    coeff = np.ctypeslib.as_array(g.coeff_deriv1, shape=(16,)).reshape(4, 4)
    dcsidx = np.ctypeslib.as_array(g.dcsidx, shape=(nx,))
    detady = np.ctypeslib.as_array(g.detady, shape=(ny,))
    dzitdz = np.ctypeslib.as_array(g.dzitdz, shape=(nz,))
    w = o.w()
    aux = o.waux()
    vel = [w[m] / w[0] for m in (1, 2, 3)]
    I = slice(ng, ng + nx)
    J = slice(ng, ng + ny)
    K = slice(ng, ng + nz)

    def deriv(f, axis):
        acc = np.zeros((nz, ny, nx))
        for l in range(1, lmax + 1):
            c = coeff[lmax - 1, l - 1]
            if axis == 0:
                d = f[K, J, ng + l:ng + l + nx] - f[K, J, ng - l:ng - l + nx]
            elif axis == 1:
                d = f[K, ng + l:ng + l + ny, I] - f[K, ng - l:ng - l + ny, I]
            else:
                d = f[ng + l:ng + l + nz, J, I] - f[ng - l:ng - l + nz, J, I]
            acc = acc + c * d
        return acc

    ux, vx, wx = (deriv(v, 0) * dcsidx[None, None, :] for v in vel)
    uy, vy, wy = (deriv(v, 1) * detady[None, :, None] for v in vel)
    uz, vz, wz = (deriv(v, 2) * dzitdz[:, None, None] for v in vel)
    omx, omy, omz = wy - vz, uz - wx, vx - uy
    rho, rhou, rhov, rhow = (w[m][K, J, I] for m in range(4))
    uu, vv, ww = rhou / rho, rhov / rho, rhow / rho
    qq = 0.5 * (uu * uu + vv * vv + ww * ww)
    tt = aux[5][K, J, I]
    mu = aux[6][K, J, I]
    pp = rho * p.rgas0 * tt
    nu = mu / rho
    gam = p.cp0 / (p.cp0 - p.rgas0)
    cp = gam / (gam - 1.0) * p.rgas0
    mach = np.sqrt(2.0 * qq) / np.sqrt(gam * p.rgas0 * tt)
    ttot = tt + qq * (gam - 1.0) / gam
    div = ux + vy + wz
    s11, s22, s33 = (2.0 * (a - div / 3.0) * mu for a in (ux, vy, wz))
    s12, s13, s23 = (uy + vx) * mu, (uz + wx) * mu, (vz + wy) * mu
    one = np.ones_like(rho)
    q = [rho, uu, vv, ww, pp, tt, rho ** 2, uu ** 2, vv ** 2, ww ** 2, pp ** 2, tt ** 2, rhou, rhov, rhow,
         rhou * uu, rhov * vv, rhow * ww, rhou * vv, mu, nu, omx ** 2, omy ** 2, omz ** 2, rho * tt, rho * tt ** 2,
         ttot, rho * ttot, ttot ** 2, rhou * tt, rhov * tt, rhow * tt, mach, mach ** 2, rhou * uu ** 2,
         rhov * uu ** 2, rhou * vv ** 2, rhov * vv ** 2, rhou * ww ** 2, rhov * ww ** 2, pp * uu, pp * vv,
         s11, s12, s13, s22, s23, s33, s11 * uu, s12 * uu, s12 * vv, s22 * vv, s13 * ww, s23 * ww,
         s11 * vv + s12 * uu, s12 * vv + s22 * uu, s11 * ux + s12 * uy + s13 * uz, s12 * vx + s22 * vy + s23 * vz,
         s13 * wx + s23 * wy + s33 * wz, s11 * vx + s12 * (ux + vy) + s22 * uy + s13 * vz + s23 * uz,
         pp * ux, pp * vy, pp * wz, pp * (uy + vx), div * div, rho * tt ** 3, rho * tt ** 4, rhou * uu ** 3,
         cp * one, gam * one]
    assert len(q) == NV
    return np.stack([a.sum(axis=0) / nz for a in q], axis=-1)


def stat_err(a, b):
    """Per statistic: max |a - b| over the plane relative to max |b| (floor 1e-300)."""
    d = np.abs(a - b).reshape(-1, a.shape[-1]).max(axis=0)
    s = np.abs(b).reshape(-1, b.shape[-1]).max(axis=0)
    return d / np.maximum(s, 1e-300)


@pytest.mark.parametrize("kind", ["channel", "bl"])
def test_oracle_stats_match_numpy(tmp_path, kind):
    from oracle_py import Oracle
    from streams_b200 import Case
    ini = channel_ini(nx=16, ny=12, nz=8) if kind == "channel" else bl_ini(nx=32, ny=24, nz=8)
    case = Case(tmp_path, ini)
    o = Oracle(tmp_path, ini)
    o.init_run()
    o.run(2)
    o.compute_stats(0)
    ref = numpy_stats(o, case)
    got = o.stats(0)
    err = stat_err(got, ref)
    assert err.max() <= 1e-12, (int(err.argmax()) + 1, err.max())
    # one sample: the average is the sample
    assert np.array_equal(o.stats(1), got)


def test_time_average_of_samples(tmp_path):
    from oracle_py import Oracle
    ini = channel_ini(nx=16, ny=12, nz=8)
    o = Oracle(tmp_path, ini)
    o.init_run()
    o.run(1)
    o.compute_stats(0)
    o.compute_stats_3d(0)
    a2, a3 = o.stats(1), o.stats(2)
    o.run(1)
    o.compute_stats(1)
    o.compute_stats_3d(1)
    b2 = o.stats(1)
    # w_stat = (w_stat*itav + w_stat_z)/(itav+1), the reference's two statements
    assert np.allclose(o.stats(0), (a2 * 1.0 + b2) / 2.0, rtol=1e-15, atol=0)
    # the 3-D point statistics from w and w_aux(6)
    w = o.w()[:, 3:-3, 3:-3, 3:-3]
    t = o.waux()[5][3:-3, 3:-3, 3:-3]
    b3 = np.stack([w[0], w[1], w[2], w[3], w[0] * t, w[0] ** 2, w[1] ** 2 / w[0], w[2] ** 2 / w[0],
                   w[3] ** 2 / w[0], w[1] * w[2] / w[0], w[1] * w[3] / w[0], w[2] * w[3] / w[0], w[0] * t ** 2,
                   (w[0] * t) ** 2], axis=-1)
    assert stat_err(o.stats(2), (a3 + b3) / 2.0).max() <= 1e-14


def test_sampled_state_after_a_step(tmp_path):
    """The state compute_stats sees after a step, which the device kernel rebuilds: the periodic
    ghost layers hold the bcswap copy of the start of stage 3 (= current interior minus the
    stage-3 increment fln), and with force_var w_aux(6) is the temperature of the updated state
    before the energy shift (= T(current) - tbdiff)."""
    from oracle_py import Oracle, lib, _d
    ini = channel_ini(nx=16, ny=12, nz=8)
    o = Oracle(tmp_path, ini)
    o.init_run()
    o.run(2)
    ng, nx, nz = o.ng, o.nx, o.nz
    w = o.w()
    fln = np.zeros((5, o.nz, o.ny, o.nx))
    lib.oracle_get_fln(o._h, _d(fln))
    J = slice(ng, ng + o.ny)
    K = slice(ng, ng + nz)
    for m in range(4):
        # rounding of (w_old + fln) - fln: a few units in the last place of the field's values
        tol = 1e-15 * np.abs(w[m]).max()
        # x ghosts i = 1-l (array index ng-l) copy interior i = nx+1-l
        for l in range(1, ng + 1):
            ghost = w[m][K, J, ng - l]
            rebuilt = w[m][K, J, ng + nx - l] - fln[m][:, :, nx - l]
            assert np.abs(ghost - rebuilt).max() <= tol, (m, l)
            assert np.abs(ghost - w[m][K, J, ng + nx - l]).max() > 100 * tol  # they are stale
            gz = w[m][ng - l, J, ng:ng + nx]
            rz = w[m][ng + nz - l, J, ng:ng + nx] - fln[m][nz - l, :, :]
            assert np.abs(gz - rz).max() <= tol, (m, l)
    # the energy shift of force_var: T of the shifted state exceeds w_aux(6) by tbdiff everywhere
    from streams_b200 import Case
    p = Case(tmp_path, ini).params()
    wi = w[:, K, J, ng:ng + nx]
    q = 0.5 * (wi[1] ** 2 + wi[2] ** 2 + wi[3] ** 2) / wi[0] ** 2
    e = wi[4] / wi[0] - q
    t_now = p.t0 + (e - p.cv_last * p.t0) / p.cv0
    d = t_now - o.waux()[5][K, J, ng:ng + nx]
    assert abs(d.mean()) > 1e-9 * p.t0  # the shift is not zero here
    assert np.ptp(d) <= 1e-12 * p.t0


@pytest.mark.parametrize("shock", [False, True], ids=["bl", "sbli"])
def test_sampled_periodic_ghosts_with_a_node_wall(tmp_path, shock):
    """Boundary layer (periodic z, node-based wall at ymin; with an impinging shock at ymax): the
    z ghost layers after a step are the stage-3 copy w - fln, except where update_ghost rewrites
    interior points with fixed values, which the copy holds too: the momentum at the wall points
    j = 1 (zero) and, with the shock, every variable at j = ny inside the shock's tanh window."""
    from oracle_py import Oracle, lib, _d
    kw = dict(mach=2.28, shock_angle=32.6, lx=60.0) if shock else {}
    o = Oracle(tmp_path, bl_ini(nx=48, ny=40, nz=16, **kw))
    o.init_run()
    o.run(2)
    ng, nx, ny, nz = o.ng, o.nx, o.ny, o.nz
    w = o.w()
    fln = np.zeros((5, nz, ny, nx))
    lib.oracle_get_fln(o._h, _d(fln))
    J = slice(ng, ng + ny)
    I = slice(ng, ng + nx)
    for m in range(4):
        tol = 1e-15 * np.abs(w[m]).max()
        for l in range(1, ng + 1):
            for ghost, src in ((ng - l, nz - l), (ng + nz - 1 + l, l - 1)):
                rebuilt = w[m][ng + src, J, I] - fln[m][src]
                if m > 0:
                    assert np.all(w[m][ghost, ng, I] == 0.0)  # j = 1
                    rebuilt[0] = 0.0
                if shock:
                    # the rows j = ny that differ are the shock window: there the copy is current
                    top = np.abs(w[m][ghost, ng + ny - 1, I] - rebuilt[-1]) > tol
                    assert 0 < top.sum() < nx
                    assert np.array_equal(w[m][ghost, ng + ny - 1, I][top], w[m][ng + src, ng + ny - 1, I][top])
                    rebuilt[-1][top] = w[m][ng + src, ng + ny - 1, I][top]
                assert np.abs(w[m][ghost, J, I] - rebuilt).max() <= tol, (m, l)


def test_stat_files_round_trip(tmp_path):
    """stat.bin / stat3d.bin (one block per statistic, Fortran order) and the averaging clock in
    field_info0.dat: a case written with statistics reloads them on restart_type = 2."""
    from streams_b200 import Case
    ini = channel_ini(nx=16, ny=12, nz=8)
    (tmp_path / "a").mkdir()
    case = Case(tmp_path / "a", ini)
    rng = np.random.default_rng(5)
    s2 = rng.standard_normal((12, 16, 70))
    s3 = rng.standard_normal((8, 12, 16, 14))
    out = tmp_path / "b"
    out.mkdir()
    case.write_state_stats(case.field(), 7, 0.25, s2, s3, 3, 0.125, out)
    # the file layout: statistic l is a contiguous (ny, nx) block
    raw = np.fromfile(out / "stat.bin", dtype=np.float64).reshape(70, 12, 16)
    assert np.array_equal(raw[4], s2[:, :, 4])
    raw3 = np.fromfile(out / "stat3d.bin", dtype=np.float64).reshape(14, 8, 12, 16)
    assert np.array_equal(raw3[13], s3[..., 13])
    back = Case(out)
    info = back.stats_info()
    assert info["itav"] == 3 and info["time_from_last_stat"] == 0.125
    assert info["enable_stat_time"] == 1 and info["enable_stat_3d"] == 1
    assert np.array_equal(back.restart_stats(0), s2)
    assert np.array_equal(back.restart_stats(2), s3)
    assert np.array_equal(back.field(), case.field())
