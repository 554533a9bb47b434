"""Post-processing of the running statistics (streams_b200.postpro, the reference's tools/postpro):
the channel's stats1d (finite-difference closures, wall folding and wall units on an analytic
laminar profile, stat.bin + flow_params.dat + y.dat -> POSTPRO/channstat.prof on statistics
sampled by the oracle) and the boundary layer's stats2d (thicknesses, skin friction and
transformations on an analytic tanh layer, Lele's staggered wall closures, and POSTPRO/cf.dat
plus the station profiles of a boundary layer sampled by the oracle)."""
from fractions import Fraction

import numpy as np
import pytest

from conftest import channel_ini


def test_closure_weights_are_the_one_sided_taylor_weights():
    from streams_b200.postpro import fd_weights
    F = Fraction
    cases = {(3, 0): [F(-3, 2), 2, F(-1, 2)], (5, 0): [F(-25, 12), 4, -3, F(4, 3), F(-1, 4)],
             (5, 1): [F(-1, 4), F(-5, 6), F(3, 2), F(-1, 2), F(1, 12)],
             (7, 2): [F(1, 30), F(-2, 5), F(-7, 12), F(4, 3), F(-1, 2), F(2, 15), F(-1, 60)]}
    for (n, x0), want in cases.items():
        assert np.allclose(fd_weights(range(n), x0), [float(v) for v in want], rtol=0, atol=1e-15)
    assert np.allclose(fd_weights(range(-3, 4), 0), [-1 / 60, 3 / 20, -3 / 4, 0, 3 / 4, -3 / 20, 1 / 60], atol=1e-15)


@pytest.mark.parametrize("order", [2, 4, 6])
def test_ddy_is_exact_for_index_polynomials(order):
    from streams_b200.postpro import ddy
    xi = np.arange(20.0)
    y = 0.1 + 0.05 * xi                   # linear map: d/dy = (d/dxi) / 0.05
    u = (xi / 7.0) ** order               # a polynomial of the stencil's degree in the index
    exact = order * (xi / 7.0) ** (order - 1) / 7.0 / 0.05
    assert np.allclose(ddy(u, y, order), exact, rtol=1e-10, atol=1e-10)


def laminar_stats(ny, nx, mu0, umax=1.5):
    """w_stat of a laminar incompressible Poiseuille channel: rho = 1, T = 1, u = umax (1 - y^2)."""
    yn = np.linspace(-1.0, 1.0, ny + 1)
    y = 0.5 * (yn[1:] + yn[:-1])
    u = umax * (1.0 - y ** 2)
    w = np.zeros((ny, nx, 70))
    rho, t, p = 1.0, 1.0, 1.0
    for m, v in {1: rho, 2: u, 5: p, 6: t, 7: rho ** 2, 8: u ** 2, 11: p ** 2, 12: t ** 2, 13: rho * u,
                 16: rho * u * u, 20: mu0, 21: mu0 / rho, 25: rho * t, 26: rho * t * t}.items():
        w[:, :, m - 1] = np.asarray(v, dtype=float).reshape(-1, 1) if np.ndim(v) else v
    return w, y


def test_stats1d_on_a_laminar_profile():
    from streams_b200.postpro import stats1d
    mu0 = 1e-3
    w, y = laminar_stats(64, 8, mu0)
    fp = {"T_wall": 1.0, "mu0": mu0, "k0": mu0 * 3.5 / 0.72, "cp0": 3.5, "gam": 1.4, "rho0": 1.0, "u0": 1.0,
          "t0": 1.0, "Mach": 0.5, "Reynolds": 1000.0}
    res = stats1d(w, y, fp, theta_wall=0.0, mach_input=0.5)
    info, prof = res["info"], res["profile"]
    assert prof.shape == (32, 27) and np.all(np.isfinite(prof))
    # tau_w = mu du/dy|wall = 3 mu0 for u = 1.5 (1 - y^2): the cell-centre closure of stats1d
    # (9/8, -1/8) is exact for a linear profile, first order in h for the curvature term
    assert info["tauw"] == pytest.approx(3.0 * mu0, rel=1e-2)
    assert info["retau"] == pytest.approx(np.sqrt(3.0 * mu0) / mu0, rel=1e-2)
    w2, y2 = laminar_stats(128, 8, mu0)
    fine = stats1d(w2, y2, fp, theta_wall=0.0, mach_input=0.5)["info"]["tauw"]
    assert abs(info["tauw"] - 3e-3) / abs(fine - 3e-3) == pytest.approx(2.0, rel=1e-6)
    # uniform density: the van Driest velocity equals u; Reynolds stresses and rms vanish
    assert np.allclose(prof[:, 10], prof[:, 9], rtol=1e-12)
    assert np.allclose(prof[:, 20:27], 0.0, atol=1e-9)
    assert np.allclose(prof[:, 6], (1.0 + y[:32]) / info["deltav"])


def test_postpro_reads_the_files_this_backend_writes(tmp_path):
    """Statistics sampled by the oracle, written as stat.bin with the grid, flow_params.dat and
    the input (restart files of a running solve), post-processed from the directory."""
    from oracle_py import Oracle
    from streams_b200 import Case, postpro
    ini = channel_ini(nx=16, ny=24, nz=8)
    case = Case(tmp_path, ini)
    o = Oracle(tmp_path, ini)
    o.init_run()
    for itav in range(3):
        o.run(1)
        o.compute_stats(itav)
    out = tmp_path / "out"
    out.mkdir()
    w_stat = o.stats(0)
    case.write_state_stats(o.w(), 3, 0.0, w_stat, None, 3, 0.0, out)
    assert (out / "flow_params.dat").exists()
    fp = postpro.read_flow_params(out / "flow_params.dat")
    assert fp["mu0"] == pytest.approx(case.info()["mu0"], rel=1e-15)
    assert np.array_equal(postpro.read_stat_bin(out / "stat.bin", 16, 24), w_stat)
    res = postpro.main(out)
    prof = np.loadtxt(out / "POSTPRO" / "channstat.prof")
    assert prof.shape == (12, 27) and np.all(np.isfinite(prof))
    assert np.allclose(prof, res["profile"], rtol=1e-9)
    text = (out / "POSTPRO" / "channinfo.dat").read_text()
    assert "Friction Reynolds number" in text and res["info"]["retau"] > 0


def tanh_layer(nx=6, ny=401, h=0.02, mu0=1e-3, delta=1.0):
    """w_stat of an incompressible-like boundary layer on a node grid: rho = 1, T = 1, p = 1,
    u = tanh(y / delta), no fluctuations."""
    y = h * np.arange(ny)
    u = np.tanh(y / delta)
    w = np.zeros((ny, nx, 70))
    for m, v in {1: 1.0, 5: 1.0, 7: 1.0, 11: 1.0, 13: u, 16: u * u, 20: mu0, 25: 1.0, 26: 1.0}.items():
        w[:, :, m - 1] = np.asarray(v, dtype=float).reshape(-1, 1) if np.ndim(v) else v
    x = np.linspace(0.0, 1.0, nx)
    fp = {"gam": 1.4, "u0": 1.0, "rho0": 1.0, "t0": 1.0, "rfac": 0.72 ** (1 / 3), "Mach": 2.0, "T_wall": 1.0}
    return w, x, y, fp


def test_stats2d_on_a_tanh_layer():
    """delta99 = atanh(0.99) delta; with uniform density delta* = ln 2 delta and theta = (1 - ln 2)
    delta (to the truncation at the layer's edge); cf = 2 mu u0 / delta from the four-point wall
    closure; the van Driest velocity equals u; no fluctuations."""
    from streams_b200.postpro import stats2d
    mu0 = 1e-3
    w, x, y, fp = tanh_layer(mu0=mu0)
    res = stats2d(w, x, y, fp, theta_wall=1.0, prandtl=0.72, ystag=0, ixstat=[2, 5])
    cf = res["cf"]
    assert cf.shape == (6, 21)
    assert np.allclose(cf[:, 0], x)
    assert cf[0, 1] == pytest.approx(np.arctanh(0.99), rel=1e-3)          # delta99
    assert cf[0, 2] == pytest.approx(np.log(2.0), rel=1e-3)                # delta*
    # theta and H: stats2d normalises u by its value at the layer's edge (u_e = tanh(4.95) =
    # 0.9999 u0 here), which moves theta by about 4e-4 against the integral with u0
    assert cf[0, 3] == pytest.approx(1.0 - np.log(2.0), rel=3e-3)          # theta
    assert np.allclose(cf[0, 4:6], cf[0, 2:4], rtol=1e-14)                 # incompressible = compressible
    assert cf[0, 6] == pytest.approx(np.log(2.0) / (1.0 - np.log(2.0)), rel=3e-3)
    assert cf[0, 13] == pytest.approx(2.0 * mu0, rel=1e-4)                 # cf
    assert cf[0, 12] == pytest.approx(np.sqrt(mu0), rel=1e-4)              # u_tau / u0
    assert cf[0, 18] == pytest.approx(np.arctanh(0.99) * np.sqrt(mu0) / mu0, rel=1e-3)   # Re_tau
    assert cf[0, 19] == 0.0 and cf[0, 20] == 0.0                           # adiabatic-like: no heat flux
    assert cf[0, 11] == 0.0                                                # no pressure fluctuation
    assert np.allclose(cf[:, 1:], cf[0, 1:])                               # the same layer at every x
    prof = res["profiles"][5]
    assert prof.shape == (401, 29)
    utau = np.sqrt(mu0)
    assert np.allclose(prof[:, 11], np.tanh(y) / utau)                     # u+
    assert np.allclose(prof[:, 12], prof[:, 11], rtol=1e-12, atol=1e-12)   # van Driest u+ = u+
    assert np.allclose(prof[:, 8], y * utau / mu0)                         # y+
    assert np.allclose(prof[:, 22:29], 0.0, atol=1e-12)                    # no fluctuations


def test_stats2d_wall_closures_on_a_staggered_grid():
    """Lele's staggered closures: wall slope (9/8, -1/8) exact for a linear profile; wall
    density extrapolated with (150, -25, 3)/128."""
    from streams_b200.postpro import stats2d
    mu0, h, ny = 1e-3, 0.01, 300
    y = h * (np.arange(ny) + 0.5)
    u = np.minimum(y / 0.5, 1.0)                                           # linear up to y = 0.5
    w = np.zeros((ny, 4, 70))
    for m, v in {1: 1.0, 5: 1.0, 7: 1.0, 11: 1.0, 13: u, 16: u * u, 20: mu0, 25: 1.0, 26: 1.0}.items():
        w[:, :, m - 1] = np.asarray(v, dtype=float).reshape(-1, 1) if np.ndim(v) else v
    yn = h * np.arange(ny + 1)
    fp = {"gam": 1.4, "u0": 1.0, "rho0": 1.0, "t0": 1.0, "rfac": 0.89, "Mach": 2.0, "T_wall": 1.0}
    res = stats2d(w, np.arange(4.0), y, fp, theta_wall=1.0, prandtl=0.72, ystag=1, yn=yn)
    assert res["cf"][0, 13] == pytest.approx(2.0 * mu0 / 0.5, rel=1e-12)   # cf = 2 tau_w / (rho u0^2)
    assert res["cf"][0, 8] == pytest.approx(1.0, rel=1e-14)                # rho_w


def test_postpro_reads_a_boundary_layer_case(tmp_path):
    """Statistics of a boundary layer sampled by the oracle, written as the run writes them
    (stat.bin, x.dat, y.dat, flow_params.dat, singleideal.ini), post-processed from the
    directory with the stations of postpro.ini."""
    from oracle_py import Oracle
    from streams_b200 import Case, postpro
    from streams_b200.cases import bl_ini
    ini = bl_ini(nx=48, ny=40, nz=16)
    case = Case(tmp_path, ini)
    o = Oracle(tmp_path, ini)
    o.init_run()
    for itav in range(2):
        o.run(1)
        o.compute_stats(itav)
    out = tmp_path / "out"
    out.mkdir()
    case.write_state_stats(o.w(), 2, 0.0, o.stats(0), None, 2, 0.0, out)
    (out / "postpro.ini").write_text("[postpro]\nixstat = 12, 36\n")
    res = postpro.main(out)
    cf = np.loadtxt(out / "POSTPRO" / "cf.dat")
    assert cf.shape == (48, 21) and np.all(np.isfinite(cf))
    assert np.allclose(cf, res["cf"], rtol=1e-9)
    assert np.all(cf[:, 1] > 0) and np.all(cf[:, 13] > 0)                  # delta99, cf
    for i in (12, 36):
        prof = np.loadtxt(out / "POSTPRO" / f"stat_{i:06d}.prof")
        assert prof.shape == (40, 29)
        # every column is finite except Griffin's (columns 16, 21: 0/0 at the wall node of a node
        # grid, as in the reference) and, at the wall node only, the density and temperature rms
        # (columns 27, 28: the square root of a variance that is zero up to rounding there, taken
        # without an absolute value as the reference takes it)
        keep = [c for c in range(29) if c not in (15, 20)]
        assert np.all(np.isfinite(prof[1:, keep]))
        assert np.all(np.isfinite(prof[0, [c for c in keep if c not in (26, 27)]]))
