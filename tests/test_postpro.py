"""Channel post-processing of the running statistics (streams_b200.postpro, the reference's
tools/postpro stats1d): finite-difference closures, the wall-folding and wall-unit bookkeeping on
an analytic laminar profile, and the whole chain stat.bin + flow_params.dat + y.dat ->
POSTPRO/channstat.prof on statistics sampled by the oracle."""
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
