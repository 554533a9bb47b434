"""The reference's own boundary-layer initialisation (init_bl with hasan_meanprofile and
add_synthetic_perturbations, singleideal.F90:3252-3423, 3587-3685, 4090-4249) in the host
set-up, checked on the CPU against tests/bl_ref.py, an independent numpy restatement of the mean
profile, on the reference's example input (tests/golden/supersonic_bl.ini, made from
examples/supersonic_bl by tests/golden/make_golden.py) with the grid reduced further.
"""
import re

import numpy as np
import pytest

from conftest import ROOT
import bl_ref


def reduced(ini: str, **sizes) -> str:
    out, sec = [], None
    for ln in ini.splitlines():
        m = re.match(r"\s*\[(\w+)\]", ln)
        if m:
            sec = m.group(1)
        k = ln.split("=")[0].strip()
        if sec == "grid" and k in sizes:
            ln = f"{k} = {sizes[k]}"
        out.append(ln)
    return "\n".join(out)


@pytest.fixture(scope="module")
def small_bl(tmp_path_factory):
    from streams_b200 import Case
    d = tmp_path_factory.mktemp("bl")
    ini = reduced((ROOT / "tests" / "golden" / "supersonic_bl.ini").read_text(), nxmax=24, nymax=48, nzmax=8,
                  nywr=32)
    case = Case(d, ini)
    return case, ini, d


def gas(case):
    p = case.params()
    s2tinf = p.sutherland_s / p.t_ref_dim
    rfac = p.prandtl ** (1.0 / 3.0)  # turbulent recovery factor of set_fluid_prop
    return p, s2tinf, rfac


def test_free_stream_reynolds_number_from_the_profile(small_bl):
    """set_bl_prop: the input friction Reynolds number (200) becomes the thickness-based one."""
    case, ini, _ = small_bl
    p, s2tinf, rfac = gas(case)
    info = case.info()
    re_delta = info["u0"] * info["rho0"] * info["l0"] / info["mu0"]
    ny = p.ny
    y = np.ctypeslib.as_array(case.grid().y, shape=(ny + 2 * p.ng,))[p.ng:p.ng + ny]
    mach = float(re.search(r"Mach\s*=\s*([0-9.eE+-]+)", ini).group(1))
    h = bl_ref.hasan(y, 1.0, mach, p.theta_wall, 200.0, 0.0, p.prandtl, 0.8, rfac, 1.4, p.powerlaw_vtexp,
                     p.visc_model == 1, s2tinf, 0, 0)
    assert abs(re_delta - h["redelta"]) <= 1e-9 * h["redelta"], (re_delta, h["redelta"])


def test_mean_density_and_draws_follow_the_profile_march(small_bl):
    """The density of every cell is the mean profile's at the cell's station (init_bl adds its
    perturbations to the velocities only); the thickness march gives delta(x), which also fixes
    how many random numbers the set-up drew (3 per cell, 4 streak phases, 3 per cell below
    delta)."""
    case, ini, _ = small_bl
    p, s2tinf, rfac = gas(case)
    nx, ny, nz, ng = p.nx, p.ny, p.nz, p.ng
    mach = float(re.search(r"Mach\s*=\s*([0-9.eE+-]+)", ini).group(1))
    g = case.grid()
    x = np.ctypeslib.as_array(g.x, shape=(nx + 2 * ng,)).copy()
    y = np.ctypeslib.as_array(g.y, shape=(ny + 2 * ng,))[ng:ng + ny].copy()
    xg = np.concatenate([x, [x[-1] + (x[-1] - x[-2])]])  # the uniform BL grid, one station further
    args = (mach, p.theta_wall, p.prandtl, 0.8, rfac, 1.4, p.powerlaw_vtexp, p.visc_model == 1, s2tinf)
    info = case.info()
    delta, deltav, cf = bl_ref.thickness_march(xg, ng, nx, info["l0"], 200.0, args)
    assert np.all(np.diff(delta[ng:]) > 0)  # the layer grows downstream
    w = case.field()
    for i in (1, nx // 2, nx):
        X = i + ng - 1
        h = bl_ref.hasan(y, delta[X], mach, p.theta_wall, delta[X] / deltav[X], 0.0, *args[2:], 0, 1)
        rho = w[0, ng:ng + nz, ng:ng + ny, ng + i - 1]
        assert np.allclose(rho, (h["rho"] * info["rho0"])[None, :], rtol=1e-9, atol=0), i
    below = sum(int(np.sum(y < delta[i + ng - 1])) for i in range(1, nx + 1)) * nz
    assert p.rng_draws == 3 * nx * ny * nz + 4 + 3 * below


def test_blvec_cache_is_read_back(small_bl, tmp_path):
    """init_bl writes blvec.bin beside the input and reads it on the next set-up, as the
    reference does; the second set-up gives the same field."""
    from streams_b200 import Case
    case, ini, d = small_bl
    assert (d / "blvec.bin").stat().st_size == 4 * 8 * (case.params().nx + 2 * case.params().ng + 1) + 8
    again = Case(d, ini)
    assert np.array_equal(again.field(), case.field())
