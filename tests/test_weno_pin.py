"""Pins of the oracle's branches that the reference's golden row never reaches (CPU tests).

The reference's own regression row (tests.ini [subsonic_channel]) is central-only, Sutherland
and without force_var.  The oracle's WENO branch, its power-law viscosity runs and force_var are
therefore checked here against things that do not come from the oracle's own code:
  * the hybrid face flux, face by face, against tests/weno_ref.py, a numpy restatement written
    from kernels_cpu.F90 (WENO-JS / WENO-Z of orders 3, 5, 7 with their near-wall reductions,
    the central split form for nkeep = 0, < 0 and > 0, x, y and z faces);
  * the eigenvector algebra against the flux Jacobian: the right eigenvectors of
    eigenvectors_x/_y/_z (kernels_cpu.F90:2728-3010) diagonalise dF/dU of the Euler flux at the
    state with eigenvalues u_n - c, u_n, u_n, u_n, u_n + c, and the left ones invert them;
  * wenorec_1d converging at its design order (3, 5, 7) on smooth periodic data, WENO-JS and
    WENO-Z;
  * force_var (singleideal_cpu.F90:890-933) holding the bulk temperature at its target.
"""
import numpy as np
import pytest

from conftest import channel_ini
import weno_ref


def _stencils(waux, faces, S, ng):
    """Stencil arrays (n, 2S) of aux fields rho, u, v, w, h, t at offsets 1-S .. S for faces
    (dir, i, j, k) with 1-based lower points; waux is (10, nz+2ng, ny+2ng, nx+2ng)."""
    names = ("rho", "u", "v", "w", "h", "t")
    st = {k: np.zeros((len(faces), 2 * S)) for k in names}
    for q, (d, i, j, k) in enumerate(faces):
        for o in range(1 - S, S + 1):
            p = [i, j, k]
            p[d] += o
            for m, name in enumerate(names):
                st[name][q, o + S - 1] = waux[m, p[2] + ng - 1, p[1] + ng - 1, p[0] + ng - 1]
    return st


def _faces(nx, ny, nz, rng, count):
    """Random faces of the three directions, plus every y face of one line (the near-wall
    faces with reduced orders and the staggered walls' zero-flux faces)."""
    out = []
    for d, n in ((0, nx), (1, ny), (2, nz)):
        for _ in range(count):
            p = [int(rng.integers(1, nx + 1)), int(rng.integers(1, ny + 1)), int(rng.integers(1, nz + 1))]
            p[d] = int(rng.integers(0, n + 1))
            out.append((d, *p))
    out += [(1, 3, j, 2) for j in range(0, ny + 1)]
    return out


CONFIGS = {
    "weno5_js": dict(sensor=-1.0, weno_scheme=3, ep_order=6),
    "weno5_z": dict(sensor=-1.0, weno_scheme=3, ep_order=6, weno_version=1),
    "weno3": dict(sensor=-1.0, weno_scheme=2, ep_order=4),
    "weno7": dict(sensor=-1.0, weno_scheme=4, ep_order=8),
    "central6": dict(sensor=1.01),
    "central8": dict(sensor=1.01, weno_scheme=4, ep_order=8),
    "central6_enthalpy": dict(sensor=1.01, nkeep=-1),
    "central6_keep2": dict(sensor=1.01, nkeep=2),
}


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_face_flux_matches_independent_restatement(name, tmp_path):
    from oracle_py import Oracle
    kw = dict(nx=20, ny=16, nz=12)
    kw.update(CONFIGS[name])
    o = Oracle(tmp_path, channel_ini(**kw))
    o.init_run()
    o.run(2)  # a developed field; w_aux of the last stage holds interior and face ghosts
    waux = o.waux()
    ng, nx, ny, nz = o.ng, o.nx, o.ny, o.nz
    faces = _faces(nx, ny, nz, np.random.default_rng(7), 40)
    got = o.face_flux(np.array(faces))
    ws, lmax_base = kw.get("weno_scheme", 3), kw.get("ep_order", 6) // 2
    stencil = max(lmax_base, ws)
    ep = [weno_ref.ep_ord_change(n, stencil, bounded) for n, bounded in ((nx, False), (ny, True), (nz, False))]
    from streams_b200 import Case
    p = Case(tmp_path, channel_ini(**kw)).params()
    gas = dict(rgas0=p.rgas0, cp0=p.cp0, cp_last=p.cp_last, t0=p.t0, rho0=p.rho0, u0=p.u0)
    weno = kw["sensor"] < 0
    exp = np.zeros_like(got)
    groups = {}
    for q, (d, i, j, k) in enumerate(faces):
        pos = (i, j, k)[d]
        order = max((ws if weno else lmax_base) + ep[d][pos], 1)
        groups.setdefault((d, order), []).append(q)
    for (d, order), idx in groups.items():
        sel = [faces[q] for q in idx]
        if weno:
            st = _stencils(waux, sel, ws, ng)
            exp[idx] = weno_ref.weno_face_flux(st, d, ws, order, kw.get("weno_version", 0), gas)
        else:
            S = max(lmax_base, ws)
            st = _stencils(waux, sel, S, ng)
            nd = (nx, ny, nz)[d]
            zero = np.array([d == 1 and (f[2] == 0 or f[2] == nd) for f in sel])  # staggered walls
            exp[idx] = weno_ref.central_face_flux(st, d, order, kw.get("nkeep", 0), gas["rgas0"], zero)
    scale = np.abs(exp).max(axis=0) + 1e-300
    err = np.abs(got - exp).max(axis=0) / scale
    assert err.max() <= 1e-14, (name, err)
    # the test reaches the reduced orders and the zero-flux faces it claims
    assert {int(o) for (_, o) in groups} == set(range(1, (ws if weno else lmax_base) + 1)), groups.keys()


def _euler_flux(U, d, gam):
    rho, mom, E = U[0], U[1:4], U[4]
    vel = mom / rho
    p = (gam - 1.0) * (E - 0.5 * rho * (vel @ vel))
    F = vel[d] * U
    F[1 + d] += p
    F[4] += vel[d] * p
    return F


@pytest.mark.parametrize("direction", [0, 1, 2])
def test_eigenvectors_diagonalise_the_flux_jacobian(direction):
    gam, rgas0 = 1.4, 1.0
    cp0 = gam / (gam - 1.0) * rgas0
    rng = np.random.default_rng(direction)
    for _ in range(20):
        rho = rng.uniform(0.5, 2.0)
        vel = rng.uniform(-1.5, 1.5, 3)
        t = rng.uniform(0.6, 2.0)
        h = cp0 * t + 0.5 * vel @ vel
        a = lambda x: np.array([x])  # noqa: E731
        b1, b2, b3, c, ci, hh, uu, vv, ww = weno_ref.roe_average(
            a(rho), a(vel[0]), a(vel[1]), a(vel[2]), a(h), a(rho), a(vel[0]), a(vel[1]), a(vel[2]), a(h),
            rgas0, cp0, cp0, 1.0)  # enthalpy datum cp_last t0 = cp0 t0: h = cp0 T
        el, er = weno_ref.eigenvectors(direction, b1, b2, b3, uu, vv, ww, c, ci, hh)
        L = el[0].T  # L[m, r] = el(r, m): the m-th characteristic field
        R = er[0].T  # R[comp, m] = er(m, comp): the m-th right eigenvector as a column
        assert np.allclose(R @ L, np.eye(5), atol=1e-12)
        U = np.array([rho, *(rho * vel), rho * (h - rgas0 * t)])
        J = np.zeros((5, 5))
        for q in range(5):
            dU = np.zeros(5)
            dU[q] = 1e-6 * max(1.0, abs(U[q]))
            J[:, q] = (_euler_flux(U + dU, direction, gam) - _euler_flux(U - dU, direction, gam)) / (2 * dU[q])
        lam = vel[direction] + np.array([-c[0], 0.0, 0.0, 0.0, c[0]])
        assert np.allclose(J @ R, R * lam[None, :], atol=1e-7 * np.abs(J).max())


def _weno_divergence_error(n, ws, version, scale=1.0):
    """Max error of (h(j+1/2) - h(j-1/2))/dx against f'(x_j) + g'(x_j) on n periodic points,
    with vp = f and vm = g the two split parts (f, g smooth and periodic).  scale is rho0 = u0
    of wenorec_1d: the smoothness indicators are multiplied by 1/scale^4 (or 1/scale^6)."""
    x = np.arange(n) / n
    dx = 1.0 / n
    f = lambda s: 1.0 + 0.5 * np.sin(2 * np.pi * s) + 0.2 * np.cos(4 * np.pi * s)  # noqa: E731
    df = lambda s: np.pi * np.cos(2 * np.pi * s) - 0.8 * np.pi * np.sin(4 * np.pi * s)  # noqa: E731
    g = lambda s: 0.3 * np.cos(2 * np.pi * s + 0.4) - 0.7  # noqa: E731
    dg = lambda s: -0.6 * np.pi * np.sin(2 * np.pi * s + 0.4)  # noqa: E731
    # faces j+1/2, j = 0..n-1: points l = 1..2ws at j + l - ws, the same 5 characteristic rows
    idx = (np.arange(n)[:, None] + np.arange(1, 2 * ws + 1)[None, :] - ws) % n
    vp = np.repeat(f(x)[idx][:, None, :], 5, axis=1)
    vm = np.repeat(g(x)[idx][:, None, :], 5, axis=1)
    h = weno_ref.wenorec_1d(vp, vm, ws, ws, version, scale, scale)[:, 0]
    div = (h - np.roll(h, 1)) / dx
    return np.abs(div - (df(x) + dg(x))).max()


@pytest.mark.parametrize("ws,design", [(2, 3), (3, 5), (4, 7)], ids=["weno3", "weno5", "weno7"])
def test_wenorec_linear_limit_has_the_design_order(ws, design):
    """With the smoothness indicators scaled far below eps (rho0 = u0 = 1e3) the WENO-JS weights
    are the ideal ones and the reconstruction is the linear upwind scheme of order 2 ws - 1:
    this pins the candidate stencils and the ideal weights."""
    ns = [16, 32, 64, 128]
    errs = [_weno_divergence_error(n, ws, 0, scale=1e3) for n in ns]
    order = np.log2(errs[-2] / errs[-1])
    assert order >= design - 0.15, (errs, order)


@pytest.mark.parametrize("version,least", [(0, 4.7), (1, 3.8)], ids=["weno5_js", "weno5_z"])
def test_wenorec_nonlinear_weights_converge(version, least):
    """With the indicators active (rho0 = u0 = 1) the nonlinear weights approach the ideal ones
    as the grid is refined.  WENO-JS (eps = 1e-6) shows its fifth order once the indicators fall
    below eps; WENO-Z with exponent 1 is fourth order at the critical points of the data."""
    ns = [256, 512, 1024]
    errs = [_weno_divergence_error(n, 3, version) for n in ns]
    order = np.log2(errs[0] / errs[-1]) / 2
    assert order >= least, (errs, order)


@pytest.mark.parametrize("ws,version", [(2, 0), (3, 0), (3, 1), (4, 0)], ids=["weno3", "weno5_js", "weno5_z", "weno7"])
def test_wenorec_step_is_non_oscillatory(ws, version):
    """A top-hat reconstructed with the indicators active stays within the data's bounds."""
    n = 64
    x = np.arange(n) / n
    f = np.where((x > 0.3) & (x < 0.6), 1.0, 0.0)
    idx = (np.arange(n)[:, None] + np.arange(1, 2 * ws + 1)[None, :] - ws) % n
    vp = np.repeat(f[idx][:, None, :], 5, axis=1)
    h = weno_ref.wenorec_1d(vp, np.zeros_like(vp), ws, ws, version, 1.0, 1.0)[:, 0]
    assert h.min() >= -1e-12 and h.max() <= 1.0 + 1e-12, (h.min(), h.max())


def test_force_var_holds_the_bulk_temperature(tmp_path):
    """force_var shifts the energy so that the bulk temperature sum(rho u T dy)/(volchan rho_b
    u_b) equals t_bulk_target after the update; recomputed here from the oracle's field."""
    from oracle_py import Oracle
    from streams_b200 import Case
    ini = channel_ini(nx=20, ny=16, nz=12, theta_wall=0.0)
    o = Oracle(tmp_path, ini)
    case = Case(tmp_path, ini)  # held: its grid arrays live as long as the case
    p = case.params()
    info = o.case_info()
    target, volchan = info["t_bulk_target"], info["volchan"]
    ng, ny = o.ng, o.ny
    dy = np.diff(np.ctypeslib.as_array(case.grid().yn, shape=(ny + 1,)))
    o.init_run()
    worst = 0.0
    for _ in range(12):
        o.run(1)
        w = o.w()[:, ng:-ng, ng:-ng, ng:-ng]
        rho, ru, rv, rw, re = w
        qq = 0.5 * ((ru / rho) ** 2 + (rv / rho) ** 2 + (rw / rho) ** 2)
        ee = re / rho - qq
        tt = p.t0 + (ee - p.cv_last * p.t0) / p.cv0
        sc = o.scalars()
        tb = (ru * tt * dy[None, :, None]).sum() / volchan / sc["rhobulk"] / sc["ubulk"]
        worst = max(worst, abs(tb - target) / target)
    assert worst <= 1e-13, worst
