"""Post-processing of the running statistics, as the reference's tools/postpro does it: the
channel's ``stats1d`` (tools/postpro/src/postpro_cha.F90:10-205) and the boundary layer's
``stats2d`` (tools/postpro/src/postpro_bl.F90:10-329), with the compressibility transformations of
comp_transform.F90 and the derivative of derivatives.F90:20-117.

Input: ``w_stat`` with the 70 z- and time-averaged statistics of ``compute_stats``
(singleideal.F90:2003-2179) as written to ``stat.bin`` (one (ny, nx) block per statistic), the
grid files (``y.dat``; for the boundary layer also ``x.dat`` and, on a staggered grid, ``yn.dat``)
and the reference values of ``flow_params.dat``.  Output: for the channel the wall-unit profiles
of ``POSTPRO/channstat.prof`` (27 columns) and the summary of ``POSTPRO/channinfo.dat``; for the
boundary layer the streamwise distributions of ``POSTPRO/cf.dat`` (21 columns) and the profiles
of ``POSTPRO/stat_<i>.prof`` (29 columns) at the stations of postpro.ini's ``ixstat``.

Usage: ``python -m streams_b200.postpro <case dir>`` (reads singleideal.ini, flow_params.dat,
the grid files, stat.bin and postpro.ini there and writes POSTPRO/).
"""
from __future__ import annotations

import os
import sys
from fractions import Fraction
from pathlib import Path

import numpy as np

NV_STAT = 70
# statistics that change sign between the two halves of the channel (1-based, avg_walls)
ASYMMETRIC = (3, 14, 19, 31, 36, 38, 40, 42, 44, 50, 52, 54, 55, 60, 64)


# --- finite differences ---------------------------------------------------------------------

def fd_weights(points, x0: int) -> np.ndarray:
    """Exact first-derivative weights at x0 on the integer stencil ``points`` (solving the
    Taylor conditions in rational arithmetic)."""
    pts = [Fraction(p - x0) for p in points]
    n = len(pts)
    a = [[p ** k for p in pts] for k in range(n)]
    rhs = [Fraction(1 if k == 1 else 0) for k in range(n)]
    # Gauss-Jordan elimination on the Vandermonde system
    for c in range(n):
        r = next(i for i in range(c, n) if a[i][c] != 0)
        a[c], a[r] = a[r], a[c]
        rhs[c], rhs[r] = rhs[r], rhs[c]
        piv = a[c][c]
        a[c] = [v / piv for v in a[c]]
        rhs[c] = rhs[c] / piv
        for i in range(n):
            if i != c and a[i][c] != 0:
                f = a[i][c]
                a[i] = [vi - f * vc for vi, vc in zip(a[i], a[c])]
                rhs[i] = rhs[i] - f * rhs[c]
    return np.array([float(v) for v in rhs])


def ddy(u: np.ndarray, y: np.ndarray, order: int) -> np.ndarray:
    """du/dy on a stretched grid as D(u)/D(y), D the index-space derivative of the given order:
    central in the interior, one-sided on the first and last order/2 points (stencil of order+1
    points), as derivatives.F90's ddy."""
    lmax = order // 2
    if lmax < 1 or lmax > 3:
        raise ValueError("order must be 2, 4 or 6")
    n = len(u)
    out = np.empty(n)
    cen = fd_weights(range(-lmax, lmax + 1), 0)
    for j in range(lmax, n - lmax):
        sl = slice(j - lmax, j + lmax + 1)
        out[j] = np.dot(cen, u[sl]) / np.dot(cen, y[sl])
    for j in range(lmax):
        wl = fd_weights(range(0, 2 * lmax + 1), j)
        out[j] = np.dot(wl, u[:2 * lmax + 1]) / np.dot(wl, y[:2 * lmax + 1])
        # mirrored closure at the top end
        ur, yr = u[n - 1 - np.arange(2 * lmax + 1)], y[n - 1 - np.arange(2 * lmax + 1)]
        out[n - 1 - j] = np.dot(wl, ur) / np.dot(wl, yr)
    return out


# --- compressibility transformations (comp_transform.F90) -----------------------------------

def transform(y: np.ndarray, u: np.ndarray, vaux: np.ndarray, name: str, staggered: bool = True):
    """Transformed wall distance and velocity (yi, ui) of the van Driest, Trettel-Larsson,
    Volpiani and Hasan transformations: integrals of f dy and g du with the trapezoidal rule
    from the wall (at y = 0, u = 0 for the staggered grid).  vaux rows: rho/rho_w, nu/nu_w,
    mu/mu_w, y+, y*, M_tau."""
    rho, nu, mu, ystar, mtau = vaux[0], vaux[1], vaux[2], vaux[4], vaux[5]
    if name == "vanDriest":
        f = np.ones_like(y)
        g = np.sqrt(rho)
    elif name == "TrettelLarsson":
        f = ddy(y / (np.sqrt(rho) * nu), y, 2)
        g = f * rho * nu
    elif name == "Volpiani":
        f = np.sqrt(rho) * (rho * nu) ** -1.5
        g = np.sqrt(rho) * (rho * nu) ** -0.5
    elif name == "Hasan":
        f = ddy(y / (np.sqrt(rho) * nu), y, 6)
        g = f * rho * nu
        kappa = 0.41
        damp_i = (1.0 - np.exp(-ystar / 17.0)) ** 2
        damp_c = (1.0 - np.exp(-ystar / (17.0 + 19.3 * mtau[0]))) ** 2
        g = g * (1.0 + kappa * damp_c * ystar) / (1.0 + kappa * damp_i * ystar)
    else:
        raise ValueError(name)
    if staggered:
        f0, g0 = np.concatenate(([1.0], f[:-1])), np.concatenate(([1.0], g[:-1]))
        y0, u0 = np.concatenate(([0.0], y[:-1])), np.concatenate(([0.0], u[:-1]))
        yi = np.cumsum(0.5 * (f + f0) * (y - y0))
        ui = np.cumsum(0.5 * (g + g0) * (u - u0))
    else:
        yi = np.concatenate(([0.0], np.cumsum(0.5 * (f[1:] + f[:-1]) * np.diff(y))))
        ui = np.concatenate(([0.0], np.cumsum(0.5 * (g[1:] + g[:-1]) * np.diff(u))))
    return yi, ui


# --- stats1d ----------------------------------------------------------------------------------

def fold_walls(w1d: np.ndarray) -> np.ndarray:
    """avg_walls: average of the two channel halves, (j, m) -> the lower half; the statistics in
    ASYMMETRIC change sign between the halves."""
    ny = w1d.shape[0]
    h = ny // 2
    lower, upper = w1d[:h], w1d[::-1][:h]
    sign = np.ones(w1d.shape[1])
    sign[[m - 1 for m in ASYMMETRIC]] = -1.0
    return 0.5 * (lower + sign * upper)


def stats1d(w_stat: np.ndarray, y: np.ndarray, fp: dict, theta_wall: float, mach_input: float) -> dict:
    """Channel profiles and wall quantities from w_stat (ny, nx, 70) and the cell-centre y(1..ny)
    of the half-height-1 channel (y in (-1, 1)); fp holds flow_params.dat's values."""
    ny = w_stat.shape[0]
    h = ny // 2
    w1 = fold_walls(w_stat.mean(axis=1))          # (ny/2, 70), statistic m at [:, m-1]
    W = lambda m: w1[:, m - 1]  # noqa: E731
    yd = 1.0 + y[:h]                              # distance from the lower wall
    ufav, vfav, tfav = W(13) / W(1), W(14) / W(1), W(25) / W(1)
    twall, mu0, k0, cp0, gam = fp["T_wall"], fp["mu0"], fp["k0"], fp["cp0"], fp["gam"]
    rho0, u0, t0 = fp["rho0"], fp["u0"], fp["t0"]
    # wall gradients from the first three cell centres (u = 0 and T = T_wall at the wall)
    a, b, c = 9.0 / 8.0, -1.0 / 8.0, 0.0
    duw = 2 * a * ufav[0] + 2.0 / 3.0 * b * ufav[1] + 2.0 / 5.0 * c * ufav[2]
    dyw = 2 * a * yd[0] + 2.0 / 3.0 * b * yd[1] + 2.0 / 5.0 * c * yd[2]
    dtw = 2 * a * tfav[0] + 2.0 / 3.0 * b * tfav[1] + 2.0 / 5.0 * c * tfav[2]
    dtw = dtw - 2.0 * twall * (a + b / 3.0 + c / 5.0)
    dudyw, dtdyw = duw / dyw, dtw / dyw
    # wall density by extrapolation of the first three cell values
    rhow = (150.0 * W(1)[0] - 25.0 * W(1)[1] + 3.0 * W(1)[2]) / 128.0
    rmuw = mu0
    rnuw = rmuw / rhow
    ttw = twall
    tauw = rmuw * dudyw
    utau = np.sqrt(tauw / rhow)
    deltav = rnuw / utau
    retau = 1.0 / deltav
    qw = -k0 * dtdyw
    ttau = qw / (rhow * cp0 * utau)
    mtau = utau / np.sqrt(gam * ttw)
    vaux = np.empty((6, h))
    vaux[0] = W(1) / rhow
    vaux[1] = W(21) / rnuw
    vaux[2] = vaux[0] * vaux[1]
    vaux[3] = yd / deltav
    vaux[4] = yd * np.sqrt(tauw * W(1)) / W(20)
    vaux[5] = mtau
    ybig = yd * np.sqrt(vaux[0]) / vaux[2]
    prof = {}
    for name in ("vanDriest", "TrettelLarsson", "Volpiani", "Hasan"):
        prof[name] = transform(yd, ufav, vaux, name)
    d_vd = ddy(prof["vanDriest"][1], prof["vanDriest"][0], 2)
    d_tl = ddy(prof["TrettelLarsson"][1], prof["TrettelLarsson"][0], 2)
    d_v = ddy(prof["Volpiani"][1], prof["Volpiani"][0], 2)
    d_h = ddy(prof["Hasan"][1], prof["Volpiani"][0], 2)
    # Griffin-Fu-Moin transformation (total-stress based), integrated from the wall
    ug = np.empty(h)
    seq = ufav[0] / ybig[0]
    seqp = seq / utau * deltav
    setl = ufav[0] / y[0]
    setlp = setl / utau * deltav
    ug[0] = seq / (1.0 + seqp - setlp) * ybig[0]
    for j in range(1, h):
        taup = 1.0 - yd[j]
        seq = 1.0 / vaux[2, j] * (ufav[j] - ufav[j - 1]) / (ybig[j] - ybig[j - 1])
        seqp = seq / utau * deltav
        setl = vaux[2, j] * (ufav[j] - ufav[j - 1]) / (yd[j] - yd[j - 1])
        setlp = setl / utau * deltav
        ug[j] = ug[j - 1] + taup * seq / (taup + seqp - setlp) * (ybig[j] - ybig[j - 1])
    d_g = ddy(ug, prof["Hasan"][0], 2)
    yvd, uvd = prof["vanDriest"]
    ytl, utl = prof["TrettelLarsson"]
    yv, uv = prof["Volpiani"]
    yh, uh = prof["Hasan"]
    rho, pp = W(1), W(5)
    cols = np.column_stack([
        yd, rho / rho0, ufav / u0, tfav / t0, pp / rho0 / u0 ** 2, W(20) / rmuw, yd / deltav, vaux[4],
        yv / deltav, ufav / utau, uvd / utau, utl / utau, uv / utau, ug / utau, uh / utau,
        yvd * d_vd / utau, ytl * d_tl / utau, yv * d_v / utau, yh * d_g / utau, yh * d_h / utau,
        (W(16) - W(13) ** 2 / rho) / tauw, (W(17) - W(14) ** 2 / rho) / tauw, (W(18) - W(15) ** 2 / rho) / tauw,
        (W(19) - W(13) * W(14) / rho) / tauw,
        np.sqrt(np.abs(W(7) - rho ** 2)) / (rhow * gam * mtau ** 2),
        np.sqrt(np.abs(W(26) / rho - tfav ** 2)) / (ttw * gam * mtau ** 2),
        np.sqrt(np.abs(W(11) - pp ** 2)) / tauw])
    info = {"theta_wall": theta_wall, "mach_bulk_input": mach_input, "mach_wall": fp["Mach"],
            "reynolds_bulk_wall": fp["Reynolds"], "retau": retau, "cf": 2.0 * tauw / (rho0 * u0 ** 2),
            "rhow_over_rhob": rhow / rho0, "utau_over_ub": utau / u0, "ttau_over_tw": ttau / twall,
            "tauw": tauw, "utau": utau, "deltav": deltav, "vfav": vfav}
    return {"profile": cols, "info": info}


# --- stats2d (boundary layer) -----------------------------------------------------------------

def _griffin(u, y, ybig, vaux3, utau, deltav):
    """Griffin's velocity transformation, integrated from the first point as stats2d does
    (tools/postpro/src/postpro_bl.F90:239-251)."""
    ug = np.empty_like(u)
    with np.errstate(divide="ignore", invalid="ignore"):
        seq = u[0] / ybig[0]
        setl = u[0] / y[0]
        ug[0] = seq / (1.0 + seq / utau * deltav - setl / utau * deltav) * ybig[0]
        for j in range(1, len(u)):
            seq = 1.0 / vaux3[j] * (u[j] - u[j - 1]) / (ybig[j] - ybig[j - 1])
            setl = vaux3[j] * (u[j] - u[j - 1]) / (y[j] - y[j - 1])
            integrand = seq / (1.0 + seq / utau * deltav - setl / utau * deltav)
            ug[j] = ug[j - 1] + integrand * (ybig[j] - ybig[j - 1])
    return ug


def stats2d(w_stat: np.ndarray, x: np.ndarray, y: np.ndarray, fp: dict, theta_wall: float, prandtl: float,
            ystag: int = 0, yn: np.ndarray | None = None, ixstat=()) -> dict:
    """Boundary-layer post-processing of the running statistics (stats2d,
    tools/postpro/src/postpro_bl.F90:10-329).

    w_stat is (ny, nx, 70) as read_stat_bin returns it; x, y the interior coordinates (y from the
    wall), yn the cell faces (staggered grids, ystag > 0).  Returns "cf": (nx, 21), the columns of
    POSTPRO/cf.dat (x, delta99, delta*, theta, incompressible delta* and theta, H, H_inc,
    rho_w, T_w, p_w, p'_w+, u_tau/u0, cf, cf_inc (van Driest II), Re_delta99, Re_theta,
    Re_delta2, Re_tau, B_q, C_h), and "profiles": {i: (ny, 29)} for each station i of ixstat
    (1-based), the columns of POSTPRO/stat_<i>.prof.  The wall values use the staggered-grid
    closures (Lele's coefficients) or, on a node grid, the four-point one-sided difference, the
    wall temperature being the boundary condition T_wall; the edge of the layer is the first
    point above delta99 where du/dy falls below 1 % of its value at delta99."""
    W = lambda i, j, m: w_stat[j, i, m - 1]
    ny, nx = w_stat.shape[0], w_stat.shape[1]
    gam, u0, rho0, t0 = fp["gam"], fp["u0"], fp["rho0"], fp["t0"]
    rfac, mach, twall = fp["rfac"], fp["Mach"], fp["T_wall"]
    rho = w_stat[:, :, 0].T
    ufav, vfav, wfav, tfav = (w_stat[:, :, m - 1].T / rho for m in (13, 14, 15, 25))   # (nx, ny)
    dufavdy = np.array([ddy(ufav[i], y, 2) for i in range(nx)])
    u99 = 0.99 * u0
    cf_rows = np.empty((nx, 21))
    wall = {}
    for i in range(nx):
        if ystag > 0:
            aad, bbd, ccd = 9.0 / 8.0, -1.0 / 8.0, 0.0
            clo = lambda f: 2.0 * aad * f[0] + 2.0 / 3.0 * bbd * f[1] + 2.0 / 5.0 * ccd * f[2]
            duw, dyw = clo(ufav[i]), clo(y)
            dtw = clo(tfav[i]) - 2.0 * twall * (aad + bbd / 3.0 + ccd / 5.0)
            aai, bbi, cci = 150.0 / 128.0, -25.0 / 128.0, 3.0 / 128.0
            ext = lambda m: aai * W(i, 0, m) + bbi * W(i, 1, m) + cci * W(i, 2, m)
            rhow, rmuw = ext(1), ext(20)
        else:
            one = lambda f: -22.0 * f[0] + 36.0 * f[1] - 18.0 * f[2] + 4.0 * f[3]
            duw, dtw, dyw = one(ufav[i]), one(tfav[i]), one(y)
            rhow, rmuw = W(i, 0, 1), W(i, 0, 20)
        dudyw, dtdyw = duw / dyw, dtw / dyw
        rnuw = rmuw / rhow
        ttw = twall
        rlamw = rmuw * gam / (gam - 1.0) / prandtl
        tauw = rmuw * dudyw
        qw = -rlamw * dtdyw
        utau = np.sqrt(abs(tauw) / rhow)
        deltav = rnuw / utau
        cf = tauw / (0.5 * rho0 * u0 ** 2)
        trec = t0 * (1.0 + 0.5 * (gam - 1.0) * rfac * mach ** 2)
        bq = qw / ((gam / (gam - 1.0)) * rhow * utau * ttw)
        ch = 0.0 if theta_wall == 1.0 else qw / u0 / (gam / (gam - 1.0)) / (ttw - trec)
        # delta99: linear interpolation below the first point above 0.99 u0 (j99 >= 1)
        j99 = 1
        for j in range(1, ny):
            if ufav[i, j - 1] > u99:
                j99 = max(j - 1, 1)
                break
        a, b = j99 - 1, j99
        delta99 = y[a] + (y[b] - y[a]) * ((u99 - ufav[i, a]) / (ufav[i, b] - ufav[i, a]))
        retau = delta99 / deltav
        prmsp_w = np.sqrt(abs(W(i, 0, 11) - W(i, 0, 5) ** 2)) / tauw
        # edge of the layer and integral thicknesses (trapezoidal rule)
        duthr = 0.01 * dufavdy[i, j99 - 1]
        jint = 1
        for j in range(j99 + 1, ny):
            if dufavdy[i, j - 1] < duthr:
                jint = j
                break
        e = jint - 1
        rhoe, pe, ue = W(i, e, 1), W(i, e, 5), ufav[i, e]
        r = w_stat[:, i, 0] / rhoe
        uu = ufav[i] / ue
        if ystag > 0:
            dy = np.diff(yn)[:jint]
            dstar = np.sum(dy * (1.0 - r[:jint] * uu[:jint]))
            theta = np.sum(dy * (r[:jint] * uu[:jint] * (1.0 - uu[:jint])))
            dstarinc = np.sum(dy * (1.0 - uu[:jint]))
            thetainc = np.sum(dy * (uu[:jint] * (1.0 - uu[:jint])))
        else:
            dyh = 0.5 * np.diff(y)[:jint]
            lo, hi = slice(0, jint), slice(1, jint + 1)
            dstar = np.sum(dyh * ((1.0 - r[lo] * uu[lo]) + (1.0 - r[hi] * uu[hi])))
            theta = np.sum(dyh * (r[lo] * uu[lo] * (1.0 - uu[lo]) + r[hi] * uu[hi] * (1.0 - uu[hi])))
            dstarinc = np.sum(dyh * ((1.0 - uu[lo]) + (1.0 - uu[hi])))
            thetainc = np.sum(dyh * (uu[lo] * (1.0 - uu[lo]) + uu[hi] * (1.0 - uu[hi])))
        # van Driest II (Hopkins and Inouye, AIAA J 1971)
        tte = pe / rhoe
        rmue = W(i, e, 20)
        mach_edge = ue / np.sqrt(gam * tte)
        rmfac = rfac * 0.2 * mach_edge ** 2
        ff = ttw / tte
        aa = np.sqrt(rmfac / ff)
        bb = (1.0 + rmfac - ff) / ff
        alpha = (2.0 * aa ** 2 - bb) / np.sqrt(4.0 * aa ** 2 + bb ** 2)
        beta = bb / np.sqrt(4.0 * aa ** 2 + bb ** 2)
        with np.errstate(divide="ignore", invalid="ignore"):
            fc = rmfac / (np.arcsin(alpha) + np.arcsin(beta)) ** 2
        cf_rows[i] = [x[i], delta99, dstar, theta, dstarinc, thetainc, dstar / theta, dstarinc / thetainc,
                      rhow, ttw, rhow * ttw, prmsp_w, utau / u0, cf, cf * fc, ue * rhoe * delta99 / rmue,
                      ue * rhoe * theta / rmue, ue * rhoe * theta / rmuw, retau, bq, ch]
        wall[i] = (rhow, rmuw, delta99, deltav, utau, ttw)
    profiles = {}
    for ist in ixstat:
        i = int(ist) - 1
        rhow, rmuw, delta99, deltav, utau, ttw = wall[i]
        rnuw = rmuw / rhow
        tauw = rhow * utau ** 2
        rr, mu = w_stat[:, i, 0], w_stat[:, i, 19]
        vaux = np.array([rr / rhow, (mu / rr) / rnuw, rr / rhow * (mu / rr) / rnuw, y / deltav,
                         y * np.sqrt(tauw * rr) / mu, np.full(ny, utau / np.sqrt(gam * ttw))])
        u = ufav[i]
        ybig = y * np.sqrt(vaux[0]) / vaux[2]
        tr = {}
        with np.errstate(divide="ignore", invalid="ignore"):
            for name in ("vanDriest", "TrettelLarsson", "Volpiani", "Hasan"):
                yi, ui = transform(y, u, vaux, name, staggered=ystag > 0)
                tr[name] = (yi, ui, ddy(ui, yi, 2))
            ug = _griffin(u, y, ybig, vaux[2], utau, deltav)
            yh = tr["Hasan"][0]
            dugdy = ddy(ug, yh, 2)
            mtau = utau / np.sqrt(gam * ttw)
            prof = np.column_stack([
                y, rr, u / u0, vfav[i] / u0, tfav[i], tfav[i] * rr, mu / mu[0],
                y / delta99, y / deltav, vaux[4], tr["Volpiani"][0] / deltav,
                u / utau, tr["vanDriest"][1] / utau, tr["TrettelLarsson"][1] / utau, tr["Volpiani"][1] / utau,
                ug / utau, tr["Hasan"][1] / utau,
                tr["vanDriest"][0] * tr["vanDriest"][2] / utau, tr["TrettelLarsson"][0] * tr["TrettelLarsson"][2] / utau,
                tr["Volpiani"][0] * tr["Volpiani"][2] / utau, yh * dugdy / utau, yh * tr["Hasan"][2] / utau,
                (w_stat[:, i, 15] - rr * u * u) / tauw, (w_stat[:, i, 16] - rr * vfav[i] ** 2) / tauw,
                (w_stat[:, i, 17] - rr * wfav[i] ** 2) / tauw, (w_stat[:, i, 18] - rr * u * vfav[i]) / tauw,
                np.sqrt(w_stat[:, i, 6] - rr ** 2) / (rhow * gam * mtau ** 2),
                np.sqrt(w_stat[:, i, 25] / rr - tfav[i] ** 2) / (ttw * gam * mtau ** 2),
                np.sqrt(np.abs(w_stat[:, i, 10] - w_stat[:, i, 4] ** 2)) / tauw])
        profiles[int(ist)] = prof
    return {"cf": cf_rows, "profiles": profiles}


def write_bl_postpro(out_dir, result: dict) -> None:
    d = Path(out_dir) / "POSTPRO"
    d.mkdir(parents=True, exist_ok=True)
    np.savetxt(d / "cf.dat", result["cf"], fmt="%20.10E", delimiter="")
    for i, prof in result["profiles"].items():
        np.savetxt(d / f"stat_{i:06d}.prof", prof, fmt="%20.10E", delimiter="")


# --- files ------------------------------------------------------------------------------------

def read_flow_params(path) -> dict:
    out = {}
    for line in Path(path).read_text().splitlines():
        if "=" in line and not line.strip().startswith(("[", ";", "#")):
            k, v = line.split("=", 1)
            out[k.strip()] = float(v.split(";")[0].replace("d", "e").replace("D", "e"))
    return out


def read_stat_bin(path, nx: int, ny: int) -> np.ndarray:
    """stat.bin (70 blocks of nx*ny doubles, Fortran order) as (ny, nx, 70)."""
    a = np.fromfile(path, dtype=np.float64)
    if a.size != NV_STAT * nx * ny:
        raise ValueError(f"{path}: {a.size} values, expected {NV_STAT * nx * ny}")
    return np.moveaxis(a.reshape(NV_STAT, ny, nx), 0, -1)


def write_channel_postpro(out_dir, result: dict) -> None:
    d = Path(out_dir) / "POSTPRO"
    d.mkdir(parents=True, exist_ok=True)
    info = result["info"]
    with open(d / "channinfo.dat", "w") as f:
        if info["theta_wall"] >= -1.0:
            f.write(f" Turbulent channel flow with constant bulk temperature and theta_wall = {info['theta_wall']}\n")
            f.write(f" Mach number based on bulk temperature: {info['mach_bulk_input']}\n")
        else:
            f.write(" Turbulent channel flow with free bulk temperature\n")
        f.write(f" Mach number based on wall temperature: {info['mach_wall']}\n")
        f.write(f" Bulk Reynolds number based on wall viscosity: {info['reynolds_bulk_wall']}\n")
        f.write(f" Friction Reynolds number: {info['retau']}\n")
        f.write(f" Skin friction coefficient: {info['cf']}\n")
        f.write(f" Wall density / bulk density: {info['rhow_over_rhob']}\n")
        f.write(f" Friction velocity/ bulk velocity: {info['utau_over_ub']}\n")
        f.write(f" Friction temperature/ wall temperature: {info['ttau_over_tw']}\n")
    np.savetxt(d / "channstat.prof", result["profile"], fmt="%20.10E", delimiter="")


def _read_ini(path) -> dict:
    ini, sec = {}, None
    for line in Path(path).read_text().splitlines():
        line = line.split(";")[0].strip()
        if line.startswith("["):
            sec = line.strip("[]").strip()
        elif "=" in line and sec:
            k, v = line.split("=", 1)
            ini[(sec, k.strip())] = v.strip()
    return ini


def main(case_dir, ixstat=None) -> dict:
    """Post-process a case directory as tools/postpro does: stats1d for a channel (flow_init 0;
    singleideal.ini, flow_params.dat, y.dat, stat.bin), stats2d for a boundary layer (flow_init 1;
    also x.dat and, on a staggered grid, yn.dat).  The boundary layer's profile stations are
    ixstat (1-based i), else postpro.ini's [postpro] ixstat, else none."""
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    case_dir = Path(case_dir)
    ini = _read_ini(case_dir / "singleideal.ini")
    flow_init = int(ini[("flow", "flow_init")])
    nx, ny, ng = int(ini[("grid", "nxmax")]), int(ini[("grid", "nymax")]), int(ini[("grid", "ng")])
    fp = read_flow_params(case_dir / "flow_params.dat")
    y = np.loadtxt(case_dir / "y.dat")[ng:ng + ny]
    w_stat = read_stat_bin(case_dir / "stat.bin", nx, ny)
    if flow_init == 0:
        res = stats1d(w_stat, y, fp, float(ini[("flow", "theta_wall")]), float(ini[("flow", "Mach")]))
        write_channel_postpro(case_dir, res)
        return res
    if flow_init != 1:
        raise SystemExit("post-processing covers channels (flow_init 0) and boundary layers (flow_init 1)")
    ystag = int(ini.get(("grid", "ystag"), "0"))
    x = np.loadtxt(case_dir / "x.dat")[ng:ng + nx]
    yn = np.loadtxt(case_dir / "yn.dat")[:ny + 1] if ystag > 0 else None
    if ixstat is None:
        ixstat = ()
        if (case_dir / "postpro.ini").exists():
            v = _read_ini(case_dir / "postpro.ini").get(("postpro", "ixstat"))
            if v:
                ixstat = [int(t) for t in v.replace(",", " ").split()]
    res = stats2d(w_stat, x, y, fp, float(ini[("flow", "theta_wall")]), float(ini[("fluid", "Prandtl")]),
                  ystag, yn, ixstat)
    write_bl_postpro(case_dir, res)
    return res


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python -m streams_b200.postpro <case dir>")
    main(os.path.abspath(sys.argv[1]))
