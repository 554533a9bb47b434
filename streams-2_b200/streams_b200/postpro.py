"""Channel-flow post-processing of the running statistics (the reference's tools/postpro
``stats1d``, tools/postpro/src/postpro_cha.F90:10-205, with the compressibility transformations of
comp_transform.F90 and the derivative of derivatives.F90:20-117).

Input: ``w_stat`` with the 70 z- and time-averaged statistics of ``compute_stats``
(singleideal.F90:2003-2179) as written to ``stat.bin`` (one (ny, nx) block per statistic), the
cell-centre ``y`` of the staggered channel grid (``y.dat``) and the reference values of
``flow_params.dat``.  Output: the wall-unit profiles of ``POSTPRO/channstat.prof`` (27 columns)
and the summary of ``POSTPRO/channinfo.dat``.

Usage: ``python -m streams_b200.postpro <case dir>`` (reads singleideal.ini, flow_params.dat,
y.dat and stat.bin there and writes POSTPRO/).
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


def main(case_dir) -> dict:
    """stats1d of a channel case directory (singleideal.ini, flow_params.dat, y.dat, stat.bin)."""
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    case_dir = Path(case_dir)
    ini = {}
    sec = None
    for line in (case_dir / "singleideal.ini").read_text().splitlines():
        line = line.split(";")[0].strip()
        if line.startswith("["):
            sec = line.strip("[]").strip()
        elif "=" in line and sec:
            k, v = line.split("=", 1)
            ini[(sec, k.strip())] = v.strip()
    if int(ini[("flow", "flow_init")]) != 0:
        raise SystemExit("stats1d post-processes channel flows (flow_init = 0)")
    nx, ny, ng = int(ini[("grid", "nxmax")]), int(ini[("grid", "nymax")]), int(ini[("grid", "ng")])
    fp = read_flow_params(case_dir / "flow_params.dat")
    y = np.loadtxt(case_dir / "y.dat")[ng:ng + ny]
    w_stat = read_stat_bin(case_dir / "stat.bin", nx, ny)
    res = stats1d(w_stat, y, fp, float(ini[("flow", "theta_wall")]), float(ini[("flow", "Mach")]))
    write_channel_postpro(case_dir, res)
    return res


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python -m streams_b200.postpro <case dir>")
    main(os.path.abspath(sys.argv[1]))
