"""Independent numpy restatement of STREAmS-2's hybrid convective face flux (test infrastructure).

Written from the Fortran of code/src/singleideal/kernels_cpu.F90, not from the C++ oracle or the
CUDA kernels, so that a misreading of the reference would have to be made twice, differently,
to pass the face-by-face comparison in tests/test_weno_pin.py:
  * central energy-preserving split form   euler_x_fluxes_hybrid_kernel  :470-612 (y, z alike)
  * Roe average (calorically perfect gas)  compute_roe_average           :3013-3089
  * left / right eigenvectors              eigenvectors_x / _y / _z      :2728-2782, 2842-2896, 2956-3010
  * local Lax-Friedrichs split, stencil max of |u_n -+ c|                 :614-675
  * WENO reconstruction of orders 1..4     wenorec_1d                    :2526-2724
  * near-wall order reduction              correct_bc_order (singleideal.F90:946-993)
  * finite-difference coefficients         get_deriv_coeffs (grid.F90:143-190)
Every function works on a batch of faces at once (leading axis).  Arrays of stencil points hold
the 2*S points of a face at offsets 1-S .. S from the face's lower point.
"""
from __future__ import annotations

import numpy as np


def deriv1_coeffs(order: int) -> np.ndarray:
    """coeff_deriv1(1:4) of get_deriv_coeffs for a central first derivative of the given order."""
    c = np.zeros(4)
    half = order // 2
    if half == 1:
        c[0] = 0.5
    elif half == 2:
        c[0], c[1] = 2.0 / 3.0, -1.0 / 12.0
    elif half == 3:
        c[0], c[1], c[2] = 0.75, -0.15, 1.0 / 60.0
    elif half == 4:
        c[0], c[1], c[2], c[3] = 4.0 / 5.0, -1.0 / 5.0, 4.0 / 105.0, -1.0 / 280.0
    return c


def coeff_table() -> np.ndarray:
    """coeff_deriv1_cpu(l, lmax) as table[lmax - 1, l - 1] (column lmax is order 2*lmax)."""
    return np.array([deriv1_coeffs(2 * lmax) for lmax in range(1, 5)])


def ep_ord_change(n: int, stencil: int, bounded: bool) -> np.ndarray:
    """Order change of the faces 0..n of one direction (correct_bc_order): faces 0 and n at
    1 - stencil, faces p and n - p at p - stencil for p < stencil, 0 elsewhere; nothing for a
    direction whose two boundaries are periodic."""
    e = np.zeros(n + 1, dtype=int)
    if bounded:
        e[0] = -stencil + 1
        for p in range(1, stencil):
            e[p] = -stencil + p
        e[n] = -stencil + 1
        for p in range(1, stencil):
            e[n - p] = -stencil + p
    return e


def wenorec_1d(vp: np.ndarray, vm: np.ndarray, iweno: int, order: int, version: int, rho0: float,
               u0: float) -> np.ndarray:
    """vhat(m) of wenorec_1d for every face: vp, vm are (n, 5, 2*iweno) with vp[:, m, l - 1] =
    vp(m, l); order is wenorec_ord (one value for all faces)."""
    i = iweno

    def P(l):  # vp(m, l) of every face and characteristic field: (n, 5)
        return vp[:, :, l - 1]

    def M(l):
        return vm[:, :, l - 1]

    u0_2 = u0 * u0
    rho0_2u0_2 = rho0 * rho0 * u0_2
    rho0_2u0_4 = rho0_2u0_2 * u0_2
    bs = np.array([1.0 / rho0_2u0_2, 1.0 / rho0_2u0_2, 1.0 / rho0_2u0_4, 1.0 / rho0_2u0_4, 1.0 / rho0_2u0_2])
    eps = 0.000001
    if order == 1:
        return P(i) + M(i + 1)
    if order == 2:
        dwe = [1.0 / 3.0, 2.0 / 3.0]
        bp = [bs * (P(i) - P(i - 1)) ** 2, bs * (P(i + 1) - P(i)) ** 2]
        bm = [bs * (M(i + 2) - M(i + 1)) ** 2, bs * (M(i + 1) - M(i)) ** 2]
        wp = [dwe[l] / (eps + bp[l]) ** 2 for l in range(2)]
        wm = [dwe[l] / (eps + bm[l]) ** 2 for l in range(2)]
        sp, sm = wp[0] + wp[1], wm[0] + wm[1]
        wp = [w / sp for w in wp]
        wm = [w / sm for w in wm]
        vminus = wp[0] * (-P(i - 1) + 3 * P(i)) + wp[1] * (P(i) + P(i + 1))
        vplus = wm[0] * (-M(i + 2) + 3 * M(i + 1)) + wm[1] * (M(i) + M(i + 1))
        return 0.5 * (vminus + vplus)
    if order == 3:
        dwe = [1.0 / 10.0, 6.0 / 10.0, 3.0 / 10.0]
        d0, d1 = 13.0 / 12.0, 1.0 / 4.0
        c0, c1, c2, c3, c4 = 1.0 / 3.0, 5.0 / 6.0, -1.0 / 6.0, -7.0 / 6.0, 11.0 / 6.0
        bp = [d0 * (P(i) - 2.0 * P(i - 1) + P(i - 2)) ** 2 + d1 * (3.0 * P(i) - 4.0 * P(i - 1) + P(i - 2)) ** 2,
              d0 * (P(i - 1) - 2.0 * P(i) + P(i + 1)) ** 2 + d1 * (P(i - 1) - P(i + 1)) ** 2,
              d0 * (P(i) - 2.0 * P(i + 1) + P(i + 2)) ** 2 + d1 * (3.0 * P(i) - 4.0 * P(i + 1) + P(i + 2)) ** 2]
        bm = [d0 * (M(i + 1) - 2.0 * M(i + 2) + M(i + 3)) ** 2 + d1 * (3.0 * M(i + 1) - 4.0 * M(i + 2) + M(i + 3)) ** 2,
              d0 * (M(i + 2) - 2.0 * M(i + 1) + M(i)) ** 2 + d1 * (M(i + 2) - M(i)) ** 2,
              d0 * (M(i + 1) - 2.0 * M(i) + M(i - 1)) ** 2 + d1 * (3.0 * M(i + 1) - 4.0 * M(i) + M(i - 1)) ** 2]
        bp = [bs * b for b in bp]
        bm = [bs * b for b in bm]
        if version == 0:
            wp = [dwe[l] / (eps + bp[l]) ** 2 for l in range(3)]
            wm = [dwe[l] / (eps + bm[l]) ** 2 for l in range(3)]
        else:
            eps40 = float(np.float32(1.0e-35))  # a default-kind real literal in the reference
            tau5p = np.abs(bp[0] - bp[2]) + eps40
            tau5m = np.abs(bm[0] - bm[2]) + eps40
            wp = [dwe[l] / ((bp[l] + eps40) / (bp[l] + tau5p)) for l in range(3)]
            wm = [dwe[l] / ((bm[l] + eps40) / (bm[l] + tau5m)) for l in range(3)]
        sp = wp[0] + wp[1] + wp[2]
        sm = wm[0] + wm[1] + wm[2]
        wp = [w / sp for w in wp]
        wm = [w / sm for w in wm]
        vminus = (wp[2] * (c0 * P(i) + c1 * P(i + 1) + c2 * P(i + 2)) +
                  wp[1] * (c2 * P(i - 1) + c1 * P(i) + c0 * P(i + 1)) +
                  wp[0] * (c0 * P(i - 2) + c3 * P(i - 1) + c4 * P(i)))
        vplus = (wm[2] * (c0 * M(i + 1) + c1 * M(i) + c2 * M(i - 1)) +
                 wm[1] * (c2 * M(i + 2) + c1 * M(i + 1) + c0 * M(i)) +
                 wm[0] * (c0 * M(i + 3) + c3 * M(i + 2) + c4 * M(i + 1)))
        return vminus + vplus
    if order == 4:
        dwe = [1.0 / 35.0, 12.0 / 35.0, 18.0 / 35.0, 4.0 / 35.0]
        d1, d2, d3 = 1.0 / 36.0, 13.0 / 12.0, 781.0 / 720.0
        bp = [d1 * (-2 * P(i - 3) + 9 * P(i - 2) - 18 * P(i - 1) + 11 * P(i)) ** 2 +
              d2 * (-P(i - 3) + 4 * P(i - 2) - 5 * P(i - 1) + 2 * P(i)) ** 2 +
              d3 * (-P(i - 3) + 3 * P(i - 2) - 3 * P(i - 1) + P(i)) ** 2,
              d1 * (P(i - 2) - 6 * P(i - 1) + 3 * P(i) + 2 * P(i + 1)) ** 2 +
              d2 * (P(i - 1) - 2 * P(i) + P(i + 1)) ** 2 +
              d3 * (-P(i - 2) + 3 * P(i - 1) - 3 * P(i) + P(i + 1)) ** 2,
              d1 * (-2 * P(i - 1) - 3 * P(i) + 6 * P(i + 1) - P(i + 2)) ** 2 +
              d2 * (P(i - 1) - 2 * P(i) + P(i + 1)) ** 2 +
              d3 * (-P(i - 1) + 3 * P(i) - 3 * P(i + 1) + P(i + 2)) ** 2,
              d1 * (-11 * P(i) + 18 * P(i + 1) - 9 * P(i + 2) + 2 * P(i + 3)) ** 2 +
              d2 * (2 * P(i) - 5 * P(i + 1) + 4 * P(i + 2) - P(i + 3)) ** 2 +
              d3 * (-P(i) + 3 * P(i + 1) - 3 * P(i + 2) + P(i + 3)) ** 2]
        bm = [d1 * (-2 * M(i + 4) + 9 * M(i + 3) - 18 * M(i + 2) + 11 * M(i + 1)) ** 2 +
              d2 * (-M(i + 4) + 4 * M(i + 3) - 5 * M(i + 2) + 2 * M(i + 1)) ** 2 +
              d3 * (-M(i + 4) + 3 * M(i + 3) - 3 * M(i + 2) + M(i + 1)) ** 2,
              d1 * (M(i + 3) - 6 * M(i + 2) + 3 * M(i + 1) + 2 * M(i)) ** 2 +
              d2 * (M(i + 2) - 2 * M(i + 1) + M(i)) ** 2 +
              d3 * (-M(i + 3) + 3 * M(i + 2) - 3 * M(i + 1) + M(i)) ** 2,
              d1 * (-2 * M(i + 2) - 3 * M(i + 1) + 6 * M(i) - M(i - 1)) ** 2 +
              d2 * (M(i + 2) - 2 * M(i + 1) + M(i)) ** 2 +
              d3 * (-M(i + 2) + 3 * M(i + 1) - 3 * M(i) + M(i - 1)) ** 2,
              d1 * (-11 * M(i + 1) + 18 * M(i) - 9 * M(i - 1) + 2 * M(i - 2)) ** 2 +
              d2 * (2 * M(i + 1) - 5 * M(i) + 4 * M(i - 1) - M(i - 2)) ** 2 +
              d3 * (-M(i + 1) + 3 * M(i) - 3 * M(i - 1) + M(i - 2)) ** 2]
        bp = [bs * b for b in bp]
        bm = [bs * b for b in bm]
        wp = [dwe[l] / (eps + bp[l]) ** 2 for l in range(4)]
        wm = [dwe[l] / (eps + bm[l]) ** 2 for l in range(4)]
        sp = wp[0] + wp[1] + wp[2] + wp[3]
        sm = wm[0] + wm[1] + wm[2] + wm[3]
        wp = [w / sp for w in wp]
        wm = [w / sm for w in wm]
        vminus = (wp[3] * (6 * P(i) + 26 * P(i + 1) - 10 * P(i + 2) + 2 * P(i + 3)) +
                  wp[2] * (-2 * P(i - 1) + 14 * P(i) + 14 * P(i + 1) - 2 * P(i + 2)) +
                  wp[1] * (2 * P(i - 2) - 10 * P(i - 1) + 26 * P(i) + 6 * P(i + 1)) +
                  wp[0] * (-6 * P(i - 3) + 26 * P(i - 2) - 46 * P(i - 1) + 50 * P(i)))
        vplus = (wm[3] * (6 * M(i + 1) + 26 * M(i) - 10 * M(i - 1) + 2 * M(i - 2)) +
                 wm[2] * (-2 * M(i + 2) + 14 * M(i + 1) + 14 * M(i) - 2 * M(i - 1)) +
                 wm[1] * (2 * M(i + 3) - 10 * M(i + 2) + 26 * M(i + 1) + 6 * M(i)) +
                 wm[0] * (-6 * M(i + 4) + 26 * M(i + 3) - 46 * M(i + 2) + 50 * M(i + 1)))
        return (vminus + vplus) / 24.0
    raise ValueError(f"wenorec order {order}")


def eigenvectors(direction: int, b1, b2, b3, uu, vv, ww, c, ci, h):
    """el(r, m) and er(m, r) of eigenvectors_x/_y/_z for every face: (n, 5, 5) arrays indexed
    [face, first Fortran index - 1, second Fortran index - 1]."""
    n = b1.shape[0]
    el = np.zeros((n, 5, 5))
    er = np.zeros((n, 5, 5))
    vel = [uu, vv, ww]
    vn = vel[direction]
    # rows of the left eigenvectors for the two acoustic fields and the entropy field
    for col, sgn in ((0, 1.0), (4, -1.0)):
        el[:, 0, col] = 0.5 * (b1 + sgn * vn * ci)
        for d in range(3):
            el[:, 1 + d, col] = -0.5 * (b2 * vel[d] + (sgn * ci if d == direction else 0.0))
        el[:, 4, col] = 0.5 * b2
    el[:, 0, 1] = 1.0 - b1
    for d in range(3):
        el[:, 1 + d, 1] = b2 * vel[d]
    el[:, 4, 1] = -b2
    # the two shear fields: the transverse momenta in increasing index order
    tang = [d for d in range(3) if d != direction]
    for col, d in zip((2, 3), tang):
        el[:, 0, col] = -vel[d]
        el[:, 1 + d, col] = 1.0
    # right eigenvectors
    er[:, 0, 0] = 1.0
    er[:, 1, 0] = 1.0
    er[:, 4, 0] = 1.0
    for d in range(3):
        if d == direction:
            er[:, 0, 1 + d] = vel[d] - c
            er[:, 1, 1 + d] = vel[d]
            er[:, 4, 1 + d] = vel[d] + c
        else:
            er[:, 0, 1 + d] = vel[d]
            er[:, 1, 1 + d] = vel[d]
            er[:, 4, 1 + d] = vel[d]
    for col, d in zip((2, 3), tang):
        er[:, col, 1 + d] = 1.0
    er[:, 0, 4] = h - vn * c
    er[:, 1, 4] = b3
    er[:, 2, 4] = vel[tang[0]]
    er[:, 3, 4] = vel[tang[1]]
    er[:, 4, 4] = h + vn * c
    return el, er


def roe_average(rho_l, u_l, v_l, w_l, h_l, rho_r, u_r, v_r, w_r, h_r, rgas0, cp0, cp_last, t0):
    """compute_roe_average for a calorically perfect gas: b1, b2, b3, c, ci, h, uu, vv, ww."""
    r = np.sqrt(rho_r / rho_l)
    rho = r * rho_l
    rp1 = 1.0 / (r + 1.0)
    uu = (r * u_r + u_l) * rp1
    vv = (r * v_r + v_l) * rp1
    ww = (r * w_r + w_l) * rp1
    h = (r * h_r + h_l) * rp1
    qq = 0.5 * (uu * uu + vv * vv + ww * ww)
    hbar = h - qq - cp_last * t0
    tt = t0 + hbar / cp0
    gamloc = cp0 / (cp0 - rgas0)
    cc = gamloc * tt * rgas0
    gm1loc = gamloc - 1.0
    c = np.sqrt(cc)
    ci = 1.0 / c
    p_rho = tt * rgas0
    p_e = rho * gm1loc
    etot = h - tt * rgas0
    b3 = etot - rho * p_rho / p_e
    b2 = p_e / (rho * cc)
    b1 = p_rho / cc - b2 * (etot - 2.0 * qq)
    return b1, b2, b3, c, ci, h, uu, vv, ww


def weno_face_flux(st: dict, direction: int, ws: int, order: int, version: int, gas: dict) -> np.ndarray:
    """Characteristic WENO flux of euler_*_hybrid_kernel's shock branch for faces whose stencil
    arrays st[name] are (n, 2*ws) with points l = 1..2*ws at offset l - ws from the face's lower
    point (names rho, u, v, w, h, t).  Returns fhat (n, 5)."""
    rgas0, cp0, cp_last, t0 = gas["rgas0"], gas["cp0"], gas["cp_last"], gas["t0"]
    il, ir = ws - 1, ws  # the points i and i+1 of the face
    b1, b2, b3, c, ci, h, uu, vv, ww = roe_average(
        st["rho"][:, il], st["u"][:, il], st["v"][:, il], st["w"][:, il], st["h"][:, il],
        st["rho"][:, ir], st["u"][:, ir], st["v"][:, ir], st["w"][:, ir], st["h"][:, ir], rgas0, cp0, cp_last, t0)
    el, er = eigenvectors(direction, b1, b2, b3, uu, vv, ww, c, ci, h)
    vname = "uvw"[direction]
    gam = cp0 / (cp0 - rgas0)
    cs = np.sqrt(gam * rgas0 * st["t"])
    vnp = st[vname]
    ev = np.full((st["rho"].shape[0], 5), -1.0)
    for l in range(2 * ws):
        ev[:, 0] = np.maximum(np.abs(vnp[:, l] - cs[:, l]), ev[:, 0])
        ev[:, 1] = np.maximum(np.abs(vnp[:, l]), ev[:, 1])
        ev[:, 4] = np.maximum(np.abs(vnp[:, l] + cs[:, l]), ev[:, 4])
    ev[:, 2] = ev[:, 1]
    ev[:, 3] = ev[:, 1]
    n = st["rho"].shape[0]
    gp = np.zeros((n, 5, 2 * ws))
    gm = np.zeros((n, 5, 2 * ws))
    for l in range(2 * ws):
        rho, u, v, w, hh = (st[k][:, l] for k in ("rho", "u", "v", "w", "h"))
        vel = [u, v, w]
        rhovn = rho * vel[direction]
        pp = rho * st["t"][:, l] * rgas0
        f = [rhovn, u * rhovn, v * rhovn, w * rhovn, hh * rhovn]
        f[1 + direction] = f[1 + direction] + pp
        q = [rho, rho * u, rho * v, rho * w, rho * hh - pp]
        for m in range(5):
            wc = np.zeros(n)
            gc = np.zeros(n)
            for r in range(5):  # the reference accumulates component by component
                wc = wc + el[:, r, m] * q[r]
                gc = gc + el[:, r, m] * f[r]
            cm = 0.5 * (gc + ev[:, m] * wc)
            gp[:, m, l] = cm
            gm[:, m, l] = gc - cm
    fi = wenorec_1d(gp, gm, ws, order, version, gas["rho0"], gas["u0"])
    out = np.zeros((n, 5))
    for m in range(5):
        acc = np.zeros(n)
        for mm in range(5):
            acc = acc + er[:, mm, m] * fi[:, mm]
        out[:, m] = acc
    return out


def central_face_flux(st: dict, direction: int, lmax: int, nkeep: int, rgas0: float, zero_flux) -> np.ndarray:
    """Energy-preserving split-form central flux of euler_*_hybrid_kernel for faces whose
    stencil arrays st[name] are (n, 2*S) with points at offsets 1-S .. S (S = columns / 2);
    lmax is the face's order half-width (one value for all faces); zero_flux a bool mask of the
    faces of force_zero_flux.  nkeep = 0, < 0 and > 0 as the reference."""
    S = st["rho"].shape[1] // 2
    n = st["rho"].shape[0]
    coeff = coeff_table()
    vname = "uvw"[direction]
    ft = [np.zeros(n) for _ in range(6)]
    for l in range(1, lmax + 1):
        uvs = [np.zeros(n) for _ in range(9)]  # 1, 2, 3, 4, 5 (enthalpy form), 5_i, 5_k, 5_p, 6
        for m in range(l):
            a, b = S - 1 - m, S - 1 - m + l  # points i-m and i-m+l
            rhoi, uui, vvi, wwi, enti, tti = (st[k][:, a] for k in ("rho", "u", "v", "w", "h", "t"))
            rhoip, uuip, vvip, wwip, entip, ttip = (st[k][:, b] for k in ("rho", "u", "v", "w", "h", "t"))
            vni, vnip = st[vname][:, a], st[vname][:, b]
            ppi = tti * rhoi * rgas0
            ppip = ttip * rhoip * rgas0
            rhom = rhoi + rhoip
            if nkeep >= 0:
                eei = enti - ppi / rhoi - 0.5 * (uui * uui + vvi * vvi + wwi * wwi)
                eeip = entip - ppip / rhoip - 0.5 * (uuip * uuip + vvip * vvip + wwip * wwip)
                eem = eei + eeip
                if nkeep == 0:
                    drhof = 1.0
                    deef = 1.0
                else:
                    drho = 2.0 * (rhoip - rhoi) / rhom
                    dee = 2.0 * (eeip - eei) / eem
                    t_r = (0.5 * drho) * (0.5 * drho)
                    t_e = (0.5 * dee) * (0.5 * dee)
                    t2r, t2e = t_r, t_e
                    sdr = 1.0 + t_r / 3.0
                    sde = 1.0 + t_e
                    sne = 1.0 + t_e / 3.0
                    for nn in range(2, nkeep + 1):
                        t_r = t2r * t_r
                        t_e = t2e * t_e
                        sdr = sdr + t_r / (1.0 + 2 * nn)
                        sde = sde + t_e
                        sne = sne + t_e / (1.0 + 2 * nn)
                    drhof = 1.0 / sdr
                    deef = sne / sde
                uv = (vni + vnip) * rhom * drhof
                uvs[0] = uvs[0] + uv * 2.0
                uvs[1] = uvs[1] + uv * (uui + uuip)
                uvs[2] = uvs[2] + uv * (vvi + vvip)
                uvs[3] = uvs[3] + uv * (wwi + wwip)
                uvs[5] = uvs[5] + uv * eem * deef
                uvs[6] = uvs[6] + uv * (uui * uuip + vvi * vvip + wwi * wwip)
                uvs[7] = uvs[7] + 4.0 * (vni * ppip + vnip * ppi)
            else:
                uv = (vni + vnip) * rhom
                uvs[0] = uvs[0] + uv * 2.0
                uvs[1] = uvs[1] + uv * (uui + uuip)
                uvs[2] = uvs[2] + uv * (vvi + vvip)
                uvs[3] = uvs[3] + uv * (wwi + wwip)
                uvs[4] = uvs[4] + uv * (enti + entip)
            uvs[8] = uvs[8] + 2.0 * (ppi + ppip)
        cl = coeff[lmax - 1, l - 1]
        for q in range(4):
            ft[q] = ft[q] + cl * uvs[q]
        ft[4] = ft[4] + cl * ((uvs[5] + uvs[6] + uvs[7]) if nkeep >= 0 else uvs[4])
        ft[5] = ft[5] + cl * uvs[8]
    fh = np.stack([0.25 * ft[q] for q in range(5)], axis=1)
    fh[zero_flux] = 0.0
    fh[:, 1 + direction] = fh[:, 1 + direction] + 0.5 * ft[5]
    return fh
