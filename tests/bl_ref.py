"""Independent numpy restatement of the reference's boundary-layer mean profile (test
infrastructure).

Written from code/src/singleideal/singleideal.F90 (hasan_meanprofile :4090-4249, set_bl_prop
:2858-2892, the thickness march of init_bl :3252-3358) and parameters.F90 (locateval, pol_int),
not from the C++ set-up, so that tests/test_init_bl.py checks the set-up's restatement against
a second reading of the Fortran.  Vectorised over the profile's 10001 points.
"""
from __future__ import annotations

import numpy as np

NY = 10000


def hasan(ye, d99, mach, theta, retau, retheta, pr, spr, rfac, gam, vtexp, visc_exp, s2tinf, imode, icompute):
    """hasan_meanprofile: returns dict(retau, retheta, redelta, th, cf, ch, mtau, deltav) and,
    with icompute, the profiles u, t, rho, mu at ye."""
    pi = 4.0 * np.arctan(1.0)
    gm1h = 0.5 * (gam - 1.0)
    tr = 1.0 + gm1h * rfac * mach ** 2
    tw = 1.0 + theta * (tr - 1.0)
    apl, vkc = 17.0, 0.41
    dy = d99 / NY
    y = np.arange(NY + 1) * dy
    yext = np.arange(2 * NY + 1) * dy
    ufac = 0.99
    u = np.minimum(1.0, y / d99)
    u = u / (u[-1] / ufac)
    if imode == 0:
        retheta = 1000.0
    else:
        retau = 200.0
    mtau = 0.1

    def visc(t):
        return t ** vtexp if visc_exp else t ** 1.5 * (1.0 + s2tinf) / (t + s2tinf)

    absdiff, niter = np.inf, 0
    while absdiff > 0.00001:
        niter += 1
        if niter > 10000:
            break
        old = retheta if imode == 0 else retau
        t = tw + (tr - tw) * (spr * u + (1.0 - spr) * u ** 2) + (1.0 - tr) * u ** 2
        rho = 1.0 / t
        mu = visc(t)
        ypl = (y / d99) * retau
        yst = ypl * np.sqrt(rho / rho[0]) * mu[0] / mu
        d = (1.0 - np.exp(-yst / (apl + 19.3 * mtau))) ** 2
        mut = mu / mu[0] * vkc * yst * d
        z1 = retheta / 425.0 - 1.0
        picole = 0.69 * (1.0 - np.exp(-0.243 * np.sqrt(z1) - 0.15 * z1))
        wake = picole / vkc * pi * np.sin(pi * (y / d99))
        uint = 1.0 / (mu / mu[0] + mut) + np.sqrt(rho[0] / rho) / retau * wake
        upl = np.concatenate([[0.0], np.cumsum(0.5 * (uint[1:] + uint[:-1]) * np.diff(ypl))])
        uinf_plus = upl[-1] / ufac
        u = upl / uinf_plus
        thi = rho * u * (1.0 - u)
        th = float(np.sum(0.5 * (thi[1:] + thi[:-1]) * np.diff(y)))
        cf = 2.0 / uinf_plus ** 2 * rho[0]
        ch = 0.5 * cf * spr / pr
        mtau = mach * np.sqrt(0.5 * cf)
        if imode == 0:
            retheta = retau * th / d99 * mu[0] / rho[0] * uinf_plus
            absdiff = abs(retheta - old)
        else:
            retau = retheta * d99 / th / mu[0] * rho[0] / uinf_plus
            absdiff = abs(retau - old)
        redelta = retheta * d99 / th
    out = dict(retau=retau, retheta=retheta, redelta=redelta, th=th, cf=cf, ch=ch, mtau=mtau, deltav=d99 / retau)
    if not icompute:
        return out
    # profiles continued linearly beyond d99 (u capped at 1), interpolated linearly onto ye; up to
    # d99 the temperature is the last iteration's, formed from the velocity before its update
    dudy = (u[-1] - u[-2]) / (yext[NY] - yext[NY - 1])
    uext = np.concatenate([u, np.minimum(u[-1] + dudy * (yext[NY + 1:] - yext[NY]), 1.0)])
    text = tw + (tr - tw) * (spr * uext + (1.0 - spr) * uext ** 2) + (1.0 - tr) * uext ** 2
    text[:NY + 1] = t
    rhoext = 1.0 / text
    muext = visc(text)
    ye = np.asarray(ye, dtype=float)
    prof = {}
    for name, f in (("u", uext), ("t", text), ("rho", rhoext), ("mu", muext)):
        v = np.ones_like(ye)
        inside = ye < yext[-1]
        v[inside] = np.interp(ye[inside], yext, f)
        prof[name] = v
    out.update(prof)
    return out


def thickness_march(xg, ng, nx, l0, retau_in, prof_args):
    """delta, deltav, cf along the stations xg(1-ng .. nx+ng+1) as init_bl marches them (thvec,
    Re_theta scaled with the momentum thickness, delta iterated to 1e-9).  xg is indexed from
    1-ng at [0]; prof_args are the hasan arguments after retheta (pr, spr, rfac, gam, vtexp,
    visc_exp, s2tinf) with mach, theta first: (mach, theta, pr, ...)."""
    mach, theta = prof_args[:2]
    rest = prof_args[2:]
    n = nx + 2 * ng + 1
    X = lambda i: i + ng - 1  # noqa: E731
    delta, deltav, cf, th, retauv = (np.zeros(n) for _ in range(5))
    h = hasan([], l0, mach, theta, retau_in, 0.0, *rest, 0, 0)
    delta[X(1)], deltav[X(1)], cf[X(1)], th[X(1)], retauv[X(1)] = l0, h["deltav"], h["cf"], h["th"], retau_in
    rth_in = h["retheta"]

    def station(i, nb, rth):
        th[X(i)] = th[X(nb)] + (1 if i > nb else -1) * 0.5 * abs(xg[X(i)] - xg[X(nb)]) * cf[X(nb)]
        rth = rth / th[X(nb)] * th[X(i)]
        d = delta[X(nb)] / th[X(nb)] * th[X(i)]
        while True:
            dold = d
            hs = hasan([], d, mach, theta, 0.0, rth, *rest, 1, 0)
            d = delta[X(nb)] * hs["retau"] / retauv[X(nb)] * np.sqrt(cf[X(nb)] / hs["cf"])
            if abs(d - dold) < 1e-9:
                break
        delta[X(i)], cf[X(i)], deltav[X(i)], retauv[X(i)] = d, hs["cf"], hs["deltav"], hs["retau"]
        return rth

    r = rth_in
    for i in range(1, ng + 1):
        r = station(1 - i, 2 - i, r)
    r = rth_in
    for i in range(2, nx + ng + 2):
        r = station(i, i - 1, r)
    return delta, deltav, cf
