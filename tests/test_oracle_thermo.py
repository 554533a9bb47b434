"""Thermally perfect gas (calorically_perfect = 0) on the CPU: the set-up's cp(T) polynomial
(set_fluid_prop, code/src/singleideal/singleideal.F90:2685-2774), the oracle's temperature
recovery against an independent numpy restatement of get_e_from_temperature_dev
(kernels_cpu.F90:7155-7176), and a constant polynomial reproducing the calorically perfect gas."""
import numpy as np
import pytest

from conftest import channel_ini


def gas_case(tmp_path, cp_poly, **kw):
    from streams_b200 import Case
    from streams_b200.cases import channel_ini as build
    return Case(tmp_path, build(16, 12, 8, cp_poly=cp_poly, **kw))


def test_set_up_scales_the_polynomial(tmp_path):
    from streams_b200.cases import SYNTHETIC_CP_POLY
    lo, hi, coef = SYNTHETIC_CP_POLY
    p = gas_case(tmp_path, SYNTHETIC_CP_POLY).params()
    tref = p.t_ref_dim
    assert (p.calorically_perfect, p.indx_cp_l, p.indx_cp_r) == (0, lo, hi)
    cp = np.array(list(p.cp_coeff)[:hi - lo + 2])
    cv = np.array(list(p.cv_coeff)[:hi - lo + 2])
    want = np.array([coef[l - lo] * tref ** l for l in range(lo, hi + 1)]) * p.rgas0
    assert np.allclose(cp[:-1], want, rtol=1e-15, atol=0)
    # cv = cp except cv(0) = cp(0) - R; the datum h(T_ref)/(R T_ref) from the integral of cp
    assert np.allclose(cv[:-1] - cp[:-1], [-p.rgas0 if l == 0 else 0.0 for l in range(lo, hi + 1)], atol=1e-15)
    hstar = coef[-1] + sum((coef[l - lo] * np.log(tref) if l == -1 else coef[l - lo] / (l + 1) * tref ** (l + 1))
                           for l in range(lo, hi + 1))
    assert cp[-1] == pytest.approx(hstar / tref * p.rgas0, rel=1e-14)
    assert cv[-1] == pytest.approx((hstar / tref - 1.0) * p.rgas0, rel=1e-14)


def e_of_t_numpy(p, t):
    """get_e_from_temperature_dev restated with numpy."""
    lo, hi = p.indx_cp_l, p.indx_cp_r
    cv = list(p.cv_coeff)
    e = np.full_like(t, cv[hi + 1 - lo])
    tr = t / p.t0
    for l in range(lo, hi + 1):
        c = cv[l - lo]
        e = e + (c * np.log(tr) if l == -1 else c / (l + 1.0) * (tr ** (l + 1) - 1.0))
    return e * p.t0


def test_temperature_recovery_inverts_the_energy(tmp_path):
    from oracle_py import Oracle
    from streams_b200.cases import SYNTHETIC_CP_POLY, channel_ini as build
    ini = build(16, 12, 8, cp_poly=SYNTHETIC_CP_POLY, mach=2.5)
    p = gas_case(tmp_path, SYNTHETIC_CP_POLY, mach=2.5).params()
    o = Oracle(tmp_path, ini)
    o.init_run()
    o.run(3)
    o.compute_dt()  # aux of the current state, interior points
    w = o.w()[:, 3:-3, 3:-3, 3:-3]
    t = o.waux()[5][3:-3, 3:-3, 3:-3]
    e = w[4] / w[0] - 0.5 * (w[1] ** 2 + w[2] ** 2 + w[3] ** 2) / w[0] ** 2
    assert np.ptp(t) > 0.05 * p.t0  # the temperature varies: cp(T) is exercised
    assert np.abs(e_of_t_numpy(p, t) - e).max() <= 1e-12 * np.abs(e).max()


def test_constant_polynomial_is_the_calorically_perfect_gas(tmp_path):
    """cp/R = gam/(gam-1) as a polynomial (all other coefficients and the datum zero) gives the
    same constants as the calorically perfect gas, so the two runs agree to round-off."""
    from oracle_py import Oracle
    from streams_b200.cases import channel_ini as build
    const = (-2, 2, (0.0, 0.0, 3.5, 0.0, 0.0, 0.0))
    out = []
    for poly in (None, const):
        o = Oracle(tmp_path, build(16, 12, 8, cp_poly=poly, sensor=-1.0))
        o.init_run()
        o.run(5)
        out.append(o.w())
    a, b = out
    for m in range(5):
        assert np.abs(a[m] - b[m]).max() <= 1e-12 * np.abs(a[m]).max(), m


def test_unsupported_gas_inputs_fail_loudly(tmp_path):
    from streams_b200 import BackendError, Case, Solver
    from streams_b200.cases import SYNTHETIC_CP_POLY, channel_ini as build
    with pytest.raises(BackendError, match="cp coefficients"):
        Case(tmp_path, build(16, 12, 8, cp_poly=SYNTHETIC_CP_POLY).replace(", 0.0\n", "\n", 1))
    case = Case(tmp_path, build(16, 12, 8, cp_poly=SYNTHETIC_CP_POLY))
    p = case.params(precision=1)
    with pytest.raises(BackendError, match="FP64"):
        Solver(p, case.grid())
