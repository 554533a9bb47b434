// Host-side case set-up; see setup.hpp.  Each function cites the reference routine it
// restates (paths relative to the STREAmS-2 repository).
#include "setup.hpp"

#include "glibc_rand.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <limits>
#include <string>
#include <thread>
#include <utility>
#include <vector>

namespace streams_b200 {

namespace {

constexpr int GRID_FROMFILE = 1, GRID_UNIFORM = 2, GRID_CHA = 3, GRID_BL = 4, GRID_SBLI = 5;
constexpr double TOL_ITER = 0.000000001;  // parameters.F90:43 (REAL64 build)

double pi() { return std::acos(-1.0); }

// get_deriv_coeffs (code/src/grid.F90:143-190)
void get_deriv_coeffs(double c1[4], double c2[5], int order1, int order2) {
  for (int l = 0; l < 4; ++l) c1[l] = 0;
  for (int l = 0; l < 5; ++l) c2[l] = 0;
  switch (order1 / 2) {
    case 1: c1[0] = 0.5; break;
    case 2: c1[0] = 2.0 / 3.0; c1[1] = -1.0 / 12.0; break;
    case 3: c1[0] = 0.75; c1[1] = -0.15; c1[2] = 1.0 / 60.0; break;
    case 4: c1[0] = 4.0 / 5.0; c1[1] = -1.0 / 5.0; c1[2] = 4.0 / 105.0; c1[3] = -1.0 / 280.0; break;
  }
  switch (order2 / 2) {
    case 1: c2[0] = -2.0; c2[1] = 1.0; break;
    case 2: c2[0] = -2.5; c2[1] = 4.0 / 3.0; c2[2] = -1.0 / 12.0; break;
    case 3: c2[0] = -245.0 / 90.0; c2[1] = 1.5; c2[2] = -0.15; c2[3] = 1.0 / 90.0; break;
    case 4:
      c2[0] = -205.0 / 72.0; c2[1] = 8.0 / 5.0; c2[2] = -1.0 / 5.0; c2[3] = 8.0 / 315.0; c2[4] = -1.0 / 560.0;
      break;
  }
}

// x^l for an integer exponent (Fortran's ** with an integer power)
double ipow(double x, int l) {
  double r = 1.0;
  for (int q = 0; q < (l < 0 ? -l : l); ++q) r = r * x;
  return l < 0 ? 1.0 / r : r;
}

// get_e_from_temperature (singleideal.F90:2661-2683)
double e_from_t(const Setup& s, double tt) {
  const int lo = s.indx_cp_l, hi = s.indx_cp_r;
  auto cv = [&](int l) { return s.cv_coeff[static_cast<size_t>(l - lo)]; };
  double ee = cv(hi + 1);
  if (s.calorically_perfect == 1) {
    ee = ee + cv(0) * (tt / s.t0 - 1.0);
  } else {
    for (int l = lo; l <= hi; ++l) {
      if (l == -1) ee = ee + cv(l) * std::log(tt / s.t0);
      else ee = ee + cv(l) / (l + 1.0) * (ipow(tt / s.t0, l + 1) - 1.0);
    }
  }
  return ee * s.t0;
}

// get_gamloc (singleideal.F90:4752-4771)
double gamloc_host(const Setup& s, double tt) {
  const int lo = s.indx_cp_l, hi = s.indx_cp_r;
  double cploc;
  if (s.calorically_perfect == 1) {
    cploc = s.cp_coeff[static_cast<size_t>(-lo)];
  } else {
    cploc = 0.0;
    for (int l = lo; l <= hi; ++l) cploc = cploc + s.cp_coeff[static_cast<size_t>(l - lo)] * ipow(tt / s.t0, l);
  }
  return cploc / (cploc - s.rgas0);
}

// velpiros_channel (singleideal.F90:3699-3724)
double velpiros_channel(double yplus, double retau) {
  double yp = yplus;
  double eta = yp / retau;
  eta = std::min(1.0, eta);
  yp = eta * retau;
  const double c = 5.3, vkc = 0.39, vkci = 1.0 / vkc;
  const double c1 = -1.0 / vkc * std::log(vkc) + c;
  const double etastar = 0.275, b_rich = 0.33, eta_rich = 11.0;
  double uinn = vkci * std::log(1.0 + vkc * yp) +
                c1 * (1.0 - std::exp(-yp / eta_rich) - yp / eta_rich * std::exp(-b_rich * yp));
  double uout = c + vkci * std::log(retau) + vkci * std::log(etastar);
  uout = uout + (1 - etastar) / (2 * vkc * etastar) * (1 - (1 - eta) * (1 - eta) / ((1 - etastar) * (1 - etastar)));
  return (eta <= etastar) ? uinn : uout;
}

std::vector<double> read_column(const std::string& path, size_t n) {
  std::ifstream f(path);
  if (!f) throw InputError("cannot open grid file " + path);
  std::vector<double> v;
  std::string tok;
  while (v.size() < n && (f >> tok)) {
    for (char& c : tok)
      if (c == 'd' || c == 'D') c = 'e';
    v.push_back(std::strtod(tok.c_str(), nullptr));
  }
  if (v.size() < n) throw InputError("grid file " + path + " is too short");
  return v;
}

// generate_grid_uniform_x / _y / _z (code/src/grid.F90:822-876)
void uniform_grid(OffsetArray& g, int nmax, int ng, double size, bool periodic, int extra) {
  double d = size / (nmax - 1);
  if (periodic) d = size / nmax;
  g.resize(1 - ng, nmax + ng + extra);
  for (int i = 1 - ng; i <= nmax + ng + extra; ++i) g(i) = (i - 1) * d;
}

// generate_grid_cha (code/src/grid.F90:431-485)
void generate_grid_cha(Setup& s, double jbgrid, double dyptarget, int nsmooy, double retaucha) {
  const int nymax = s.nymax, ng = s.ng, nh = nymax / 2 + 1;
  double alfc = 4.0 / 3.0 * std::pow(retaucha, 0.75) * 2.0 / nymax;
  for (int j = 1; j <= nh; ++j) {
    double rj = static_cast<double>(j - 1);
    double q = rj / jbgrid;
    s.yn(j) = 1.0 / (1.0 + q * q);
    s.yn(j) = s.yn(j) * (rj * dyptarget + std::pow(0.75 * alfc * rj, 4.0 / 3.0) * (q * q));
  }
  double ynf = s.yn(nh);
  for (int j = 1; j <= nh; ++j) s.yn(j) = s.yn(j) / ynf;
  std::vector<double> ynold(nh + 1);
  for (int l = 1; l <= nsmooy; ++l) {
    for (int j = 1; j <= nh; ++j) ynold[j] = s.yn(j);
    for (int j = 2; j <= nymax / 2; ++j) {
      double fsm = 6.0 - 2.0 * (std::tanh((s.yn(j) - 0.75) / 0.15) + 1.0) * 0.5;
      double fsl = 0.5 * (6.0 - fsm);
      s.yn(j) = fsl * ynold[j - 1] + fsm * ynold[j] + fsl * ynold[j + 1];
      s.yn(j) = s.yn(j) / 6.0;
    }
  }
  for (int j = 1; j <= nh; ++j) s.yn(j) = s.yn(j) - 1.0;
  for (int j = 1; j <= nymax / 2; ++j) s.yn(nymax + 2 - j) = -s.yn(j);
  for (int j = 1; j <= nymax; ++j) s.yg(j) = 0.5 * (s.yn(j) + s.yn(j + 1));
  for (int j = 1; j <= ng; ++j) {
    s.yg(nymax + j) = 2.0 - s.yg(nymax + 1 - j);
    s.yg(1 - j) = -2.0 - s.yg(j);
  }
}

// Tanh-stretched staggered channel grid used by the synthetic channel cases:
// yn(j) = tanh(b*(2(j-1)/ny-1))/tanh(b), cell centres midway, ghosts mirrored about the walls
// exactly as generate_grid_cha mirrors them.
void generate_grid_tanh(Setup& s, double b) {
  const int nymax = s.nymax, ng = s.ng;
  for (int j = 1; j <= nymax + 1; ++j)
    s.yn(j) = std::tanh(b * (2.0 * (j - 1) / nymax - 1.0)) / std::tanh(b);
  for (int j = 1; j <= nymax; ++j) s.yg(j) = 0.5 * (s.yn(j) + s.yn(j + 1));
  for (int j = 1; j <= ng; ++j) {
    s.yg(nymax + j) = 2.0 - s.yg(nymax + 1 - j);
    s.yg(1 - j) = -2.0 - s.yg(j);
  }
}

// generate_grid_bl (code/src/grid.F90:310-336), followed by generate_grid_geoprogression
// (:338-368, GRID_BL) or generate_grid_uni_extension (:370-386, GRID_SBLI) above the wall-resolved
// part, and generate_yg (:388-429): smoothing, staggered or node-based yg, mirrored ghosts.
void generate_grid_bl(Setup& s, double jbgrid, double dyptarget, int nymaxwr, double rlywr, double retau,
                      int nsmooy, bool sbli) {
  const int nymax = s.nymax, ng = s.ng;
  const double alfc = 4.0 / 3.0 * std::pow(retau * rlywr, 0.75) / (nymaxwr + 1);
  for (int j = 1; j <= nymaxwr + 1 + ng; ++j) {
    const double rj = static_cast<double>(j - 1);
    const double q = rj / jbgrid;
    s.yn(j) = 1.0 / (1.0 + q * q);
    s.yn(j) = s.yn(j) * (rj * dyptarget + std::pow(0.75 * alfc * rj, 4.0 / 3.0) * (q * q));
  }
  const double ynf = s.yn(nymaxwr + 1);
  for (int j = 1; j <= nymaxwr + ng + 1; ++j) s.yn(j) = s.yn(j) / ynf * rlywr;
  if (nymaxwr < nymax) {
    const double dy1 = s.yn(nymaxwr + 2) - s.yn(nymaxwr + 1);
    if (!sbli) {
      const double rlygp = s.domain_size[1] - rlywr;
      const int nygp = nymax + 1 - (nymaxwr + 1);
      double rgp = 1.01;
      for (int it = 0; it < 100000; ++it) {
        const double rgpold = rgp;
        rgp = 1.0 - (1.0 - rgp) / dy1 * rlygp;
        rgp = std::pow(rgp, 1.0 / nygp);
        if (std::fabs(rgp - rgpold) < TOL_ITER) break;
      }
      for (int j = 1; j <= nygp + ng; ++j) s.yn(nymaxwr + 1 + j) = s.yn(nymaxwr + j) + dy1 * std::pow(rgp, j - 1.0);
    } else {
      for (int j = nymaxwr + 2; j <= nymax + 1 + ng; ++j) s.yn(j) = s.yn(j - 1) + dy1;
    }
  }
  std::vector<double> tmp(static_cast<size_t>(nymax + 2 + ng));
  for (int l = 1; l <= nsmooy; ++l) {
    for (int j = 1; j <= nymax + 1 + ng; ++j) tmp[j] = s.yn(j);
    for (int j = 2; j <= nymax + ng; ++j) s.yn(j) = (tmp[j - 1] + 4.0 * tmp[j] + tmp[j + 1]) / 6.0;
  }
  if (s.is_y_staggered) {
    for (int j = 1; j <= nymax + ng; ++j) s.yg(j) = 0.5 * (s.yn(j) + s.yn(j + 1));
    s.domain_size[1] = s.yn(nymax + 1) - s.yn(1);
    for (int j = 1; j <= ng; ++j) s.yg(1 - j) = -s.yg(j);
  } else {
    for (int j = 1; j <= nymax + ng; ++j) s.yg(j) = s.yn(j);
    s.domain_size[1] = s.yg(nymax) - s.yg(1);
    for (int j = 1; j <= ng; ++j) s.yg(1 - j) = -s.yg(1 + j);
  }
}

// locateval (code/src/parameters.F90:145-164): bisection index il with xx(il) <= x < xx(il+1)
// for an ascending table (1-based; 0 below the table, n at or above its end).
int locateval(const double* xx, int n, double x) {
  int il = 0, juu = n + 1;
  while (juu - il > 1) {
    const int jm = (juu + il) / 2;
    if ((xx[n - 1] > xx[0]) == (x > xx[jm - 1])) il = jm; else juu = jm;
  }
  return il;
}

// read_grid (code/src/grid.F90:877-959)
void read_grid(Setup& s, bool rebuild_ghost) {
  const int ng = s.ng;
  int i1 = 1 - ng, i2 = s.nxmax + ng + 1, j1 = 1 - ng, j2 = s.nymax + ng, k1 = 1 - ng, k2 = s.nzmax + ng;
  if (rebuild_ghost) {
    i1 = 1; i2 = s.nxmax; j1 = 1; j2 = s.nymax; k1 = 1; k2 = s.nzmax;
  }
  auto xv = read_column(s.dir + "/x.dat", i2 - i1 + 1);
  for (int i = i1; i <= i2; ++i) s.xg(i) = xv[i - i1];
  auto yv = read_column(s.dir + "/y.dat", j2 - j1 + 1);
  for (int j = j1; j <= j2; ++j) s.yg(j) = yv[j - j1];
  auto zv = read_column(s.dir + "/z.dat", k2 - k1 + 1);
  for (int k = k1; k <= k2; ++k) s.zg(k) = zv[k - k1];
  std::ifstream ds(s.dir + "/domain_size.dat");
  if (ds) {
    ds >> s.domain_size[0] >> s.domain_size[1] >> s.domain_size[2];
  } else {
    s.domain_size[0] = s.xg(s.nxmax) - s.xg(1);
    s.domain_size[1] = s.yg(s.nymax) - s.yg(1);
    s.domain_size[2] = s.zg(s.nzmax) - s.zg(1);
  }
  if (s.is_y_staggered) {
    auto ynv = read_column(s.dir + "/yn.dat", s.nymax + 1);
    for (int j = 1; j <= s.nymax + 1; ++j) s.yn(j) = ynv[j - 1];
  }
  if (rebuild_ghost) {
    for (int i = 1; i <= ng; ++i) {
      s.xg(1 - i) = 2.0 * s.xg(2 - i) - s.xg(3 - i);
      s.xg(s.nxmax + i) = 2.0 * s.xg(s.nxmax + i - 1) - s.xg(s.nxmax + i - 2);
    }
    s.xg(s.nxmax + ng + 1) = 2.0 * s.xg(s.nxmax + ng) - s.xg(s.nxmax + ng - 1);
    for (int j = 1; j <= ng; ++j) {
      s.yg(1 - j) = 2.0 * s.yg(2 - j) - s.yg(3 - j);
      s.yg(s.nymax + j) = 2.0 * s.yg(s.nymax + j - 1) - s.yg(s.nymax + j - 2);
    }
    for (int k = 1; k <= ng; ++k) {
      s.zg(1 - k) = 2.0 * s.zg(2 - k) - s.zg(3 - k);
      s.zg(s.nzmax + k) = 2.0 * s.zg(s.nzmax + k - 1) - s.zg(s.nzmax + k - 2);
    }
  }
}

// compute_metrics (code/src/grid.F90:71-141) for one direction
void metrics_1d(const OffsetArray& g, int n, int mm, const double* c, const double* cc, OffsetArray& d,
                OffsetArray& d2) {
  d.resize(1, n);
  d2.resize(1, n);
  for (int i = 1; i <= n; ++i) {
    double v = 0.0;
    for (int l = 1; l <= mm; ++l) v = v + c[l - 1] * (g(i + l) - g(i - l));
    d(i) = v;
    double v2 = cc[0] * g(i);
    for (int l = 1; l <= mm; ++l) v2 = v2 + cc[l] * (g(i + l) + g(i - l));
    d2(i) = v2;
  }
}

// set_fluid_prop (singleideal.F90:2685-2774): constant cp, or the cp(T) polynomial of a
// thermally perfect gas (coefficients of cp/R in T_ref units, scaled to T/t0 and times rgas0)
void set_fluid_prop(Setup& s) {
  const IniFile& c = s.ini;
  s.t_ref_dim = c.get_double("flow", "T_ref");
  s.prandtl = c.get_double("fluid", "Prandtl");
  s.gam = c.get_double("fluid", "gam");
  s.visc_model = c.get_int("fluid", "visc_model");
  s.sutherland_s = c.get_double("fluid", "s_suth");
  s.powerlaw_vtexp = c.get_double("fluid", "vt_exp");
  s.calorically_perfect = c.get_int("fluid", "calorically_perfect");
  if (s.calorically_perfect == 0) {
    s.indx_cp_l = c.get_int("fluid", "indx_cp_l");
    s.indx_cp_r = c.get_int("fluid", "indx_cp_r");
    if (s.indx_cp_l > 0 || s.indx_cp_r < 0 || s.indx_cp_r - s.indx_cp_l + 2 > STREAMS_B200_MAX_CP)
      throw InputError("cp polynomial: indx_cp_l <= 0 <= indx_cp_r with at most " +
                       std::to_string(STREAMS_B200_MAX_CP) + " coefficients");
  } else if (s.calorically_perfect == 1) {
    s.indx_cp_l = 0;
    s.indx_cp_r = 0;
  } else {
    throw InputError("calorically_perfect must be 0 or 1");
  }
  s.rfac_type = c.get_int_or("fluid", "rfac_type", 0);
  s.rfac = (s.rfac_type == 0) ? std::pow(s.prandtl, 1.0 / 3.0) : std::pow(s.prandtl, 1.0 / 2.0);
  const int lo = s.indx_cp_l, hi = s.indx_cp_r;
  const size_t ncoef = static_cast<size_t>(hi - lo + 2);
  s.cp_coeff.assign(ncoef, 0.0);
  s.cv_coeff.assign(ncoef, 0.0);
  auto cp = [&](int l) -> double& { return s.cp_coeff[static_cast<size_t>(l - lo)]; };
  auto cv = [&](int l) -> double& { return s.cv_coeff[static_cast<size_t>(l - lo)]; };
  double bcoeff = 0.0;
  if (s.calorically_perfect == 0) {
    const std::vector<double> tmp = c.get_double_array("fluid", "cp_coeff");
    if (tmp.size() != ncoef)
      throw InputError("Error! Check number of cp coefficients (" + std::to_string(ncoef) + " expected)");
    s.cp_coeff = tmp;
    const double tr = s.t_ref_dim;
    double hstar = cp(hi + 1);
    for (int l = lo; l <= hi; ++l) {
      if (l == -1) hstar = hstar + cp(l) * std::log(tr);
      else hstar = hstar + cp(l) / (l + 1) * ipow(tr, l + 1);
    }
    bcoeff = hstar / tr;
    double cp_tref = 0.0;
    for (int l = lo; l <= hi; ++l) cp_tref = cp_tref + cp(l) * ipow(tr, l);
    cp_tref = cp_tref * s.rgas0;
    const double cv_tref = cp_tref - s.rgas0;
    s.gam = cp_tref / cv_tref;
    for (int l = lo; l <= hi; ++l) {
      cp(l) = cp(l) * ipow(tr, l);
      cv(l) = cp(l);
    }
    cv(0) = cp(0) - 1.0;
  }
  s.gm1 = s.gam - 1.0;
  s.gm = 1.0 / s.gm1;
  if (s.calorically_perfect == 1) {
    cv(0) = s.gm;
    cp(0) = s.gm * s.gam;
    bcoeff = cv(0) + 1.0;
  }
  cp(hi + 1) = bcoeff;
  cv(hi + 1) = bcoeff - 1.0;
  for (auto& v : s.cv_coeff) v = v * s.rgas0;
  for (auto& v : s.cp_coeff) v = v * s.rgas0;
}

struct ChanPre {
  double rmb, tw_over_tr;
};

// first part of set_chan_prop (singleideal.F90:2894-2940)
ChanPre chan_prop_pre(Setup& s) {
  s.t_wall = s.t0;
  double rmb, rmtw, trec_over_tb, tw_over_tb, tb_over_tw, tw_over_tr = 0;
  if (s.theta_wall >= -1.0) {
    double thtmp = s.theta_wall;
    rmb = s.mach;
    double gamloc = s.gam;
    for (int l = 1; l <= 50; ++l) {
      double gamlocold = gamloc;
      double gamlocgm1 = gamloc - 1.0;
      trec_over_tb = 1.0 + gamlocgm1 / 2.0 * s.rfac * (rmb * rmb);
      tw_over_tb = 1.0 + thtmp * (trec_over_tb - 1.0);
      tb_over_tw = 1.0 / tw_over_tb;
      tw_over_tr = 1.0 / (trec_over_tb * tb_over_tw);
      s.t_bulk_target = tb_over_tw * s.t_wall;
      gamloc = gamloc_host(s, s.t_bulk_target);
      if (std::fabs(gamloc - gamlocold) < 1.0e-9) break;
    }
    rmtw = rmb * std::sqrt(tb_over_tw);
    s.mach = rmtw;
  } else {
    double thtmp = -1.0;
    rmtw = s.mach;
    rmb = std::sqrt(rmtw * rmtw / (1.0 - s.gm1 / 2.0 * s.rfac * thtmp * (rmtw * rmtw)));
    trec_over_tb = 1.0 + s.gm1 / 2.0 * s.rfac * (rmb * rmb);
    tw_over_tb = 1.0 + thtmp * (trec_over_tb - 1.0);
    tb_over_tw = 1.0 / tw_over_tb;
    tw_over_tr = 1.0 / (trec_over_tb * tb_over_tw);
  }
  return {rmb, tw_over_tr};
}

// set_oblique_shock (singleideal.F90:2953-3016): post-shock state of the impinging shock of
// angle shock_angle through the free stream, and the tanh smoothing length at the top
void set_oblique_shock(Setup& s) {
  const IniFile& c = s.ini;
  const double gam = s.gam, gm1 = s.gm1, mach = s.mach;
  s.xshock_imp = c.get_double("flow", "xshock_imp") * s.l0;
  s.shock_angle = c.get_double("flow", "shock_angle") * pi() / 180.0;
  const double xshock_top = s.xshock_imp - s.yg(s.nymax) / std::tan(s.shock_angle);
  std::vector<double> xg1(static_cast<size_t>(s.nxmax));
  for (int i = 1; i <= s.nxmax; ++i) xg1[i - 1] = s.xg(i);
  const int ig_shock = locateval(xg1.data(), s.nxmax, xshock_top);
  if (ig_shock < 1) throw InputError("the shock meets the top boundary upstream of the domain");
  s.tanhfacs = s.dxg(ig_shock);
  const double sins = std::sin(s.shock_angle), coss = std::cos(s.shock_angle);
  const double mach_normal = mach * sins;
  const double mach_normal2 = mach_normal * mach_normal;
  double mach_normal_past = (1.0 + 0.5 * gm1 * mach_normal2) / (gam * mach_normal2 - 0.5 * gm1);
  mach_normal_past = std::sqrt(mach_normal_past);
  const double vel_ratio = (2.0 + gm1 * mach_normal2) / ((gam + 1.0) * mach_normal2);
  const double rho_ratio = 1.0 / vel_ratio;
  const double p_ratio = 1.0 + 2.0 * gam / (gam + 1.0) * (mach_normal2 - 1.0);
  const double t_ratio = p_ratio / rho_ratio;
  const double defl_tan = 2.0 * coss / sins * ((mach * mach) * (sins * sins) - 1.0) /
                          (2.0 + (mach * mach) * (gam + std::cos(2.0 * s.shock_angle)));
  const double defl = std::atan(defl_tan);
  const double mach_past = mach_normal_past / std::sin(s.shock_angle - defl);
  const double t_past = s.t0 * t_ratio;
  const double c_past = std::sqrt(gam * s.rgas0 * t_past);
  const double u_past = mach_past * c_past * std::cos(defl);
  const double v_past = mach_past * c_past * std::sin(defl);
  const double rho_past = s.rho0 * rho_ratio;
  const double e_past = e_from_t(s, t_past);
  const double etot_past = e_past + 0.5 * (u_past * u_past + v_past * v_past);
  s.winf_past_shock[0] = rho_past;
  s.winf_past_shock[1] = rho_past * u_past;
  s.winf_past_shock[2] = -rho_past * v_past;
  s.winf_past_shock[3] = 0.0;
  s.winf_past_shock[4] = rho_past * etot_past;
}

// set_flow_params (singleideal.F90:2776-2856) for the channel
void set_bl_prop(Setup& s);

void set_flow_params(Setup& s, double reynolds_bulk_target) {
  const IniFile& c = s.ini;
  s.reynolds = c.get_double("flow", "Reynolds");
  s.mach = c.get_double("flow", "Mach");
  s.theta_wall = c.get_double("flow", "theta_wall");
  if (s.bctags[3] == 7) set_oblique_shock(s);
  double gm1h = 0.5 * s.gm1;
  s.t_recovery = s.t0 * (1.0 + gm1h * s.rfac * (s.mach * s.mach));
  s.t_wall = s.theta_wall * (s.t_recovery - s.t0) + s.t0;
  if (s.flow_init == 0) {
    ChanPre pre = chan_prop_pre(s);
    bool visc_exp = (s.visc_model == 1);
    double s2tinf = s.sutherland_s / s.t_ref_dim;
    const int nh = s.nymax / 2;
    std::vector<double> ynh(nh + 1);
    for (int j = 1; j <= nh + 1; ++j) ynh[j - 1] = s.yn(j);
    auto rebulk = [&](double retau) {
      return get_reynolds_cha(retau, pre.rmb, pre.tw_over_tr, s2tinf, s.powerlaw_vtexp, visc_exp, s.gam, s.rfac, nh,
                              ynh.data());
    };
    if (reynolds_bulk_target > 0) {
      // choose the friction Reynolds number whose bulk Reynolds number is the target
      double lo = 5.0, hi = 20000.0;
      for (int it = 0; it < 200; ++it) {
        double mid = 0.5 * (lo + hi);
        if (rebulk(mid) < reynolds_bulk_target) lo = mid; else hi = mid;
        if (hi - lo <= 1e-13 * hi) break;
      }
      s.reynolds = 0.5 * (lo + hi);
    }
    s.reynolds_friction = s.reynolds;
    s.reynolds = rebulk(s.reynolds_friction);
  } else if (s.flow_init == 1) {
    // set_bl_prop (singleideal.F90:2858-2892) converts the input friction Reynolds number into
    // the free-stream one with hasan_meanprofile; the synthetic boundary layer states both
    const IniFile& ci = s.ini;
    if (s.bctags[0] == 9) throw InputError("the laminar boundary layer (xmin = 9) is not supported");
    if (ci.has_section("synthetic")) {
      s.reynolds_friction = ci.get_double_or("synthetic", "reynolds_tau", s.reynolds);
      s.reynolds = ci.get_double("synthetic", "reynolds_delta");
    } else {
      set_bl_prop(s);
    }
  } else {
    throw InputError("flow_init other than 0 (channel) or 1 (boundary layer) is not supported");
  }
  s.p0 = s.rho0 * s.rgas0 * s.t0;
  s.c0 = std::sqrt(s.gam * s.rgas0 * s.t0);
  s.u0 = s.mach * s.c0;
  double e0 = e_from_t(s, s.t0);
  double etot0 = e0 + 0.5 * (s.u0 * s.u0);
  s.s0 = std::log(s.p0 / std::pow(s.rho0, s.gam));
  s.ttot0 = s.t0 * (1.0 + gm1h * (s.mach * s.mach));
  s.ptot0 = s.p0 * std::pow(1.0 + gm1h * (s.mach * s.mach), s.gam / s.gm1);
  s.winf[0] = s.rho0;
  s.winf[1] = s.rho0 * s.u0 * std::cos(s.aoa);
  s.winf[2] = s.rho0 * s.u0 * std::sin(s.aoa);
  s.winf[3] = 0.0;
  s.winf[4] = s.rho0 * etot0;
  if (std::fabs(s.u0) < TOL_ITER) {
    s.mu0 = s.c0 * s.rho0 * s.l0 / s.reynolds;
    s.u0 = s.c0;
  } else {
    s.mu0 = s.u0 * s.rho0 * s.l0 / s.reynolds;
  }
}



// init_channel (singleideal.F90:4344-4419) with the per-rank seeding of an MPI run
void init_channel(Setup& s) {
  const int nxmax = s.nxmax, nymax = s.nymax, nzmax = s.nzmax;
  const double lz = s.domain_size[2];
  double u0_02 = 0.02 * s.u0;
  if (s.rand_type == 0) u0_02 = 0.0;
  double u0_05 = 0.05 * s.u0;
  int nroll = static_cast<int>(lz / s.yn(nymax + 1));
  const int nxl = nxmax / s.x_split, nyl = nymax / s.y_split, nzl = nzmax / s.z_split;
  const int nprocs = s.x_split * s.y_split * s.z_split;
  const double PI = pi();
  for (int rank = 0; rank < nprocs; ++rank) {
    // MPI_Cart_create(reorder=false) row-major rank order: the last dimension varies fastest
    int cx = rank / (s.y_split * s.z_split);
    int cy = (rank / s.z_split) % s.y_split;
    int cz = rank % s.z_split;
    // init_crandom_f(myrank+1) at initialize (singleideal.F90:315-325); rand_type 0 seeds 0 and rescales by 0
    double rescale = 1.0;
    unsigned seed = static_cast<unsigned>(rank + 1);
    if (s.rand_type == 0) {
      seed = 0;
      rescale = 0.0;
    }
    GlibcRand rnd(seed);
    for (int kl = 1; kl <= nzl; ++kl)
      for (int jl = 1; jl <= nyl; ++jl)
        for (int il = 1; il <= nxl; ++il) {
          const int i = cx * nxl + il, j = cy * nyl + jl, k = cz * nzl + kl;
          double rho = s.rho0;
          double yj = s.yg(j);
          double wm2 = 1.5 * s.rho0 * s.u0 * (1.0 - (yj / s.l0) * (yj / s.l0));
          double uu = wm2 / rho, vv = 0.0 / rho, ww = 0.0 / rho;
          double rr[3];
          for (int l = 0; l < 3; ++l) {
            int ir = rnd();
            rr[l] = rescale * static_cast<double>(ir) / RAND_MAX;
            rr[l] = rr[l] - 0.5;
          }
          double ufluc = u0_02 * rr[0], vfluc = u0_02 * rr[1], wfluc = u0_02 * rr[2];
          double zk = s.zg(k);
          vfluc = vfluc + u0_05 * std::sin(0.5 * PI * yj / s.l0) * std::cos(2 * PI * zk / lz * nroll);
          wfluc = wfluc + u0_05 * std::sin(0.5 * PI * yj / s.l0) * std::sin(2 * PI * zk / lz * nroll);
          uu = uu + ufluc;
          vv = vv + vfluc;
          ww = ww + wfluc;
          double rhouu = rho * uu, rhovv = rho * vv, rhoww = rho * ww;
          s.w[s.widx(i, j, k, 0)] = rho;
          s.w[s.widx(i, j, k, 1)] = rhouu;
          s.w[s.widx(i, j, k, 2)] = rhovv;
          s.w[s.widx(i, j, k, 3)] = rhoww;
          double tt = s.p0 / s.rgas0 / rho;
          double ee = e_from_t(s, tt);
          s.w[s.widx(i, j, k, 4)] = rho * ee + 0.5 * (rhouu * rhouu + rhovv * rhovv + rhoww * rhoww) / rho;
        }
  }
}

// Synthetic channel field: Poiseuille u (peak 1.5 u0), v = w = 0, rho = rho0, T = T_wall,
// plus uniform random perturbations of +-amp*u0 on u, v, w from glibc rand (seed), drawn in
// k, j, i order, three per cell.
void init_channel_synthetic(Setup& s, double amp, int seed) {
  GlibcRand rnd(static_cast<unsigned>(seed));
  for (int k = 1; k <= s.nzmax; ++k)
    for (int j = 1; j <= s.nymax; ++j)
      for (int i = 1; i <= s.nxmax; ++i) {
        double rr[3];
        for (int l = 0; l < 3; ++l) rr[l] = 2.0 * (static_cast<double>(rnd()) / RAND_MAX) - 1.0;
        double rho = s.rho0;
        double yj = s.yg(j) / s.l0;
        double uu = 1.5 * s.u0 * (1.0 - yj * yj) + amp * s.u0 * rr[0];
        double vv = amp * s.u0 * rr[1];
        double ww = amp * s.u0 * rr[2];
        double rhouu = rho * uu, rhovv = rho * vv, rhoww = rho * ww;
        double ee = e_from_t(s, s.t_wall);
        s.w[s.widx(i, j, k, 0)] = rho;
        s.w[s.widx(i, j, k, 1)] = rhouu;
        s.w[s.widx(i, j, k, 2)] = rhovv;
        s.w[s.widx(i, j, k, 3)] = rhoww;
        s.w[s.widx(i, j, k, 4)] = rho * ee + 0.5 * (rhouu * rhouu + rhovv * rhovv + rhoww * rhoww) / rho;
      }
}

// Synthetic spatially developing boundary layer (the benchmark's boundary-layer workload; it
// replaces init_bl, singleideal.F90:3252-3423, whose hasan_meanprofile is not restated):
//   thickness   delta(x) = l0 (1 + (x/l0) 0.27^1.2 / Re^0.2)^(5/6)   (the Urbin-Knight growth that
//               recyc_prepare reports), viscous length deltav(x) = (l0/Re_tau) (delta/l0)^(1/8)
//   mean flow   u = u0 min(y/delta, 1)^(1/7), Crocco-Busemann temperature
//               T = T_w + (T_r - T_w) u/u0 + (t0 - T_r) (u/u0)^2, rho = p0 / (R T),
//               v from continuity exactly as init_bl integrates it, w = 0
//   field       mean + uniform random perturbations of +-amp u0 on u, v, w (glibc rand, seed of
//               the single rank, 3 draws per cell in k, j, i order, as init_bl draws them)
void init_bl_synthetic(Setup& s, double amp) {
  const int nx = s.nxmax, ny = s.nymax, nz = s.nzmax, ng = s.ng;
  const int nxg = nx + 2 * ng + 1;  // xg(1-ng : nx+ng+1)
  s.deltavec.assign(nxg, 0.0);
  s.deltavvec.assign(nxg, 0.0);
  const double grow = std::pow(0.27, 1.2) / std::pow(s.reynolds, 0.2);
  for (int i = 1 - ng; i <= nx + ng + 1; ++i) {
    const double d = s.l0 * std::pow(1.0 + s.xg(i) / s.l0 * grow, 5.0 / 6.0);
    s.deltavec[i + ng - 1] = d;
    s.deltavvec[i + ng - 1] = s.l0 / s.reynolds_friction * std::pow(d / s.l0, 0.125);
  }
  // wmean(1-ng:nx+ng+1, 1:ny, 4)
  const int wi = nx + 2 * ng + 1;
  s.wmean.assign(static_cast<size_t>(wi) * ny * 4, 0.0);
  auto WM = [&](int i, int j, int m) -> double& {
    return s.wmean[(static_cast<size_t>(m - 1) * ny + (j - 1)) * wi + (i + ng - 1)];
  };
  for (int i = 1 - ng; i <= nx + ng + 1; ++i) {
    const double delta = s.deltavec[i + ng - 1];
    for (int j = 1; j <= ny; ++j) {
      const double yy = s.yg(j);
      const double eta = std::min(std::max(yy, 0.0) / delta, 1.0);
      const double ub = std::pow(eta, 1.0 / 7.0);
      const double tt = s.t_wall + (s.t_recovery - s.t_wall) * ub + (s.t0 - s.t_recovery) * ub * ub;
      const double rho = s.p0 / (s.rgas0 * tt);
      WM(i, j, 1) = rho;
      WM(i, j, 2) = rho * ub * s.u0;
    }
  }
  for (int i = 1 - ng; i <= nx + ng; ++i)
    for (int j = 2; j <= ny; ++j) {
      const double vi_j = -(WM(i + 1, j, 2) - WM(i, j, 2)) / (s.xg(i + 1) - s.xg(i));
      const double vi_jm = -(WM(i + 1, j - 1, 2) - WM(i, j - 1, 2)) / (s.xg(i + 1) - s.xg(i));
      const double vi = 0.5 * (vi_j + vi_jm);
      WM(i, j, 3) = WM(i, j - 1, 3) + vi * (s.yg(j) - s.yg(j - 1));
    }
  const unsigned seed = s.rand_type == 0 ? 0u : 1u;
  const double rescale = s.rand_type == 0 ? 0.0 : 1.0;
  GlibcRand rnd(seed);
  const double ua = 2.0 * amp * s.u0;
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double rho = WM(i, j, 1);
        double rr[3];
        for (int l = 0; l < 3; ++l) rr[l] = rescale * static_cast<double>(rnd()) / RAND_MAX - 0.5;
        const double uu = WM(i, j, 2) / rho + ua * rr[0];
        const double vv = WM(i, j, 3) / rho + ua * rr[1];
        const double ww = WM(i, j, 4) / rho + ua * rr[2];
        const double rhouu = rho * uu, rhovv = rho * vv, rhoww = rho * ww;
        s.w[s.widx(i, j, k, 0)] = rho;
        s.w[s.widx(i, j, k, 1)] = rhouu;
        s.w[s.widx(i, j, k, 2)] = rhovv;
        s.w[s.widx(i, j, k, 3)] = rhoww;
        const double tt = s.p0 / s.rgas0 / rho;
        const double ee = e_from_t(s, tt);
        s.w[s.widx(i, j, k, 4)] = rho * ee + 0.5 * (rhouu * rhouu + rhovv * rhovv + rhoww * rhoww) / rho;
      }
  s.rng_seed = seed;
  s.rng_draws = 3LL * nx * ny * nz;
}

// hasan_meanprofile (singleideal.F90:4090-4249): mean velocity, temperature, density and
// viscosity of a compressible turbulent boundary layer of thickness d99 on a fine uniform grid of
// 10000 intervals (inner law with a van Driest damped mixing length, Coles wake of strength from
// Re_theta, Crocco-Busemann-type temperature with spr), iterated until Re_theta (imode 0, Re_tau
// given) or Re_tau (imode 1, Re_theta given) changes by less than 1e-5; with icompute /= 0 the
// profiles are interpolated linearly (pol_int with m = 2) onto ye(1:n).  Same operations and
// order as the reference: the profiles and the thicknesses are reproducible bit for bit.
struct HasanState {
  double retau = 0, retheta = 0, redelta = 0, th = 0, cf = 0, ch = 0, mtau = 0, deltav = 0;
};
void hasan_meanprofile(int n, double d99, double mach, double theta, HasanState& h, double pr, double spr,
                       double rfac, double gam, double vtexp, bool visc_exp, double s2tinf, const double* ye,
                       double* ue, double* te, double* rhoe, double* mue, int imode, int icompute) {
  constexpr int ny = 10000, nyext = 2 * ny;
  const double pi_h = 4.0 * std::atan(1.0);
  const double gm1h = 0.5 * (gam - 1.0);
  const double tr = 1.0 + gm1h * rfac * (mach * mach);
  const double tw = 1.0 + theta * (tr - 1.0);
  const double apl = 17.0, vkc = 0.41;
  const int nitermax = 10000;
  const double tol = 0.00001;
  const double dy = d99 / ny;
  // index j = 1..ny+1 of the reference at [j-1]
  std::vector<double> y(ny + 1), u(ny + 1), t(ny + 1), rho(ny + 1), mu(ny + 1), ypl(ny + 1), upl(ny + 1),
      yst(ny + 1), d(ny + 1), mut(ny + 1), wake(ny + 1), swake(ny + 1);
  std::vector<double> yext(nyext + 1), uext(nyext + 1), text(nyext + 1), rhoext(nyext + 1), muext(nyext + 1);
  for (int j = 1; j <= ny + 1; ++j) y[j - 1] = (j - 1) * dy;
  for (int j = 1; j <= nyext + 1; ++j) yext[j - 1] = (j - 1) * dy;
  // sin(pi y/d99) of the wake function does not change between iterations
  for (int j = 0; j <= ny; ++j) swake[j] = std::sin(pi_h * (y[j] / d99));
  const double ufac = 0.99;
  for (int j = 0; j <= ny; ++j) u[j] = std::min(1.0, y[j] / d99);
  const double uinf = u[ny] / ufac;
  for (int j = 0; j <= ny; ++j) u[j] = u[j] / uinf;
  int niter = 0;
  double& retau = h.retau;
  double& retheta = h.retheta;
  if (imode == 0) retheta = 1000.0; else retau = 200.0;
  h.mtau = 0.1;
  double absdiff = std::numeric_limits<double>::max();
  auto visc = [&](double tt) {
    return visc_exp ? std::pow(tt, vtexp) : std::pow(tt, 1.5) * (1.0 + s2tinf) / (tt + s2tinf);
  };
  double uinf_plus = 0.0;
  while (absdiff > tol) {
    ++niter;
    if (niter > nitermax) break;
    const double rethetaold = retheta, retauold = retau;
    // the Coles wake strength depends on retheta only (the reference forms it at every point)
    const double z1 = retheta / 425.0 - 1.0;
    const double picole = 0.69 * (1.0 - std::exp(-0.243 * std::sqrt(z1) - 0.15 * z1));
    for (int j = 0; j <= ny; ++j) {
      t[j] = tw + (tr - tw) * (spr * u[j] + (1.0 - spr) * (u[j] * u[j])) + (1.0 - tr) * (u[j] * u[j]);
      rho[j] = 1.0 / t[j];
      mu[j] = visc(t[j]);
      ypl[j] = (y[j] / d99) * retau;
      yst[j] = ypl[j] * std::sqrt(rho[j] / rho[0]) * mu[0] / mu[j];
      const double e = 1.0 - std::exp(-yst[j] / (apl + 19.3 * h.mtau));
      d[j] = e * e;
      mut[j] = mu[j] / mu[0] * vkc * yst[j] * d[j];
      wake[j] = picole / vkc * pi_h * swake[j];
    }
    upl[0] = 0.0;
    for (int j = 1; j <= ny; ++j) {
      const double uint_inn_j = 1.0 / (mu[j] / mu[0] + mut[j]);
      const double uint_inn_jm = 1.0 / (mu[j - 1] / mu[0] + mut[j - 1]);
      const double uint_out_j = std::sqrt(rho[0] / rho[j]) / retau * wake[j];
      const double uint_out_jm = std::sqrt(rho[0] / rho[j - 1]) / retau * wake[j - 1];
      const double uint_j = uint_inn_j + uint_out_j;
      const double uint_jm = uint_inn_jm + uint_out_jm;
      const double uint = 0.5 * (uint_j + uint_jm);
      upl[j] = upl[j - 1] + uint * (ypl[j] - ypl[j - 1]);
    }
    uinf_plus = upl[ny] / ufac;
    for (int j = 0; j <= ny; ++j) u[j] = upl[j] / uinf_plus;
    h.th = 0.0;
    for (int j = 1; j <= ny; ++j) {
      const double thint_j = rho[j] * u[j] * (1.0 - u[j]);
      const double thint_jm = rho[j - 1] * u[j - 1] * (1.0 - u[j - 1]);
      const double thint = 0.5 * (thint_j + thint_jm);
      h.th = h.th + thint * (y[j] - y[j - 1]);
    }
    h.cf = 2.0 / (uinf_plus * uinf_plus) * rho[0];
    h.ch = 0.5 * h.cf * spr / pr;
    h.mtau = mach * std::sqrt(0.5 * h.cf);
    if (imode == 0) {
      retheta = retau * h.th / d99 * mu[0] / rho[0] * uinf_plus;
      absdiff = std::fabs(retheta - rethetaold);
    } else {
      retau = retheta * d99 / h.th / mu[0] * rho[0] / uinf_plus;
      absdiff = std::fabs(retau - retauold);
    }
    h.redelta = retheta * d99 / h.th;
  }
  h.deltav = d99 / retau;
  if (icompute == 0) return;
  for (int j = 0; j <= ny; ++j) {
    uext[j] = u[j];
    text[j] = t[j];
  }
  const double dudy = (uext[ny] - uext[ny - 1]) / (yext[ny] - yext[ny - 1]);
  for (int j = ny + 1; j <= nyext; ++j) {
    uext[j] = uext[ny] + dudy * (yext[j] - yext[ny]);
    uext[j] = std::min(uext[j], 1.0);
    text[j] = tw + (tr - tw) * (spr * uext[j] + (1.0 - spr) * (uext[j] * uext[j])) + (1.0 - tr) * (uext[j] * uext[j]);
  }
  for (int j = 0; j <= nyext; ++j) {
    rhoext[j] = 1.0 / text[j];
    muext[j] = visc(text[j]);
  }
  for (int j = 0; j < n; ++j) ue[j] = rhoe[j] = te[j] = mue[j] = 1.0;
  ue[0] = uext[0];
  rhoe[0] = rhoext[0];
  te[0] = text[0];
  mue[0] = muext[0];
  for (int j = 0; j < n; ++j) {
    const double yy = ye[j];
    if (!(yy < yext[nyext])) continue;
    // locateval (parameters.F90:145-164) on the uniform yext, then pol_int (Neville, :120-143)
    // with m = 2 on the pair jjj, jjj+1
    int il = 0, juu = nyext + 2;
    while (juu - il > 1) {
      const int jm = (juu + il) / 2;
      if ((yext[nyext] > yext[0]) == (yy > yext[jm - 1])) il = jm; else juu = jm;
    }
    const int jjj = std::min(std::max(il, 1), nyext + 1 + 1 - 2);
    const double x1 = yext[jjj - 1], x2 = yext[jjj];
    auto lin = [&](const std::vector<double>& f) {
      double v = (yy - x2) * f[jjj - 1] + (x1 - yy) * f[jjj];
      return v / (x1 - x2);
    };
    ue[j] = lin(uext);
    rhoe[j] = lin(rhoext);
    te[j] = lin(text);
    mue[j] = lin(muext);
  }
}

// set_bl_prop (singleideal.F90:2858-2892): the input Reynolds number of a turbulent boundary
// layer is the friction one; the free-stream (thickness-based) one follows from the mean profile
void set_bl_prop(Setup& s) {
  const bool visc_exp = s.visc_model == 1;
  const double s2tinf = s.sutherland_s / s.t_ref_dim;
  s.reynolds_friction = s.reynolds;
  const int ny = s.nymax;
  std::vector<double> yvec(ny), uv(ny), tv(ny), rv(ny), mv(ny);
  for (int j = 1; j <= ny; ++j) yvec[j - 1] = s.yg(j);
  HasanState h;
  h.retau = s.reynolds_friction;
  hasan_meanprofile(ny, s.l0, s.mach, s.theta_wall, h, s.prandtl, 0.8, s.rfac, s.gam, s.powerlaw_vtexp, visc_exp,
                    s2tinf, yvec.data(), uv.data(), tv.data(), rv.data(), mv.data(), 0, 0);
  s.reynolds = h.redelta;
}

// blvec.bin (init_bl, singleideal.F90:3293-3297, 3360-3364): one Fortran unformatted record
// holding cfvec, thvec, deltavec, deltavvec over xg(1-ng .. nxmax+ng+1)
bool read_blvec(const std::string& path, size_t n, std::vector<double>& cf, std::vector<double>& th,
                std::vector<double>& de, std::vector<double>& dv) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  int32_t len = 0;
  f.read(reinterpret_cast<char*>(&len), 4);
  if (!f || static_cast<size_t>(len) != 4 * n * 8) throw InputError(path + ": unexpected record length");
  for (auto* v : {&cf, &th, &de, &dv}) {
    v->resize(n);
    f.read(reinterpret_cast<char*>(v->data()), static_cast<std::streamsize>(n * 8));
  }
  if (!f) throw InputError(path + ": short read");
  return true;
}
void write_blvec(const std::string& path, const std::vector<double>& cf, const std::vector<double>& th,
                 const std::vector<double>& de, const std::vector<double>& dv) {
  std::ofstream f(path, std::ios::binary);
  if (!f) return;  // the file is a cache of the reference's; a read-only directory only loses it
  const int32_t len = static_cast<int32_t>(4 * cf.size() * 8);
  f.write(reinterpret_cast<const char*>(&len), 4);
  for (const auto* v : {&cf, &th, &de, &dv}) f.write(reinterpret_cast<const char*>(v->data()), v->size() * 8);
  f.write(reinterpret_cast<const char*>(&len), 4);
}

// init_bl (singleideal.F90:3252-3423) and add_synthetic_perturbations (:3587-3685) for the single
// block: the thickness delta(x) and viscous length along x from the mean profile at the inflow
// (Re_tau given) and a momentum-thickness march in both directions (Re_theta given, delta
// iterated to 1e-9), the mean field wmean from the profile at every station, v from continuity,
// +-1 % random velocity perturbations (3 draws per cell in k, j, i order), then the streak /
// vortex perturbations of add_synthetic_perturbations (4 phase draws) with +-1.5 % random
// perturbations scaled by y/l0 below the local thickness (3 draws per such cell).
void init_bl(Setup& s) {
  const int nx = s.nxmax, ny = s.nymax, nz = s.nzmax, ng = s.ng;
  const int nxt = nx + 2 * ng + 1;  // stations 1-ng .. nx+ng+1
  auto X = [&](int i) { return i + ng - 1; };
  const bool visc_exp = s.visc_model == 1;
  const double s2tinf = s.sutherland_s / s.t_ref_dim, vtexp = s.powerlaw_vtexp, spr = 0.8;
  std::vector<double> yvec(ny), uvec(ny), tvec(ny), rhovec(ny), viscvec(ny);
  for (int j = 1; j <= ny; ++j) yvec[j - 1] = s.yg(j);
  std::vector<double> cfvec, thvec, deltavec, deltavvec;
  const std::string blvec = s.dir + "/blvec.bin";
  if (!read_blvec(blvec, nxt, cfvec, thvec, deltavec, deltavvec)) {
    cfvec.assign(nxt, 0.0);
    thvec.assign(nxt, 0.0);
    deltavec.assign(nxt, 0.0);
    deltavvec.assign(nxt, 0.0);
    std::vector<double> retauvec(nxt, 0.0);
    auto hasan = [&](double d99, HasanState& h, int imode) {
      hasan_meanprofile(ny, d99, s.mach, s.theta_wall, h, s.prandtl, spr, s.rfac, s.gam, vtexp, visc_exp, s2tinf,
                        yvec.data(), uvec.data(), tvec.data(), rhovec.data(), viscvec.data(), imode, 0);
    };
    HasanState h;
    h.retau = s.reynolds_friction;
    hasan(s.l0, h, 0);
    const double retheta_inflow = h.retheta;
    deltavec[X(1)] = s.l0;
    deltavvec[X(1)] = h.deltav;
    cfvec[X(1)] = h.cf;
    thvec[X(1)] = h.th;
    retauvec[X(1)] = s.reynolds_friction;
    // one station from its neighbour nb (the previous one of the march)
    auto station = [&](int i, int nb, double& retheta) {
      thvec[X(i)] = thvec[X(nb)] + (i > nb ? 1.0 : -1.0) * 0.5 * std::fabs(s.xg(i) - s.xg(nb)) * cfvec[X(nb)];
      retheta = retheta / thvec[X(nb)] * thvec[X(i)];
      double delta = deltavec[X(nb)] / thvec[X(nb)] * thvec[X(i)];
      HasanState hs;
      while (true) {
        const double deltaold = delta;
        hs = HasanState();
        hs.retheta = retheta;
        hasan(delta, hs, 1);
        delta = deltavec[X(nb)] * hs.retau / retauvec[X(nb)] * std::sqrt(cfvec[X(nb)] / hs.cf);
        if (std::fabs(delta - deltaold) < 0.000000001) break;
      }
      deltavec[X(i)] = delta;
      cfvec[X(i)] = hs.cf;
      deltavvec[X(i)] = hs.deltav;
      retauvec[X(i)] = hs.retau;
    };
    double retheta = retheta_inflow;
    for (int i = 1; i <= ng; ++i) station(1 - i, 2 - i, retheta);
    retheta = retheta_inflow;
    for (int i = 2; i <= nx + ng + 1; ++i) station(i, i - 1, retheta);
    write_blvec(blvec, cfvec, thvec, deltavec, deltavvec);
  }
  s.deltavec = deltavec;
  s.deltavvec = deltavvec;
  // wmean(1-ng:nx+ng+1, 1:ny, 4) from the profile of every station (independent stations)
  s.wmean.assign(static_cast<size_t>(nxt) * ny * 4, 0.0);
  auto WM = [&](int i, int j, int m) -> double& {
    return s.wmean[(static_cast<size_t>(m - 1) * ny + (j - 1)) * nxt + X(i)];
  };
  {
    const unsigned nthr = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nthr; ++t)
      pool.emplace_back([&, t] {
        std::vector<double> uv(ny), tv(ny), rv(ny), mv(ny);
        for (int i = 1 - ng + static_cast<int>(t); i <= nx + ng + 1; i += static_cast<int>(nthr)) {
          HasanState hs;
          hs.retau = deltavec[X(i)] / deltavvec[X(i)];
          hasan_meanprofile(ny, deltavec[X(i)], s.mach, s.theta_wall, hs, s.prandtl, spr, s.rfac, s.gam, vtexp,
                            visc_exp, s2tinf, yvec.data(), uv.data(), tv.data(), rv.data(), mv.data(), 0, 1);
          for (int j = 1; j <= ny; ++j) {
            WM(i, j, 1) = rv[j - 1] * s.rho0;
            WM(i, j, 2) = rv[j - 1] * uv[j - 1] * s.u0 * s.rho0;
          }
        }
      });
    for (auto& th : pool) th.join();
  }
  for (int i = 1 - ng; i <= nx + ng; ++i)
    for (int j = 2; j <= ny; ++j) {
      const double vi_j = -(WM(i + 1, j, 2) - WM(i, j, 2)) / (s.xg(i + 1) - s.xg(i));
      const double vi_jm = -(WM(i + 1, j - 1, 2) - WM(i, j - 1, 2)) / (s.xg(i + 1) - s.xg(i));
      const double vi = 0.5 * (vi_j + vi_jm);
      WM(i, j, 3) = WM(i, j - 1, 3) + vi * (s.yg(j) - s.yg(j - 1));
    }
  const unsigned seed = s.rand_type == 0 ? 0u : 1u;
  const double rescale = s.rand_type == 0 ? 0.0 : 1.0;
  GlibcRand rnd(seed);
  long long draws = 0;
  auto crandom = [&]() {
    ++draws;
    return rescale * static_cast<double>(rnd()) / RAND_MAX;
  };
  const double u0_02 = s.rand_type == 0 ? 0.0 : 0.02 * s.u0;
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double rho = WM(i, j, 1);
        double rr[3];
        for (int l = 0; l < 3; ++l) rr[l] = crandom();
        for (int l = 0; l < 3; ++l) rr[l] = rr[l] - 0.5;
        const double uu = WM(i, j, 2) / rho + u0_02 * rr[0];
        const double vv = WM(i, j, 3) / rho + u0_02 * rr[1];
        const double ww = WM(i, j, 4) / rho + u0_02 * rr[2];
        const double rhouu = rho * uu, rhovv = rho * vv, rhoww = rho * ww;
        s.w[s.widx(i, j, k, 0)] = rho;
        s.w[s.widx(i, j, k, 1)] = rhouu;
        s.w[s.widx(i, j, k, 2)] = rhovv;
        s.w[s.widx(i, j, k, 3)] = rhoww;
        const double tt = s.p0 / s.rgas0 / rho;
        const double ee = e_from_t(s, tt);
        s.w[s.widx(i, j, k, 4)] = rho * ee + 0.5 * (rhouu * rhouu + rhovv * rhovv + rhoww * rhoww) / rho;
      }
  // add_synthetic_perturbations
  double sp[5][7] = {{12.0, 1.2, -0.25, 0.12, 10.0, 120.0, 0.0},
                     {0.3, 0.3, -0.06, 1.2, 0.9, 0.333, 1.0},
                     {0.45, 0.2, -0.05, 0.6, 0.9, 0.25, 1.0},
                     {0.6, 0.08, -0.04, 0.4, 0.9, 0.2, 1.0},
                     {0.5, 0.04, -0.03, 0.2, 0.9, 0.166, 1.0}};
  const double pi_p = pi();
  const double lz = s.domain_size[2];
  const double rho_wall = WM(1, 1, 1);
  const double tau_wall = cfvec[X(1)] * s.rho0 * (s.u0 * s.u0) * 0.5;
  const double u_tau = std::sqrt(tau_wall / rho_wall);
  sp[0][0] = sp[0][0] * deltavvec[X(1)];
  sp[0][3] = sp[0][3] * u_tau / deltavvec[X(1)];
  sp[0][4] = sp[0][4] * u_tau;
  const double lz_plus = lz / deltavvec[X(1)];
  const long long n_streaks = std::llround(lz_plus / sp[0][5]);
  sp[0][5] = lz / static_cast<double>(n_streaks);
  for (int l = 1; l < 5; ++l) {
    sp[l][0] = sp[l][0] * deltavec[X(1)];
    sp[l][3] = sp[l][3] * s.u0 / deltavec[X(1)];
    sp[l][4] = sp[l][4] * s.u0;
    sp[l][5] = sp[l][5] * lz;
    const double rr = crandom();
    sp[l][6] = sp[l][6] * 2.0 * pi_p * rr;
  }
  const double u0_03 = s.rand_type == 0 ? 0.0 : 0.03 * s.u0;
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double rhofac = WM(i, 1, 1) / WM(i, j, 1);
        rhofac = std::sqrt(rhofac) * s.u0;
        double up = 0.0, vp = 0.0, wp = 0.0;
        const double xx = s.xg(i), yy = s.yg(j), zz = s.zg(k);
        for (int l = 1; l < 5; ++l) {
          const double arg_sin = sp[l][3] * xx / sp[l][4];
          const double arg_cos = 2.0 * pi_p * zz / sp[l][5] + sp[l][6];
          const double ys = yy / sp[l][0];
          const double ufy = ys * std::exp(-ys);
          const double vfy = (ys * ys) * std::exp(-(ys * ys));
          up = up + sp[l][1] * ufy * std::sin(arg_sin) * std::cos(arg_cos);
          vp = vp + sp[l][2] * vfy * std::sin(arg_sin) * std::cos(arg_cos);
          const double dup_dx = sp[l][1] * ufy * sp[l][3] / sp[l][4] * std::cos(arg_sin);
          const double dvfy_dy = 2.0 * ys / sp[l][0] * std::exp(-(ys * ys)) * (1.0 - (ys * ys));
          const double dvp_dy = sp[l][2] * dvfy_dy * std::sin(arg_sin);
          wp = wp - (dup_dx + dvp_dy) * std::sin(arg_cos) * sp[l][5] / (2.0 * pi_p);
        }
        up = up * rhofac;
        vp = vp * rhofac;
        wp = wp * rhofac;
        const double delta = deltavec[X(i)];
        if (yy < delta) {
          double rr3[3];
          for (int l = 0; l < 3; ++l) rr3[l] = crandom();
          for (int l = 0; l < 3; ++l) rr3[l] = rr3[l] - 0.5;
          up = up + u0_03 * rr3[0] * (yy / s.l0);
          vp = vp + u0_03 * rr3[1] * (yy / s.l0);
          wp = wp + u0_03 * rr3[2] * (yy / s.l0);
        }
        double* w1 = &s.w[s.widx(i, j, k, 0)];
        double& w2 = s.w[s.widx(i, j, k, 1)];
        double& w3 = s.w[s.widx(i, j, k, 2)];
        double& w4 = s.w[s.widx(i, j, k, 3)];
        const double rho = *w1;
        w2 = w2 + up * *w1;
        w3 = w3 + vp * *w1;
        w4 = w4 + wp * *w1;
        const double tt = s.p0 / s.rgas0 / rho;
        const double ee = e_from_t(s, tt);
        s.w[s.widx(i, j, k, 4)] = rho * ee + 0.5 * (w2 * w2 + w3 * w3 + w4 * w4) / *w1;
      }
  s.rng_seed = seed;
  s.rng_draws = draws;
}

// recyc_prepare (singleideal.F90:1512-1588), single block
void recyc_prepare(Setup& s) {
  const int nx = s.nxmax, ny = s.nymax, ng = s.ng;
  s.x_recyc = s.ini.get_double("bc", "x_recyc") * s.l0;
  const double bexprecyc_base = 0.13, my_eta0 = 0.08, my_deltablend = 1.10;
  std::vector<double> xg1(static_cast<size_t>(nx));
  for (int i = 1; i <= nx; ++i) xg1[i - 1] = s.xg(i);
  int ig_recyc = locateval(xg1.data(), nx, s.x_recyc);
  s.i_recyc = ig_recyc;
  if (s.i_recyc < ng) {
    s.i_recyc = ng;
    ig_recyc = s.i_recyc;
  }
  auto DV = [&](int i) { return s.deltavec[i + ng - 1]; };
  auto DVV = [&](int i) { return s.deltavvec[i + ng - 1]; };
  s.betarecyc = DVV(ig_recyc) / DVV(1);
  s.glund1 = std::pow(DV(ig_recyc) / DV(1), bexprecyc_base);
  const int n = ny + 2 * ng;
  s.yplus_inflow.assign(n, 0.0); s.eta_inflow.assign(n, 0.0); s.yplus_recyc.assign(n, 0.0);
  s.eta_recyc.assign(n, 0.0); s.eta_recyc_blend.assign(n, 0.0);
  for (int j = 1 - ng; j <= ny + ng; ++j) {
    const double y = s.yg(j);
    const size_t q = static_cast<size_t>(j + ng - 1);
    s.yplus_inflow[q] = y / DVV(1);
    s.eta_inflow[q] = y / DV(1);
    s.yplus_recyc[q] = y / DVV(ig_recyc);
    s.eta_recyc[q] = y / DV(ig_recyc);
    const double r = DV(1) / DV(ig_recyc);
    s.eta_recyc_blend[q] = y * (std::pow(r, bexprecyc_base) +
                                0.5 * (1.0 + std::tanh(std::log(std::fabs(s.eta_recyc[q]) / my_eta0) / my_deltablend)) *
                                    (r - std::pow(r, bexprecyc_base)));
  }
  const double alfa_blend = 4.0, beta_blend = 0.2, c_blend = 1.0 - 2.0 * beta_blend;
  s.map_j_inn.assign(ny, 0); s.map_j_out.assign(ny, 0); s.map_j_out_blend.assign(ny, 0);
  s.weta_inflow.assign(ny, 0.0);
  const double* yr = &s.yplus_recyc[ng];  // yplus_recyc(1:ny)
  const double* er = &s.eta_recyc[ng];
  const double* eb = &s.eta_recyc_blend[ng];
  for (int j = 1; j <= ny; ++j) {
    const size_t q = static_cast<size_t>(j + ng - 1);
    s.map_j_inn[j - 1] = locateval(yr, ny, s.yplus_inflow[q]);
    s.map_j_out[j - 1] = locateval(er, ny, s.eta_inflow[q]);
    s.map_j_out_blend[j - 1] = locateval(eb, ny, s.eta_inflow[q]);
    s.weta_inflow[j - 1] = 0.5 * (1.0 + std::tanh((alfa_blend * (s.eta_inflow[q] - beta_blend)) /
                                                  (beta_blend + s.eta_inflow[q] * c_blend)) /
                                            std::tanh(alfa_blend));
  }
  // jbl_inflow (init_bl, singleideal.F90:3281): last y node below l0
  std::vector<double> y1(static_cast<size_t>(ny));
  for (int j = 1; j <= ny; ++j) y1[j - 1] = s.yg(j);
  s.jbl_inflow = locateval(y1.data(), ny, s.l0);
  // the mean inflow planes wmean(1-i, j, m), i = 1..ng, that bcrecyc_subroutine_3 rescales
  const int wi = nx + 2 * ng + 1;
  s.wmean_inflow.assign(static_cast<size_t>(4) * ny * ng, 0.0);
  for (int m = 1; m <= 4; ++m)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= ng; ++i)
        s.wmean_inflow[(static_cast<size_t>(m - 1) * ny + (j - 1)) * ng + (i - 1)] =
            s.wmean[(static_cast<size_t>(m - 1) * ny + (j - 1)) * wi + (1 - i + ng - 1)];
}

// read_field (code/src/field.F90:1853-1905): rst.bin = nv global arrays, Fortran order, native REAL64
void read_rst(Setup& s) {
  const std::string path = s.dir + "/rst.bin";
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) throw InputError("cannot open " + path);
  std::vector<double> plane(static_cast<size_t>(s.nxmax));
  for (int m = 0; m < 5; ++m)
    for (int k = 1; k <= s.nzmax; ++k)
      for (int j = 1; j <= s.nymax; ++j) {
        if (std::fread(plane.data(), sizeof(double), plane.size(), f) != plane.size()) {
          std::fclose(f);
          throw InputError("rst.bin is too short");
        }
        for (int i = 1; i <= s.nxmax; ++i) s.w[s.widx(i, j, k, m)] = plane[i - 1];
      }
  std::fclose(f);
}

void read_field_info(Setup& s) {
  IniFile fi = IniFile::parse_file(s.dir + "/field_info0.dat");
  s.icyc0 = fi.get_int("field_info", "icyc0");
  s.time0 = fi.get_double("field_info", "time0");
  s.itav = fi.get_int_or("field_info", "itav", 0);
  s.time_from_last_stat = fi.get_double_or("field_info", "time_from_last_stat", 0.0);
}

// read_stats / read_stats_3d (singleideal.F90:1646-1700, 1728-1783): per statistic one global
// plane (nx*ny) or volume (nx*ny*nz) in Fortran order, transposed into w_stat(l, i, j[, k])
void read_stats_files(Setup& s) {
  auto read_blocks = [&](const std::string& name, int nv, size_t block, std::vector<double>& out) {
    const std::string path = s.dir + "/" + name;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw InputError("cannot open " + path + " (restart_type = 2)");
    out.assign(static_cast<size_t>(nv) * block, 0.0);
    std::vector<double> b(block);
    for (int l = 0; l < nv; ++l) {
      if (std::fread(b.data(), sizeof(double), block, f) != block) {
        std::fclose(f);
        throw InputError(name + " is too short");
      }
      for (size_t q = 0; q < block; ++q) out[q * nv + l] = b[q];
    }
    std::fclose(f);
  };
  const size_t n2 = static_cast<size_t>(s.nxmax) * s.nymax;
  if (s.enable_stat_time > 0) read_blocks("stat.bin", 70, n2, s.w_stat);
  if (s.enable_stat_3d > 0) read_blocks("stat3d.bin", 14, n2 * s.nzmax, s.w_stat_3d);
}

}  // namespace

// get_reynolds_cha (singleideal.F90:3052-3172), itransf = 0
double get_reynolds_cha(double retau, double rm, double trat, double s2tinf, double vtexp, bool visc_exp, double gam,
                        double rfac, int ny, const double* yn_in) {
  const int N = ny + 1;
  auto yn = [&](int j) { return yn_in[j - 1]; };
  double gm1h = 0.5 * (gam - 1.0);
  double tr = 1.0 + gm1h * rfac * (rm * rm);
  double tw = trat * tr;
  std::vector<double> yplus(N + 1, 0.0), uplus(N + 1, 0.0), ycplus(N + 1, 0.0), ucplus(N + 1, 0.0),
      yplusold(N + 1, 0.0), ucplusold(N + 1, 0.0), density(N + 1, 0.0), viscosity(N + 1, 0.0),
      temperature(N + 1, 0.0), uu(N + 1, 0.0);
  for (int j = 2; j <= N; ++j) ycplus[j] = (yn(j) - yn(1)) / (yn(N) - yn(1)) * retau;
  yplus = ycplus;
  yplusold = yplus;
  for (int outer = 0; outer < 100000; ++outer) {
    for (int j = 1; j <= N; ++j) uplus[j] = 0.0;
    for (int j = 2; j <= N; ++j) uplus[j] = velpiros_channel(yplus[j], retau);
    ucplus = uplus;
    for (int inner = 0; inner < 100000; ++inner) {
      ucplusold = ucplus;
      for (int j = 1; j <= N; ++j) {
        uu[j] = ucplus[j] / ucplus[ny];
        double fuu = uu[j];
        temperature[j] = tw + (tr - tw) * fuu + (1.0 - tr) * (uu[j] * uu[j]);
        density[j] = 1.0 / temperature[j];
        if (visc_exp)
          viscosity[j] = std::pow(temperature[j], vtexp);
        else
          viscosity[j] = std::pow(temperature[j], 1.5) * (1.0 + s2tinf) / (temperature[j] + s2tinf);
      }
      for (int j = 2; j <= N; ++j) {
        double du = uplus[j] - uplus[j - 1];
        double rhow_over_rho = density[1] / density[j];
        double rhow_over_rhojm = density[1] / density[j - 1];
        double rmu_over_rmuw = viscosity[j] / viscosity[1];
        double rmu_over_rmuwjm = viscosity[j - 1] / viscosity[1];
        double ucij = std::sqrt(rhow_over_rho) * std::sqrt(rmu_over_rmuw);
        double ucijm = std::sqrt(rhow_over_rhojm) * std::sqrt(rmu_over_rmuwjm);
        ucplus[j] = ucplus[j - 1] + 0.5 * (ucij + ucijm) * du;
      }
      double res = 0.0;
      for (int j = 1; j <= N; ++j) res = res + std::fabs(ucplus[j] - ucplusold[j]);
      res = res / N;
      if (res < TOL_ITER) break;
    }
    for (int j = 1; j <= N; ++j) yplus[j] = 0.0;
    for (int j = 2; j <= N; ++j) {
      double dy = ycplus[j] - ycplus[j - 1];
      double rhow_over_rho = density[1] / density[j];
      double rhow_over_rhojm = density[1] / density[j - 1];
      double rmu_over_rmuw = viscosity[j] / viscosity[1];
      double rmu_over_rmuwjm = viscosity[j - 1] / viscosity[1];
      double r3 = rmu_over_rmuw * rmu_over_rmuw * rmu_over_rmuw;
      double r3m = rmu_over_rmuwjm * rmu_over_rmuwjm * rmu_over_rmuwjm;
      double ycij = std::sqrt(rhow_over_rho) * std::sqrt(r3);
      ycij = 1.0 / ycij;
      double ycijm = std::sqrt(rhow_over_rhojm) * std::sqrt(r3m);
      ycijm = 1.0 / ycijm;
      yplus[j] = yplus[j - 1] + 0.5 * (ycij + ycijm) * dy;
    }
    // the reference overwrites (does not accumulate) res in this loop: only j = ny+1 counts
    double res = 0.0;
    for (int j = 1; j <= N; ++j) res = std::fabs(yplus[j] - yplusold[j]);
    res = res / N;
    if (res < TOL_ITER) break;
    yplusold = yplus;
  }
  double rhosum = 0.0, rhousum = 0.0, ysum = 0.0;
  for (int j = 1; j <= ny; ++j) {
    double dy = yn(j + 1) - yn(j);
    ysum = ysum + dy;
    rhosum = rhosum + 0.5 * (density[j] + density[j + 1]) * dy;
    rhousum = rhousum + 0.5 * (density[j] * ucplus[j] + density[j + 1] * ucplus[j + 1]) * dy;
  }
  rhosum = rhosum / ysum;
  rhousum = rhousum / ysum;
  double ubulk = rhousum / rhosum;
  return retau * ubulk * rhosum / density[1];
}

Setup setup_from_dir(const std::string& dir) {
  return setup_from_ini(IniFile::parse_file(dir + "/singleideal.ini"), dir);
}

Setup setup_from_ini(const IniFile& ini, const std::string& dir) {
  Setup s;
  s.ini = ini;
  s.dir = dir;
  const IniFile& c = s.ini;

  // equation initialize (singleideal.F90:284-864), Cartesian subset
  s.rand_type = c.get_int("numerics", "rand_type");
  s.l0 = c.get_double_or("ref_prop", "l0", 1.0);
  s.t0 = c.get_double_or("ref_prop", "t0", 1.0);
  s.rho0 = c.get_double_or("ref_prop", "rho0", 1.0);
  s.rgas0 = c.get_double_or("ref_prop", "rgas0", 1.0);
  int grid_dim = c.get_int_or("grid", "grid_dim", 1);
  if (grid_dim != 1) throw InputError("grid_dim = 2 (curvilinear) is not supported by the B200 backend");
  s.flow_init = c.get_int("flow", "flow_init");
  s.channel_case = (s.flow_init == 0 || s.flow_init == 4);
  s.aoa = c.get_double_or("flow", "aoa", 0.0) * pi() / 180.0;
  const char* bcn[6] = {"xmin", "xmax", "ymin", "ymax", "zmin", "zmax"};
  for (int l = 0; l < 6; ++l) s.bctags[l] = c.get_int("bc", bcn[l]);
  for (int d = 0; d < 3; ++d) {
    if (s.bctags[2 * d] == 0 || s.bctags[2 * d + 1] == 0) {
      s.bctags[2 * d] = s.bctags[2 * d + 1] = 0;
      s.periodic[d] = true;
    }
  }
  for (int l = 0; l < 6; ++l) s.bctags_nr[l] = c.get_int("bc", std::string(bcn[l]) + "_nr");
  s.restart_type = c.get_int("controls", "restart_type");
  if (s.restart_type < 0 || s.restart_type > 2) throw InputError("restart_type must be 0, 1 or 2");
  // [output] statistics keys (singleideal.F90:542-551, 818)
  s.dtstat = c.get_double_or("output", "dtstat", -1.0);
  s.enable_stat_time = c.get_int_or("output", "enable_stat_time", 1);
  s.enable_stat_3d = c.get_int_or("output", "enable_stat_3d", 0);
  s.grid_type = c.get_int("grid", "grid_type");
  bool rebuild_ghost = (s.grid_type == GRID_FROMFILE);
  if (s.restart_type > 0) s.grid_type = GRID_FROMFILE;
  s.nxmax = c.get_int("grid", "nxmax");
  s.nymax = c.get_int("grid", "nymax");
  s.nzmax = c.get_int("grid", "nzmax");
  s.ng = c.get_int("grid", "ng");
  s.domain_size[0] = c.get_double("grid", "domain_size_x");
  s.domain_size[1] = c.get_double("grid", "domain_size_y");
  s.domain_size[2] = c.get_double("grid", "domain_size_z");
  s.metrics_order = c.get_int("grid", "metrics_order");
  int ystag = c.get_int_or("grid", "ystag", 0);
  s.is_y_staggered = (ystag > 0) || s.channel_case;
  s.ep_order = c.get_int("numerics", "ep_order");
  if (s.ep_order != s.metrics_order) throw InputError("ep_order must be equal to metrics_order");
  if (s.nzmax == 1) throw InputError("2D runs (nzmax = 1) are not supported by the B200 backend");
  s.ndim = 3;
  if (s.ng < 3) throw InputError("the B200 backend needs ng >= 3");

  const bool synthetic = c.has_section("synthetic");

  // grid%initialize (code/src/grid.F90:192-308)
  s.xg.resize(1 - s.ng, s.nxmax + s.ng + 1);
  s.yg.resize(1 - s.ng, s.nymax + s.ng);
  s.zg.resize(1 - s.ng, s.nzmax + s.ng);
  s.yn.resize(1, s.nymax + 1 + s.ng);
  if (s.grid_type == GRID_FROMFILE && !synthetic) {
    read_grid(s, rebuild_ghost);
  } else {
    uniform_grid(s.xg, s.nxmax, s.ng, s.domain_size[0], s.periodic[0], 1);
    OffsetArray zt;
    uniform_grid(zt, s.nzmax, s.ng, s.domain_size[2], s.periodic[2], 0);
    s.zg = zt;
    if (synthetic && c.has_key("synthetic", "y_stretch")) {
      generate_grid_tanh(s, c.get_double("synthetic", "y_stretch"));
    } else if (s.grid_type == GRID_UNIFORM) {
      OffsetArray yt;
      uniform_grid(yt, s.nymax, s.ng, s.domain_size[1], s.periodic[1], 0);
      for (int j = 1 - s.ng; j <= s.nymax + s.ng; ++j) s.yg(j) = yt(j);
    } else if (s.grid_type == GRID_CHA) {
      generate_grid_cha(s, c.get_double("grid", "jbgrid"), c.get_double("grid", "dyptarget"),
                        static_cast<int>(std::lround(c.get_double("grid", "ysmoosteps"))),
                        c.get_double("flow", "Reynolds"));
    } else if (s.grid_type == GRID_BL || s.grid_type == GRID_SBLI) {
      generate_grid_bl(s, c.get_double("grid", "jbgrid"), c.get_double("grid", "dyptarget"),
                       static_cast<int>(std::lround(c.get_double("grid", "nywr"))), c.get_double("grid", "lywr"),
                       c.get_double("flow", "Reynolds"),
                       static_cast<int>(std::lround(c.get_double("grid", "ysmoosteps"))), s.grid_type == GRID_SBLI);
    } else {
      throw InputError("grid_type " + std::to_string(s.grid_type) + " is not supported by the B200 backend");
    }
  }
  for (auto& v : s.xg.data) v *= s.l0;
  for (auto& v : s.yg.data) v *= s.l0;
  for (auto& v : s.zg.data) v *= s.l0;
  for (auto& v : s.yn.data) v *= s.l0;
  for (auto& v : s.domain_size) v *= s.l0;
  {
    double c1[4], c2[5];
    get_deriv_coeffs(c1, c2, s.metrics_order, s.metrics_order);
    const int mm = s.metrics_order / 2;
    metrics_1d(s.xg, s.nxmax, mm, c1, c2, s.dxg, s.d2xg);
    metrics_1d(s.yg, s.nymax, mm, c1, c2, s.dyg, s.d2yg);
    metrics_1d(s.zg, s.nzmax, mm, c1, c2, s.dzg, s.d2zg);
  }

  // fluid and flow
  set_fluid_prop(s);
  double re_bulk_target = synthetic ? c.get_double_or("synthetic", "reynolds_bulk", -1.0) : -1.0;
  set_flow_params(s, re_bulk_target);

  s.nkeep = c.get_int_or("numerics", "nkeep", 0);
  s.weno_scheme = c.get_int("numerics", "weno_scheme");
  if (s.weno_scheme < 1 || s.weno_scheme > 4) throw InputError("weno_scheme must be 1, 2, 3 or 4");
  // the face stencils reach max(ep_order/2, weno_scheme) points beyond a face into the ghosts
  if (s.ng < std::max(s.ep_order / 2, s.weno_scheme))
    throw InputError("ng must be at least max(ep_order/2, weno_scheme) = " +
                     std::to_string(std::max(s.ep_order / 2, s.weno_scheme)));
  s.weno_version = c.get_int("numerics", "weno_version");
  if (s.weno_scheme != 3 && s.weno_version == 1) throw InputError("weno_version 1 supported only for weno_scheme = 3");
  s.flux_splitting = c.get_int_or("numerics", "flux_splitting", 0);
  if (s.flux_splitting != 0 && s.flux_splitting != 1) throw InputError("flux_splitting must be 0 or 1");
  s.visc_order = c.get_int("numerics", "visc_order");
  if (s.visc_order != s.ep_order) throw InputError("viscous order must be equal to ep_order");
  s.conservative_viscous = c.get_int("numerics", "conservative_viscous");
  if (s.conservative_viscous != 0 && s.conservative_viscous != 1)
    throw InputError("conservative_viscous must be 0 or 1");
  for (int i = 0; i < 4; ++i) get_deriv_coeffs(s.coeff_deriv1[i], s.coeff_deriv2[i], 2 * (i + 1), 2 * (i + 1));
  s.sensor_threshold = c.get_double("numerics", "sensor_threshold");
  s.x_split = c.get_int("mpi", "x_split");
  s.y_split = c.get_int("mpi", "y_split");
  s.z_split = c.get_int("mpi", "z_split");
  if (s.nxmax % s.x_split || s.nzmax % s.z_split || s.y_split != 1)
    throw InputError("inconsistent mpi split (nxmax/nzmax multiples of x/z split, y_split = 1)");

  // bc_preproc (singleideal.F90:4703-4750)
  s.eul_imin = 1; s.eul_imax = s.nxmax; s.eul_jmin = 1; s.eul_jmax = s.nymax; s.eul_kmin = 1; s.eul_kmax = s.nzmax;
  for (int l = 0; l < 6; ++l) {
    if (s.bctags[l] == 6 && s.is_y_staggered) {
      s.force_zero_flux[l] = 1;
      s.bctags_nr[l] = 0;
    }
    int offset = (s.bctags_nr[l] != 0) ? 1 : 0;
    switch (l) {
      case 0: s.eul_imin += offset; break;
      case 1: s.eul_imax -= offset; break;
      case 2: s.eul_jmin += offset; break;
      case 3: s.eul_jmax -= offset; break;
      case 4: s.eul_kmin += offset; break;
      case 5: s.eul_kmax -= offset; break;
    }
  }
  for (int l = 0; l < 6; ++l) {
    const int t = s.bctags[l];
    if (t != 0 && t != 2 && t != 6 && t != 10 && !(t == 7 && l == 3))
      throw InputError("boundary tag " + std::to_string(t) + " is not supported by the B200 backend yet");
    const int nr = s.bctags_nr[l];
    if (nr != 0 && nr != 1 && nr != 2 && nr != 3 && nr != 6)
      throw InputError("non-reflecting type " + std::to_string(nr) + " is not supported");
    if (nr != 0 && l >= 4) throw InputError("non-reflecting treatment is supported on x and y boundaries");
  }
  if (s.bctags[0] == 6 || s.bctags[1] == 6 || s.bctags[4] == 6 || s.bctags[5] == 6)
    throw InputError("viscous walls are supported on the y boundaries only");
  for (int l = 1; l < 6; ++l)
    if (s.bctags[l] == 10) throw InputError("recycling inflow (tag 10) is supported at xmin only");

  // correct_bc_order (singleideal.F90:946-993)
  const int n3[3] = {s.nxmax, s.nymax, s.nzmax};
  for (int d = 0; d < 3; ++d) s.ep_ord[d].assign(n3[d] + 1, 0);
  s.correct_bound_ord = c.get_int_or("bc", "correct_bound_ord", 0);
  if (s.correct_bound_ord > 0) {
    int st = std::max(s.ep_order / 2, s.weno_scheme);
    for (int d = 0; d < 3; ++d) {
      if (s.bctags[2 * d] == 0 && s.bctags[2 * d + 1] == 0) continue;
      auto& e = s.ep_ord[d];
      const int n = n3[d];
      e[0] = -st + 1;
      for (int i = 1; i <= st - 1; ++i) e[i] = -st + i;
      e[n] = -st + 1;
      for (int i = 1; i <= st - 1; ++i) e[n - i] = -st + i;
    }
  }

  // runge_kutta_initialize (singleideal.F90:4773-4795)
  s.rk_type = c.get_int("numerics", "rk_type");
  if (s.rk_type != 1) throw InputError("only rk_type = 1 (Wray RK3) is supported");
  s.nrk = 3;
  s.rhork[0] = 0.0; s.rhork[1] = -17.0 / 60.0; s.rhork[2] = -5.0 / 12.0;
  s.gamrk[0] = 8.0 / 15.0; s.gamrk[1] = 5.0 / 12.0; s.gamrk[2] = 3.0 / 4.0;
  s.cfl = c.get_double("controls", "cfl");
  s.num_iter = c.get_int("controls", "num_iter");
  s.print_control = c.get_int("output", "print_control");
  s.iter_dt_recompute = c.get_int("controls", "iter_dt_recompute");

  // local grid of the single block (field.F90 set_local_grid)
  const int ng = s.ng;
  s.x.resize(s.nxmax + 2 * ng);
  s.y.resize(s.nymax + 2 * ng);
  s.z.resize(s.nzmax + 2 * ng);
  for (int i = 1 - ng; i <= s.nxmax + ng; ++i) s.x[i + ng - 1] = s.xg(i);
  for (int j = 1 - ng; j <= s.nymax + ng; ++j) s.y[j + ng - 1] = s.yg(j);
  for (int k = 1 - ng; k <= s.nzmax + ng; ++k) s.z[k + ng - 1] = s.zg(k);
  s.ynl.resize(s.nymax + 1);
  for (int j = 1; j <= s.nymax + 1; ++j) s.ynl[j - 1] = s.yn(j);
  auto loc = [](const OffsetArray& d, const OffsetArray& d2, int n, std::vector<double>& a, std::vector<double>& as,
                std::vector<double>& a2) {
    a.resize(n); as.resize(n); a2.resize(n);
    for (int i = 1; i <= n; ++i) {
      a[i - 1] = 1.0 / d(i);
      as[i - 1] = a[i - 1] * a[i - 1];
      a2[i - 1] = -d2(i) * as[i - 1];
    }
  };
  loc(s.dxg, s.d2xg, s.nxmax, s.dcsidx, s.dcsidxs, s.dcsidx2);
  loc(s.dyg, s.d2yg, s.nymax, s.detady, s.detadys, s.detady2);
  loc(s.dzg, s.d2zg, s.nzmax, s.dzitdz, s.dzitdzs, s.dzitdz2);

  // initial_conditions (singleideal.F90:3018-3051): winf everywhere, then the case initialiser
  s.w.assign(s.ncells_ghost() * 5, 0.0);
  for (int m = 0; m < 5; ++m) {
    const size_t n = s.ncells_ghost();
    for (size_t q = 0; q < n; ++q) s.w[m * n + q] = s.winf[m];
  }
  // volchan (init_channel, singleideal.F90:4364-4366)
  s.volchan = s.yn(s.nymax + 1) - s.yn(1);
  s.volchan = s.volchan * s.nxmax;
  s.volchan = s.volchan * s.nzmax;
  if (synthetic) {
    std::string kind = "channel_poiseuille";
    if (c.has_key("synthetic", "kind")) {
      std::istringstream is(c.raw("synthetic", "kind"));
      is >> kind;
    }
    if (kind == "channel_poiseuille") {
      if (s.flow_init != 0) throw InputError("the synthetic channel field needs flow_init = 0");
      init_channel_synthetic(s, c.get_double_or("synthetic", "amp", 0.1), c.get_int_or("synthetic", "seed", 1));
    } else if (kind == "bl_powerlaw") {
      if (s.flow_init != 1) throw InputError("the synthetic boundary-layer field needs flow_init = 1");
      init_bl_synthetic(s, c.get_double_or("synthetic", "amp", 0.05));
    } else {
      throw InputError("unknown synthetic initial field " + kind);
    }
    // a synthetic case restarted from its own rst.bin: the set-up above fixes the parameters,
    // grid and inflow data, the field and the clock come from the restart files
    if (s.restart_type == 1) {
      read_rst(s);
      read_field_info(s);
    }
  } else {
    if (s.flow_init == 1) init_bl(s);
    else init_channel(s);
    if (s.restart_type == 1) {
      read_rst(s);
      read_field_info(s);
    }
  }
  if (s.restart_type == 2) {
    // restart with statistics: the field and clock as for restart_type = 1, then the averages
    read_rst(s);
    read_field_info(s);
    read_stats_files(s);
  }
  s.recyc = s.bctags[0] == 10;
  if (s.recyc) {
    if (s.flow_init != 1 || s.wmean.empty()) throw InputError("recycling inflow needs the boundary-layer initialisation");
    recyc_prepare(s);
  }
  return s;
}

void Setup::fill_params(streams_b200_params* p, int precision) const {
  *p = streams_b200_params{};
  p->nx = nxmax; p->ny = nymax; p->nz = nzmax; p->ng = ng;
  p->ep_order = ep_order; p->nkeep = nkeep; p->weno_scheme = weno_scheme; p->weno_version = weno_version;
  p->flux_splitting = flux_splitting; p->conservative_viscous = conservative_viscous;
  p->sensor_threshold = sensor_threshold;
  for (int l = 0; l < 6; ++l) {
    p->bctags[l] = bctags[l];
    p->force_zero_flux[l] = force_zero_flux[l];
  }
  p->eul_imin = eul_imin; p->eul_imax = eul_imax; p->eul_jmin = eul_jmin;
  p->eul_jmax = eul_jmax; p->eul_kmin = eul_kmin; p->eul_kmax = eul_kmax;
  p->is_y_staggered = is_y_staggered ? 1 : 0;
  p->visc_model = visc_model; p->calorically_perfect = calorically_perfect;
  p->mu0 = mu0; p->t0 = t0; p->rgas0 = rgas0; p->rho0 = rho0; p->u0 = u0; p->l0 = l0;
  p->sutherland_s = sutherland_s; p->t_ref_dim = t_ref_dim; p->powerlaw_vtexp = powerlaw_vtexp;
  p->prandtl = prandtl;
  p->cp0 = cp_coeff[static_cast<size_t>(-indx_cp_l)]; p->cv0 = cv_coeff[static_cast<size_t>(-indx_cp_l)];
  p->cp_last = cp_coeff.back(); p->cv_last = cv_coeff.back();
  p->indx_cp_l = indx_cp_l; p->indx_cp_r = indx_cp_r;
  for (size_t q = 0; q < cp_coeff.size() && q < STREAMS_B200_MAX_CP; ++q) {
    p->cp_coeff[q] = cp_coeff[q];
    p->cv_coeff[q] = cv_coeff[q];
  }
  p->channel_case = channel_case ? 1 : 0;
  p->theta_wall = theta_wall; p->t_wall = t_wall; p->t_bulk_target = t_bulk_target; p->volchan = volchan;
  p->nrk = nrk;
  for (int l = 0; l < 3; ++l) {
    p->rhork[l] = rhork[l];
    p->gamrk[l] = gamrk[l];
  }
  p->cfl = cfl;
  p->precision = precision;
  for (int l = 0; l < 6; ++l) p->bctags_nr[l] = bctags_nr[l];
  for (int m = 0; m < 5; ++m) p->winf[m] = winf[m];
  p->p0 = p0;
  p->recyc = recyc ? 1 : 0;
  p->i_recyc = i_recyc;
  p->jbl_inflow = jbl_inflow;
  p->betarecyc = betarecyc;
  p->rng_seed = rng_seed;
  p->rng_draws = rng_draws;
  p->xshock_imp = xshock_imp; p->shock_angle = shock_angle; p->tanhfacs = tanhfacs;
  for (int m = 0; m < 5; ++m) p->winf_past_shock[m] = winf_past_shock[m];
}

void Setup::fill_grid(streams_b200_grid* g) const {
  g->x = x.data(); g->y = y.data(); g->z = z.data(); g->yn = ynl.data();
  g->dcsidx = dcsidx.data(); g->detady = detady.data(); g->dzitdz = dzitdz.data();
  g->dcsidxs = dcsidxs.data(); g->detadys = detadys.data(); g->dzitdzs = dzitdzs.data();
  g->coeff_deriv1 = &coeff_deriv1[0][0];
  g->ep_ord_x = ep_ord[0].data(); g->ep_ord_y = ep_ord[1].data(); g->ep_ord_z = ep_ord[2].data();
  g->dcsidx2 = dcsidx2.data(); g->detady2 = detady2.data(); g->dzitdz2 = dzitdz2.data();
  g->coeff_deriv2 = &coeff_deriv2[0][0];
  if (recyc) {
    g->wmean_inflow = wmean_inflow.data();
    g->yplus_inflow = yplus_inflow.data(); g->eta_inflow = eta_inflow.data();
    g->yplus_recyc = yplus_recyc.data(); g->eta_recyc = eta_recyc.data();
    g->weta_inflow = weta_inflow.data();
    g->map_j_inn = map_j_inn.data(); g->map_j_out = map_j_out.data();
  }
}

void write_restart_inputs(const Setup& s, const std::string& dir) {
  write_restart_state(s, s.w.data(), s.icyc0, s.time0, dir);
}

namespace {

void write_rst(const Setup& s, const double* w, const std::string& dir) {
  FILE* f = std::fopen((dir + "/rst.bin").c_str(), "wb");
  if (!f) throw InputError("cannot write rst.bin");
  std::vector<double> plane(static_cast<size_t>(s.nxmax));
  for (int m = 0; m < 5; ++m)
    for (int k = 1; k <= s.nzmax; ++k)
      for (int j = 1; j <= s.nymax; ++j) {
        for (int i = 1; i <= s.nxmax; ++i) plane[i - 1] = w[s.widx(i, j, k, m)];
        std::fwrite(plane.data(), sizeof(double), plane.size(), f);
      }
  std::fclose(f);
}

// field_info0.dat with every key that read_field_info (singleideal.F90:2546-2590) reads
// unconditionally; the output clocks other than the statistics' start afresh
void write_field_info(const std::string& dir, int icyc, double time, const StatsOut* st) {
  FILE* fi = std::fopen((dir + "/field_info0.dat").c_str(), "w");
  if (!fi) throw InputError("cannot write field_info0.dat");
  std::fprintf(fi,
               "[field_info]\nicyc0 = %d\ntime0 = %.17e\nitav = %d\nitslice_p3d = 0\ntime_from_last_rst = 0.0\n"
               "time_from_last_write = 0.0\ntime_from_last_stat = %.17e\ntime_from_last_slice = 0.0\n"
               "time_from_last_probe = 0.0\nistore = 1\n",
               icyc, time, st ? st->itav : 0, st ? st->time_from_last_stat : 0.0);
  std::fclose(fi);
}

// write_stats / write_stats_3d (singleideal.F90:1786-1834, 1922-1965): one block per statistic
void write_stats_files(const Setup& s, const std::string& dir, const StatsOut& st) {
  auto write_blocks = [&](const std::string& name, const double* a, int nv, size_t block) {
    FILE* f = std::fopen((dir + "/" + name).c_str(), "wb");
    if (!f) throw InputError("cannot write " + name);
    std::vector<double> b(block);
    for (int l = 0; l < nv; ++l) {
      for (size_t q = 0; q < block; ++q) b[q] = a[q * nv + l];
      std::fwrite(b.data(), sizeof(double), block, f);
    }
    std::fclose(f);
  };
  const size_t n2 = static_cast<size_t>(s.nxmax) * s.nymax;
  if (st.w_stat) write_blocks("stat.bin", st.w_stat, 70, n2);
  if (st.w_stat_3d) write_blocks("stat3d.bin", st.w_stat_3d, 14, n2 * s.nzmax);
}

}  // namespace

// The files of a restart from a conserved field w of the case: grid files, rst.bin (per
// variable, Fortran order, interior points: the single-block layout of the reference's MPI-IO
// file, code/src/field.F90:1853-1966), field_info0.dat, the statistics files when given, and
// singleideal.ini = the case's input with restart_type = 1, or 2 with statistics.
void write_restart_state(const Setup& s, const double* w, int icyc, double time, const std::string& dir,
                         const StatsOut* st) {
  auto col = [&](const std::string& name, const OffsetArray& a, int lo, int hi) {
    FILE* f = std::fopen((dir + "/" + name).c_str(), "w");
    if (!f) throw InputError("cannot write " + dir + "/" + name);
    for (int i = lo; i <= hi; ++i) std::fprintf(f, "%.17e\n", a(i));
    std::fclose(f);
  };
  col("x.dat", s.xg, 1 - s.ng, s.nxmax + s.ng + 1);
  col("y.dat", s.yg, 1 - s.ng, s.nymax + s.ng);
  col("z.dat", s.zg, 1 - s.ng, s.nzmax + s.ng);
  col("yn.dat", s.yn, 1, s.nymax + 1);
  write_run_output(s, w, icyc, time, dir, st);
  IniFile ini = s.ini;
  ini.set("controls", "restart_type", st ? "2" : "1");
  if (st) {
    ini.set("output", "enable_stat_time", st->w_stat ? "1" : "0");
    ini.set("output", "enable_stat_3d", st->w_stat_3d ? "1" : "0");
  }
  FILE* fin = std::fopen((dir + "/singleideal.ini").c_str(), "w");
  if (!fin) throw InputError("cannot write singleideal.ini");
  const std::string text = ini.to_text();
  std::fwrite(text.data(), 1, text.size(), fin);
  std::fclose(fin);
}

// flow_params.dat as set_flow_params writes it (singleideal.F90:2818-2852): the reference values
// that post-processing (tools/postpro) reads beside stat.bin
void write_flow_params(const Setup& s, const std::string& dir) {
  FILE* f = std::fopen((dir + "/flow_params.dat").c_str(), "w");
  if (!f) throw InputError("cannot write flow_params.dat");
  const double cp0 = s.cp_coeff[static_cast<size_t>(-s.indx_cp_l)];
  const double cv0 = s.cv_coeff[static_cast<size_t>(-s.indx_cp_l)];
  const double k0 = s.mu0 * cp0 / s.prandtl;
  std::fprintf(f, "[flow_params]\n");
  const std::pair<const char*, double> kv[] = {
      {"u0", s.u0}, {"p0", s.p0}, {"rho0", s.rho0}, {"t0", s.t0}, {"c0", s.c0}, {"l0", s.l0},
      {"cp0", cp0}, {"cv0", cv0}, {"mu0", s.mu0}, {"k0", k0}, {"gam", s.gam}, {"T_wall", s.t_wall},
      {"theta_wall", s.theta_wall}, {"rfac", s.rfac}, {"powerlaw_vtexp", s.powerlaw_vtexp},
      {"T_ref_dim", s.t_ref_dim}, {"Reynolds", s.reynolds}, {"Mach", s.mach}, {"Prandtl", s.prandtl}};
  for (const auto& p : kv) std::fprintf(f, "%s = %.17e\n", p.first, p.second);
  std::fclose(f);
}

void write_run_output(const Setup& s, const double* w, int icyc, double time, const std::string& dir,
                      const StatsOut* st) {
  write_flow_params(s, dir);
  write_rst(s, w, dir);
  if (st) write_stats_files(s, dir, *st);
  write_field_info(dir, icyc, time, st);
}

}  // namespace streams_b200
