// CPU oracle: restatement of the STREAmS-2 CPU backend time advance.  See oracle.hpp.
// All line references are to code/src/singleideal/kernels_cpu.F90 unless stated otherwise.
#include "oracle.hpp"

#include <algorithm>
#include <cmath>
#include <limits>

#include "flops.hpp"
#include "par_for.hpp"

namespace streams_oracle {

namespace {

// wenorec_1d (kernels_cpu.F90:2526-2724).  vp, vm: [5][8] with Fortran index l = 1..8 at [m][l-1].
template <class T>
void wenorec_1d(const T vp[5][8], const T vm[5][8], T vhat[5], int iweno, int ord, int version, double rho0,
                double u0, bool rusanov = false) {
  using std::fabs;
  auto VP = [&](int m, int l) { return vp[m][l - 1]; };
  auto VM = [&](int m, int l) { return vm[m][l - 1]; };
  double u0_2 = u0 * u0;
  double rho0_2u0_2 = rho0 * rho0 * u0_2;
  double rho0_2u0_4 = rho0_2u0_2 * u0_2;
  double betascale[5];
  betascale[0] = 1.0 / rho0_2u0_2;
  betascale[1] = betascale[0];
  betascale[2] = 1.0 / rho0_2u0_4;
  betascale[3] = betascale[2];
  betascale[4] = betascale[0];
  if (rusanov) {
    // wenorec_1d_rusanov (kernels_cpu.F90:2325-2523): scales of the conserved variables
    betascale[0] = 1.0 / rho0_2u0_2;
    betascale[1] = 1.0 / rho0_2u0_4;
    betascale[2] = betascale[1];
    betascale[3] = betascale[1];
    betascale[4] = betascale[1] / u0_2;
  }
  const int i = iweno;
  if (ord == 1) {
    for (int m = 0; m < 5; ++m) vhat[m] = VP(m, i) + VM(m, i + 1);
  } else if (ord == 2) {
    double dwe[2] = {1.0 / 3.0, 2.0 / 3.0};
    for (int m = 0; m < 5; ++m) {
      T bp[2], bm[2];
      bp[0] = (VP(m, i) - VP(m, i - 1)) * (VP(m, i) - VP(m, i - 1));
      bp[1] = (VP(m, i + 1) - VP(m, i)) * (VP(m, i + 1) - VP(m, i));
      bp[1] = betascale[m] * bp[1];
      bp[0] = betascale[m] * bp[0];
      bm[0] = (VM(m, i + 2) - VM(m, i + 1)) * (VM(m, i + 2) - VM(m, i + 1));
      bm[1] = (VM(m, i + 1) - VM(m, i)) * (VM(m, i + 1) - VM(m, i));
      bm[1] = betascale[m] * bm[1];
      bm[0] = betascale[m] * bm[0];
      T sump = 0.0, summ = 0.0;
      for (int l = 0; l < 2; ++l) {
        T tp = 0.000001 + bp[l], tm = 0.000001 + bm[l];
        bp[l] = dwe[l] / (tp * tp);
        bm[l] = dwe[l] / (tm * tm);
        sump = sump + bp[l];
        summ = summ + bm[l];
      }
      for (int l = 0; l < 2; ++l) {
        bp[l] = bp[l] / sump;
        bm[l] = bm[l] / summ;
      }
      T vminus = bp[0] * (-VP(m, i - 1) + 3 * VP(m, i)) + bp[1] * (VP(m, i) + VP(m, i + 1));
      T vplus = bm[0] * (-VM(m, i + 2) + 3 * VM(m, i + 1)) + bm[1] * (VM(m, i) + VM(m, i + 1));
      vhat[m] = 0.5 * (vminus + vplus);
    }
  } else if (ord == 3) {
    const double dwe[3] = {1.0 / 10.0, 6.0 / 10.0, 3.0 / 10.0};
    const double d0 = 13.0 / 12.0, d1 = 1.0 / 4.0;
    const double c0 = 1.0 / 3.0, c1 = 5.0 / 6.0, c2 = -1.0 / 6.0, c3 = -7.0 / 6.0, c4 = 11.0 / 6.0;
    auto sq = [](T a) { return a * a; };
    for (int m = 0; m < 5; ++m) {
      T bp[3], bm[3];
      bp[2] = d0 * sq(VP(m, i) - 2.0 * VP(m, i + 1) + VP(m, i + 2)) +
              d1 * sq(3.0 * VP(m, i) - 4.0 * VP(m, i + 1) + VP(m, i + 2));
      bp[1] = d0 * sq(VP(m, i - 1) - 2.0 * VP(m, i) + VP(m, i + 1)) + d1 * sq(VP(m, i - 1) - VP(m, i + 1));
      bp[0] = d0 * sq(VP(m, i) - 2.0 * VP(m, i - 1) + VP(m, i - 2)) +
              d1 * sq(3.0 * VP(m, i) - 4.0 * VP(m, i - 1) + VP(m, i - 2));
      bp[2] = betascale[m] * bp[2];
      bp[1] = betascale[m] * bp[1];
      bp[0] = betascale[m] * bp[0];
      bm[2] = d0 * sq(VM(m, i + 1) - 2.0 * VM(m, i) + VM(m, i - 1)) +
              d1 * sq(3.0 * VM(m, i + 1) - 4.0 * VM(m, i) + VM(m, i - 1));
      bm[1] = d0 * sq(VM(m, i + 2) - 2.0 * VM(m, i + 1) + VM(m, i)) + d1 * sq(VM(m, i + 2) - VM(m, i));
      bm[0] = d0 * sq(VM(m, i + 1) - 2.0 * VM(m, i + 2) + VM(m, i + 3)) +
              d1 * sq(3.0 * VM(m, i + 1) - 4.0 * VM(m, i + 2) + VM(m, i + 3));
      bm[2] = betascale[m] * bm[2];
      bm[1] = betascale[m] * bm[1];
      bm[0] = betascale[m] * bm[0];
      if (version == 0) {
        T sump = 0.0, summ = 0.0;
        for (int l = 0; l < 3; ++l) {
          T tp = 0.000001 + bp[l], tm = 0.000001 + bm[l];
          bp[l] = dwe[l] / (tp * tp);
          bm[l] = dwe[l] / (tm * tm);
          sump = sump + bp[l];
          summ = summ + bm[l];
        }
        for (int l = 0; l < 3; ++l) {
          bp[l] = bp[l] / sump;
          bm[l] = bm[l] / summ;
        }
      } else {
        // eps40 is a default-kind (single precision) literal in the reference
        const double eps40 = static_cast<double>(1.e-35f);
        T tau5p = fabs(bp[0] - bp[2]) + eps40;
        T tau5m = fabs(bm[0] - bm[2]) + eps40;
        for (int l = 0; l < 3; ++l) {
          bp[l] = (bp[l] + eps40) / (bp[l] + tau5p);
          bm[l] = (bm[l] + eps40) / (bm[l] + tau5m);
        }
        T sump = 0.0, summ = 0.0;
        for (int l = 0; l < 3; ++l) {
          bp[l] = dwe[l] / bp[l];
          bm[l] = dwe[l] / bm[l];
          sump = sump + bp[l];
          summ = summ + bm[l];
        }
        for (int l = 0; l < 3; ++l) {
          bp[l] = bp[l] / sump;
          bm[l] = bm[l] / summ;
        }
      }
      T vminus = bp[2] * (c0 * VP(m, i) + c1 * VP(m, i + 1) + c2 * VP(m, i + 2)) +
                      bp[1] * (c2 * VP(m, i - 1) + c1 * VP(m, i) + c0 * VP(m, i + 1)) +
                      bp[0] * (c0 * VP(m, i - 2) + c3 * VP(m, i - 1) + c4 * VP(m, i));
      T vplus = bm[2] * (c0 * VM(m, i + 1) + c1 * VM(m, i) + c2 * VM(m, i - 1)) +
                     bm[1] * (c2 * VM(m, i + 2) + c1 * VM(m, i + 1) + c0 * VM(m, i)) +
                     bm[0] * (c0 * VM(m, i + 3) + c3 * VM(m, i + 2) + c4 * VM(m, i + 1));
      vhat[m] = vminus + vplus;
    }
  } else if (ord == 4) {
    const double dwe[4] = {1.0 / 35.0, 12.0 / 35.0, 18.0 / 35.0, 4.0 / 35.0};
    const double d1 = 1.0 / 36.0, d2 = 13.0 / 12.0, d3 = 781.0 / 720.0;
    auto sq = [](T a) { return a * a; };
    for (int m = 0; m < 5; ++m) {
      T bp[4], bm[4];
      bp[3] = d1 * sq(-11 * VP(m, i) + 18 * VP(m, i + 1) - 9 * VP(m, i + 2) + 2 * VP(m, i + 3)) +
              d2 * sq(2 * VP(m, i) - 5 * VP(m, i + 1) + 4 * VP(m, i + 2) - VP(m, i + 3)) +
              d3 * sq(-VP(m, i) + 3 * VP(m, i + 1) - 3 * VP(m, i + 2) + VP(m, i + 3));
      bp[2] = d1 * sq(-2 * VP(m, i - 1) - 3 * VP(m, i) + 6 * VP(m, i + 1) - VP(m, i + 2)) +
              d2 * sq(VP(m, i - 1) - 2 * VP(m, i) + VP(m, i + 1)) +
              d3 * sq(-VP(m, i - 1) + 3 * VP(m, i) - 3 * VP(m, i + 1) + VP(m, i + 2));
      bp[1] = d1 * sq(VP(m, i - 2) - 6 * VP(m, i - 1) + 3 * VP(m, i) + 2 * VP(m, i + 1)) +
              d2 * sq(VP(m, i - 1) - 2 * VP(m, i) + VP(m, i + 1)) +
              d3 * sq(-VP(m, i - 2) + 3 * VP(m, i - 1) - 3 * VP(m, i) + VP(m, i + 1));
      bp[0] = d1 * sq(-2 * VP(m, i - 3) + 9 * VP(m, i - 2) - 18 * VP(m, i - 1) + 11 * VP(m, i)) +
              d2 * sq(-VP(m, i - 3) + 4 * VP(m, i - 2) - 5 * VP(m, i - 1) + 2 * VP(m, i)) +
              d3 * sq(-VP(m, i - 3) + 3 * VP(m, i - 2) - 3 * VP(m, i - 1) + VP(m, i));
      for (int l = 3; l >= 0; --l) bp[l] = betascale[m] * bp[l];
      bm[3] = d1 * sq(-11 * VM(m, i + 1) + 18 * VM(m, i) - 9 * VM(m, i - 1) + 2 * VM(m, i - 2)) +
              d2 * sq(2 * VM(m, i + 1) - 5 * VM(m, i) + 4 * VM(m, i - 1) - VM(m, i - 2)) +
              d3 * sq(-VM(m, i + 1) + 3 * VM(m, i) - 3 * VM(m, i - 1) + VM(m, i - 2));
      bm[2] = d1 * sq(-2 * VM(m, i + 2) - 3 * VM(m, i + 1) + 6 * VM(m, i) - VM(m, i - 1)) +
              d2 * sq(VM(m, i + 2) - 2 * VM(m, i + 1) + VM(m, i)) +
              d3 * sq(-VM(m, i + 2) + 3 * VM(m, i + 1) - 3 * VM(m, i) + VM(m, i - 1));
      bm[1] = d1 * sq(VM(m, i + 3) - 6 * VM(m, i + 2) + 3 * VM(m, i + 1) + 2 * VM(m, i)) +
              d2 * sq(VM(m, i + 2) - 2 * VM(m, i + 1) + VM(m, i)) +
              d3 * sq(-VM(m, i + 3) + 3 * VM(m, i + 2) - 3 * VM(m, i + 1) + VM(m, i));
      bm[0] = d1 * sq(-2 * VM(m, i + 4) + 9 * VM(m, i + 3) - 18 * VM(m, i + 2) + 11 * VM(m, i + 1)) +
              d2 * sq(-VM(m, i + 4) + 4 * VM(m, i + 3) - 5 * VM(m, i + 2) + 2 * VM(m, i + 1)) +
              d3 * sq(-VM(m, i + 4) + 3 * VM(m, i + 3) - 3 * VM(m, i + 2) + VM(m, i + 1));
      for (int l = 3; l >= 0; --l) bm[l] = betascale[m] * bm[l];
      T sump = 0.0, summ = 0.0;
      for (int l = 0; l < 4; ++l) {
        T tp = 0.000001 + bp[l], tm = 0.000001 + bm[l];
        bp[l] = dwe[l] / (tp * tp);
        bm[l] = dwe[l] / (tm * tm);
        sump = sump + bp[l];
        summ = summ + bm[l];
      }
      for (int l = 0; l < 4; ++l) {
        bp[l] = bp[l] / sump;
        bm[l] = bm[l] / summ;
      }
      T vminus = bp[3] * (6 * VP(m, i) + 26 * VP(m, i + 1) - 10 * VP(m, i + 2) + 2 * VP(m, i + 3)) +
                      bp[2] * (-2 * VP(m, i - 1) + 14 * VP(m, i) + 14 * VP(m, i + 1) - 2 * VP(m, i + 2)) +
                      bp[1] * (2 * VP(m, i - 2) - 10 * VP(m, i - 1) + 26 * VP(m, i) + 6 * VP(m, i + 1)) +
                      bp[0] * (-6 * VP(m, i - 3) + 26 * VP(m, i - 2) - 46 * VP(m, i - 1) + 50 * VP(m, i));
      T vplus = bm[3] * (6 * VM(m, i + 1) + 26 * VM(m, i) - 10 * VM(m, i - 1) + 2 * VM(m, i - 2)) +
                     bm[2] * (-2 * VM(m, i + 2) + 14 * VM(m, i + 1) + 14 * VM(m, i) - 2 * VM(m, i - 1)) +
                     bm[1] * (2 * VM(m, i + 3) - 10 * VM(m, i + 2) + 26 * VM(m, i + 1) + 6 * VM(m, i)) +
                     bm[0] * (-6 * VM(m, i + 4) + 26 * VM(m, i + 3) - 46 * VM(m, i + 2) + 50 * VM(m, i + 1));
      vhat[m] = (vminus + vplus) / 24.0;
    }
  }
}

// eigenvectors_x / _y / _z (kernels_cpu.F90:2728-2782, 2842-2896, 2956-3010).
// el[r][c], er[r][c] hold the reference's el(r+1,c+1), er(r+1,c+1).
template <class T>
void eigenvectors(int dir, T b1, T b2, T b3, T uu, T vv, T ww, T c, T ci,
                  T h, T el[5][5], T er[5][5]) {
  const T vel[3] = {uu, vv, ww};
  const T vn = vel[dir];
  // left eigenvectors: columns 1 and 5 (acoustic), 2 (entropy), 3 and 4 (tangential)
  el[0][0] = 0.5 * (b1 + vn * ci);
  el[1][0] = -0.5 * (dir == 0 ? b2 * uu + ci : b2 * uu);
  el[2][0] = -0.5 * (dir == 1 ? b2 * vv + ci : b2 * vv);
  el[3][0] = -0.5 * (dir == 2 ? b2 * ww + ci : b2 * ww);
  el[4][0] = 0.5 * b2;
  el[0][1] = 1.0 - b1;
  el[1][1] = b2 * uu;
  el[2][1] = b2 * vv;
  el[3][1] = b2 * ww;
  el[4][1] = -b2;
  el[0][4] = 0.5 * (b1 - vn * ci);
  el[1][4] = -0.5 * (dir == 0 ? b2 * uu - ci : b2 * uu);
  el[2][4] = -0.5 * (dir == 1 ? b2 * vv - ci : b2 * vv);
  el[3][4] = -0.5 * (dir == 2 ? b2 * ww - ci : b2 * ww);
  el[4][4] = 0.5 * b2;
  // tangential components: x -> (v, w), y -> (u, w), z -> (u, v)
  const int t1 = (dir == 0) ? 1 : 0;
  const int t2 = (dir == 2) ? 1 : 2;
  for (int r = 0; r < 5; ++r) el[r][2] = el[r][3] = 0.0;
  el[0][2] = -vel[t1];
  el[1 + t1][2] = 1.0;
  el[0][3] = -vel[t2];
  el[1 + t2][3] = 1.0;
  // right eigenvectors
  for (int r = 0; r < 5; ++r)
    for (int cc = 0; cc < 5; ++cc) er[r][cc] = 0.0;
  er[0][0] = 1.0; er[1][0] = 1.0; er[4][0] = 1.0;
  for (int d = 0; d < 3; ++d) {
    if (d == dir) {
      er[0][1 + d] = vel[d] - c;
      er[1][1 + d] = vel[d];
      er[4][1 + d] = vel[d] + c;
    } else {
      er[0][1 + d] = vel[d];
      er[1][1 + d] = vel[d];
      er[4][1 + d] = vel[d];
    }
  }
  er[2][1 + t1] = 1.0;
  er[3][1 + t2] = 1.0;
  er[0][4] = h - vn * c;
  er[1][4] = b3;
  er[2][4] = vel[t1];
  er[3][4] = vel[t2];
  er[4][4] = h + vn * c;
}

}  // namespace

Solver::Solver(const Setup& setup) : s(setup) {
  nx = s.nxmax; ny = s.nymax; nz = s.nzmax; ng = s.ng;
  sx = nx + 2 * ng; sy = ny + 2 * ng; sz = nz + 2 * ng;
  w = s.w;
  w_aux.assign(ncg() * 10, 0.0);
  // initial_conditions: w_aux(:,:,:,6) = t0 (singleideal.F90:3032)
  for (size_t q = 0; q < ncg(); ++q) w_aux[5 * ncg() + q] = s.t0;
  fl.assign(nint_() * 5, 0.0);
  fln.assign(nint_() * 5, 0.0);
  fhat.assign(ncg() * 5, 0.0);
  wallprop.assign(static_cast<size_t>(sx) * sz * 3, 0.0);
  time = s.time0;
  icyc = s.icyc0;
  random_plane.assign(static_cast<size_t>(ny) * nz * 3, 0.5);  // recyc_prepare's neutral plane
  rng = streams_b200::GlibcRand(s.rng_seed);
  rng.discard(s.rng_draws);
}

// get_temperature_from_e_dev (kernels_cpu.F90:7116-7152)
double Solver::temp_from_e(double ee, double t_start) const {
  const double t0 = s.t0;
  const double ebar = ee - cv(s.indx_cp_r + 1) * t0;
  if (s.calorically_perfect == 1) return t0 + ebar / cv(0);
  double t_old = t_start, tt = t_start;
  for (int iter = 1; iter <= 50; ++iter) {
    double den = 0.0, num = 0.0;
    for (int l = s.indx_cp_l; l <= s.indx_cp_r; ++l) {
      const double t_pow = std::pow(t_old / t0, l);
      if (l == -1) {
        den = den + cv(l) * t_pow;
        num = num + cv(l) * std::log(t_old / t0);
      } else {
        const double t_powp = (t_old / t0) * t_pow;
        den = den + cv(l) * t_pow;
        num = num + cv(l) * (t_powp - 1.0) / (l + 1.0);
      }
    }
    num = num * t0;
    tt = t_old + (ebar - num) / den;
    if (std::fabs(tt - t_old) < 1e-12) break;
    t_old = tt;
  }
  return tt;
}

// get_e_from_temperature_dev (kernels_cpu.F90:7155-7176)
double Solver::e_from_temp(double tt) const {
  const double t0 = s.t0;
  double ee = cv(s.indx_cp_r + 1);
  if (s.calorically_perfect == 1) {
    ee = ee + cv(0) * (tt / t0 - 1.0);
  } else {
    for (int l = s.indx_cp_l; l <= s.indx_cp_r; ++l) {
      if (l == -1) ee = ee + cv(l) * std::log(tt / t0);
      else ee = ee + cv(l) / (l + 1.0) * (std::pow(tt / t0, l + 1) - 1.0);
    }
  }
  return ee * t0;
}

// cp(T) of get_gamloc_dev (kernels_cpu.F90:7096-7113) and of the viscous routines
double Solver::cploc_at(double tt) const {
  if (s.calorically_perfect == 1) return cp(0);
  double cploc = 0.0;
  for (int l = s.indx_cp_l; l <= s.indx_cp_r; ++l) cploc = cploc + cp(l) * std::pow(tt / s.t0, l);
  return cploc;
}

double Solver::gamloc_at(double tt) const {
  const double cploc = cploc_at(tt);
  return cploc / (cploc - s.rgas0);
}

// base_cpu%bcswap (code/src/base_cpu.F90:1326-1435) on one block: face halos of periodic directions
void Solver::bcswap() {
  if (s.periodic[0])
    par_for(1, nz, [&](int k) {
      for (int j = 1; j <= ny; ++j)
        for (int l = 1; l <= ng; ++l)
          for (int m = 0; m < 5; ++m) {
            W(nx + l, j, k, m) = W(l, j, k, m);
            W(1 - l, j, k, m) = W(nx + 1 - l, j, k, m);
          }
    });
  if (s.periodic[1])
    par_for(1, nz, [&](int k) {
      for (int l = 1; l <= ng; ++l)
        for (int i = 1; i <= nx; ++i)
          for (int m = 0; m < 5; ++m) {
            W(i, ny + l, k, m) = W(i, l, k, m);
            W(i, 1 - l, k, m) = W(i, ny + 1 - l, k, m);
          }
    });
  if (s.periodic[2])
    par_for(1, ng, [&](int l) {
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i)
          for (int m = 0; m < 5; ++m) {
            W(i, j, nz + l, m) = W(i, j, l, m);
            W(i, j, 1 - l, m) = W(i, j, nz + 1 - l, m);
          }
    });
}

// base_cpu%bcswap_var (code/src/base_cpu.F90:1835-1912) for w_aux(:,:,:,m)
void Solver::bcswap_var(int m) {
  if (s.periodic[0])
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int l = 1; l <= ng; ++l) {
          A(nx + l, j, k, m) = A(l, j, k, m);
          A(1 - l, j, k, m) = A(nx + 1 - l, j, k, m);
        }
  if (s.periodic[1])
    for (int k = 1; k <= nz; ++k)
      for (int l = 1; l <= ng; ++l)
        for (int i = 1; i <= nx; ++i) {
          A(i, ny + l, k, m) = A(i, l, k, m);
          A(i, 1 - l, k, m) = A(i, ny + 1 - l, k, m);
        }
  if (s.periodic[2])
    for (int l = 1; l <= ng; ++l)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          A(i, j, nz + l, m) = A(i, j, l, m);
          A(i, j, 1 - l, m) = A(i, j, nz + 1 - l, m);
        }
}

// update_ghost (singleideal_cpu.F90:1064-1138): the faces in the order ilat = 1..6
void Solver::update_ghost(int do_swap) {
  for (int ilat = 1; ilat <= 6; ++ilat) {
    switch (s.bctags[ilat - 1]) {
      case 2: bcextr(ilat); break;
      case 6: if (s.is_y_staggered) bcwall_staggered(ilat); else bcwall(ilat); break;
      case 7: if (ilat == 4) bcshock(); break;
      case 10: if (ilat == 1) bcrecyc(); break;
      default: break;
    }
  }
  if (do_swap == 1) bcswap();
}

// bcwall_staggered_subroutine (kernels_cpu.F90:6612-6678)
void Solver::bcwall_staggered(int ilat) {
  if (ilat != 3 && ilat != 4) return;
  const double twall = s.t_wall, rgas0 = s.rgas0;
  par_for(1, nz, [&](int k) {
    for (int l = 1; l <= ng; ++l)
      for (int i = 1; i <= nx; ++i) {
        const int js = (ilat == 3) ? l : ny + 1 - l;
        const int jg = (ilat == 3) ? 1 - l : ny + l;
        double rho = W(i, js, k, 0);
        double uu = W(i, js, k, 1) / rho;
        double vv = W(i, js, k, 2) / rho;
        double ww = W(i, js, k, 3) / rho;
        double rhoe = W(i, js, k, 4);
        double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        double ee = rhoe / rho - qq;
        double tt = temp_from_e(ee, A(i, js, k, 6));
        double pp = rho * tt * rgas0;
        tt = 2.0 * twall - tt;
        ee = e_from_temp(tt);
        rho = pp / tt / rgas0;
        W(i, jg, k, 0) = rho;
        W(i, jg, k, 1) = -rho * uu;
        W(i, jg, k, 2) = -rho * vv;
        W(i, jg, k, 3) = -rho * ww;
        W(i, jg, k, 4) = rho * (ee + qq);
      }
  });
}

// bcwall_subroutine (kernels_cpu.F90:6478-6525): wall node j = 1 at rest and at T_wall, ghosts
// mirrored about it (T_g = 2 T_w - T, p_g = p, velocity reversed); ymin only, as the reference
void Solver::bcwall(int ilat) {
  if (ilat != 3) return;
  const double twall = s.t_wall, rgas0 = s.rgas0;
  par_for(1, nz, [&](int k) {
    for (int i = 1; i <= nx; ++i) {
      W(i, 1, k, 1) = 0.0;
      W(i, 1, k, 2) = 0.0;
      W(i, 1, k, 3) = 0.0;
      double ee = e_from_temp(twall);
      W(i, 1, k, 4) = W(i, 1, k, 0) * ee;
      for (int l = 1; l <= ng; ++l) {
        double rho = W(i, 1 + l, k, 0);
        double uu = W(i, 1 + l, k, 1) / rho;
        double vv = W(i, 1 + l, k, 2) / rho;
        double ww = W(i, 1 + l, k, 3) / rho;
        double rhoe = W(i, 1 + l, k, 4);
        double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        ee = rhoe / rho - qq;
        double tt = temp_from_e(ee, A(i, 1 + l, k, 6));
        double pp = rho * tt * rgas0;
        tt = 2.0 * twall - tt;
        ee = e_from_temp(tt);
        rho = pp / tt / rgas0;
        W(i, 1 - l, k, 0) = rho;
        W(i, 1 - l, k, 1) = -rho * uu;
        W(i, 1 - l, k, 2) = -rho * vv;
        W(i, 1 - l, k, 3) = -rho * ww;
        W(i, 1 - l, k, 4) = rho * (ee + qq);
      }
    }
  });
}

// bcshock_subroutine (kernels_cpu.F90:6159-6196), ymax
void Solver::bcshock() {
  const double tanhlen = 8.0 * s.tanhfacs;
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i)
      for (int l = 0; l <= ng; ++l) {
        const double xsh = s.xshock_imp - Y(ny + l) / std::tan(s.shock_angle);
        const double xx = X(i) - xsh;
        if (std::fabs(xx) > tanhlen) {
          for (int m = 0; m < 5; ++m) W(i, ny + l, k, m) = W(i, ny, k, m);
        } else {
          const double tanhf = 0.5 * (1.0 + std::tanh(xx / s.tanhfacs));
          for (int m = 0; m < 5; ++m) {
            const double dwinf = s.winf_past_shock[m] - s.winf[m];
            W(i, ny + l, k, m) = s.winf[m] + dwinf * tanhf;
          }
        }
      }
}

// bcextr_subroutine (kernels_cpu.F90:6323-6390): zeroth-order extrapolation of all variables
void Solver::bcextr(int ilat) {
  for (int m = 0; m < 5; ++m) {
    if (ilat == 1 || ilat == 2) {
      const int is = ilat == 1 ? 1 : nx;
      for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
          for (int l = 1; l <= ng; ++l) W(ilat == 1 ? 1 - l : nx + l, j, k, m) = W(is, j, k, m);
    } else if (ilat == 3 || ilat == 4) {
      const int js = ilat == 3 ? 1 : ny;
      for (int k = 1; k <= nz; ++k)
        for (int i = 1; i <= nx; ++i)
          for (int l = 1; l <= ng; ++l) W(i, ilat == 3 ? 1 - l : ny + l, k, m) = W(i, js, k, m);
    } else {
      const int ks = ilat == 5 ? 1 : nz;
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i)
          for (int l = 1; l <= ng; ++l) W(i, j, ilat == 5 ? 1 - l : nz + l, m) = W(i, j, ks, m);
    }
  }
}

// recyc_exchange (singleideal_cpu.F90:935-999) on one block: the plane i_recyc+1-i, i = 1..ng,
// shifted in z by nzmax/2 (recyc_exchange_subroutine_1..3, kernels_cpu.F90:5003-5060), then
// bcrecyc_subroutine_1..3 (:5810-5947): spanwise means, fluctuations, rescaled inflow ghosts.
void Solver::bcrecyc() {
  const int kshift = s.nzmax / 2;
  const int ir = s.i_recyc;
  const size_t pl = static_cast<size_t>(ng) * ny * nz;
  std::vector<double> wr(pl * 5);
  auto WR = [&](int i, int j, int k, int m) -> double& {
    return wr[(static_cast<size_t>(m - 1) * nz + (k - 1)) * ny * ng + static_cast<size_t>(j - 1) * ng + (i - 1)];
  };
  for (int k = 1; k <= nz; ++k) {
    const int ks = ((k - kshift - 1) % nz + nz) % nz + 1;
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= ng; ++i)
        for (int m = 1; m <= 5; ++m) WR(i, j, k, m) = W(ir + 1 - i, j, ks, m - 1);
  }
  std::vector<double> av(static_cast<size_t>(ng) * ny * 5);
  auto AV = [&](int i, int j, int m) -> double& { return av[(static_cast<size_t>(m - 1) * ny + (j - 1)) * ng + (i - 1)]; };
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= ng; ++i)
      for (int m = 1; m <= 5; ++m) {
        double a = 0.0;
        for (int k = 1; k <= nz; ++k) a = a + WR(i, j, k, m);
        AV(i, j, m) = a;
      }
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= ng; ++i) {
      const double ufav = AV(i, j, 2) / AV(i, j, 1);
      const double vfav = AV(i, j, 3) / AV(i, j, 1);
      const double wfav = AV(i, j, 4) / AV(i, j, 1);
      const double rhom = AV(i, j, 1) / s.nzmax;
      for (int k = 1; k <= nz; ++k) {
        WR(i, j, k, 2) = WR(i, j, k, 2) / WR(i, j, k, 1) - ufav;
        WR(i, j, k, 3) = WR(i, j, k, 3) / WR(i, j, k, 1) - vfav;
        WR(i, j, k, 4) = WR(i, j, k, 4) / WR(i, j, k, 1) - wfav;
        WR(i, j, k, 1) = WR(i, j, k, 1) - rhom;
      }
    }
  const double p0 = s.p0, rgas0 = s.rgas0, betarecyc = s.betarecyc;
  double u0_02 = 0.02 * s.u0;
  if (s.rand_type == 0) u0_02 = 0.0;
  auto yo = [&](const std::vector<double>& v, int j) { return v[static_cast<size_t>(j + ng - 1)]; };
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const double eta = yo(s.eta_inflow, j);
      const double etamin = std::min(eta, 1.0);
      const double weta = s.weta_inflow[j - 1];
      const double weta1 = 1.0 - weta;
      const double bdamp = 0.5 * (1.0 - std::tanh(4.0 * (yo(s.eta_inflow, j) - 2.0)));
      const int j_inn = s.map_j_inn[j - 1], j_out = s.map_j_out[j - 1];
      const double disty_inn = (yo(s.yplus_inflow, j) - yo(s.yplus_recyc, j_inn)) /
                               (yo(s.yplus_recyc, j_inn + 1) - yo(s.yplus_recyc, j_inn));
      const double disty_out = (yo(s.eta_inflow, j) - yo(s.eta_recyc, j_out)) /
                               (yo(s.eta_recyc, j_out + 1) - yo(s.eta_recyc, j_out));
      for (int i = 1; i <= ng; ++i) {
        auto WMI = [&](int m) { return s.wmean_inflow[(static_cast<size_t>(m - 1) * ny + (j - 1)) * ng + (i - 1)]; };
        const double rhomean = WMI(1);
        const double uumean = WMI(2) / rhomean, vvmean = WMI(3) / rhomean, wwmean = WMI(4) / rhomean;
        double rhofluc, ufluc, vfluc, wfluc;
        if (j == 1 || j_inn >= ny || j_out >= ny) {
          rhofluc = ufluc = vfluc = wfluc = 0.0;
        } else {
          auto mix = [&](int m, int jj, double d) { return WR(i, jj, k, m) * (1.0 - d) + WR(i, jj + 1, k, m) * d; };
          const double rhof_inn = mix(1, j_inn, disty_inn), rhof_out = mix(1, j_out, disty_out);
          const double uf_inn = mix(2, j_inn, disty_inn), uf_out = mix(2, j_out, disty_out);
          const double vf_inn = mix(3, j_inn, disty_inn), vf_out = mix(3, j_out, disty_out);
          const double wf_inn = mix(4, j_inn, disty_inn), wf_out = mix(4, j_out, disty_out);
          rhofluc = rhof_inn * weta1 + rhof_out * weta;
          ufluc = uf_inn * weta1 + uf_out * weta;
          vfluc = vf_inn * weta1 + vf_out * weta;
          wfluc = wf_inn * weta1 + wf_out * weta;
          rhofluc = rhofluc * bdamp;
          ufluc = ufluc * bdamp * betarecyc;
          vfluc = vfluc * bdamp * betarecyc;
          wfluc = wfluc * bdamp * betarecyc;
          auto RP = [&](int c) { return random_plane[(static_cast<size_t>(c - 1) * nz + (k - 1)) * ny + (j - 1)]; };
          ufluc = ufluc + u0_02 * (RP(1) - 0.5) * etamin;
          vfluc = vfluc + u0_02 * (RP(2) - 0.5) * etamin;
          wfluc = wfluc + u0_02 * (RP(3) - 0.5) * etamin;
        }
        rhofluc = std::max(-0.75 * rhomean, rhofluc);
        rhofluc = std::min(4.0 * rhomean, rhofluc);
        const double rho = rhomean + rhofluc;
        const double tt = p0 / rho / rgas0;
        const double uu = uumean + ufluc, vv = vvmean + vfluc, ww = wwmean + wfluc;
        const double rhou = rho * uu, rhov = rho * vv, rhow = rho * ww;
        const double ee = e_from_temp(tt);
        W(1 - i, j, k, 0) = rho;
        W(1 - i, j, k, 1) = rhou;
        W(1 - i, j, k, 2) = rhov;
        W(1 - i, j, k, 3) = rhow;
        W(1 - i, j, k, 4) = rho * ee + 0.5 * (rhou * rhou + rhov * rhov + rhow * rhow) / rho;
      }
    }
}

// euler_z's draw of the recycling plane (singleideal_cpu.F90:841): get_crandom_f on
// inflow_random_plane(2:jbl_inflow, 1:nz, 1:3), first index outermost (crandom_f.F90:81-93)
void Solver::draw_random_plane() {
  const double rescale = s.rng_seed == 0 ? 0.0 : 1.0;
  for (int j = 2; j <= s.jbl_inflow; ++j)
    for (int k = 1; k <= nz; ++k)
      for (int c = 1; c <= 3; ++c)
        random_plane[(static_cast<size_t>(c - 1) * nz + (k - 1)) * ny + (j - 1)] =
            rescale * static_cast<double>(rng()) / RAND_MAX;
}

// eval_aux_subroutine (kernels_cpu.F90:6960-7011)
void Solver::eval_aux(int i0, int i1, int j0, int j1, int k0, int k1) {
  const double t0 = s.t0, rgas0 = s.rgas0;
  const double mu0 = s.mu0, vtexp = s.powerlaw_vtexp, ss = s.sutherland_s, trd = s.t_ref_dim;
  const int vm = s.visc_model;
  par_for(k0, k1, [&](int k) {
    for (int j = j0; j <= j1; ++j)
      for (int i = i0; i <= i1; ++i) {
        double rho = W(i, j, k, 0), rhou = W(i, j, k, 1), rhov = W(i, j, k, 2), rhow = W(i, j, k, 3),
               rhoe = W(i, j, k, 4);
        double ri = 1.0 / rho;
        double uu = rhou * ri, vv = rhov * ri, ww = rhow * ri;
        double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        double ee = rhoe / rho - qq;
        double tt = temp_from_e(ee, A(i, j, k, 6));
        double pp = rho * tt * rgas0;
        A(i, j, k, 1) = rho;
        A(i, j, k, 2) = uu;
        A(i, j, k, 3) = vv;
        A(i, j, k, 4) = ww;
        A(i, j, k, 5) = (rhoe + pp) / rho;
        A(i, j, k, 6) = tt;
        double mu = 0.0;
        if (vm == 1)
          mu = mu0 * std::pow(tt / t0, vtexp);
        else if (vm == 2)
          mu = mu0 * std::pow(tt / t0, 1.5) * (1.0 + ss / trd) / (tt / t0 + ss / trd);
        A(i, j, k, 7) = mu;
      }
  });
}

// compute_aux (singleideal_cpu.F90:281-330)
void Solver::compute_aux(int central, int ghost) {
  if (central == 1 && ghost == 1) {
    eval_aux(1 - ng, nx + ng, 1 - ng, ny + ng, 1 - ng, nz + ng);
  } else if (central == 1 && ghost == 0) {
    eval_aux(1, nx, 1, ny, 1, nz);
  } else if (central == 0 && ghost == 1) {
    eval_aux(1 - ng, 0, 1 - ng, ny + ng, 1 - ng, nz + ng);
    eval_aux(nx + 1, nx + ng, 1 - ng, ny + ng, 1 - ng, nz + ng);
    eval_aux(1 - ng, nx + ng, 1 - ng, 0, 1 - ng, nz + ng);
    eval_aux(1 - ng, nx + ng, ny + 1, ny + ng, 1 - ng, nz + ng);
    eval_aux(1 - ng, nx + ng, 1 - ng, ny + ng, 1 - ng, 0);
    eval_aux(1 - ng, nx + ng, 1 - ng, ny + ng, nz + 1, nz + ng);
  }
}

// Hybrid convective flux at one face (euler_x_fluxes_hybrid_kernel kernels_cpu.F90:425-689,
// euler_z_hybrid_kernel :1063-1325, euler_y_hybrid_kernel :1808-2071).  The face lies between
// the point (i,j,k) and its neighbour +1 along dir.
template <class T>
void Solver::face_flux_t(int dir, int i, int j, int k, T fh[5]) const {
  using std::fabs;
  using std::log;
  using std::max;
  using std::pow;
  using std::sqrt;
  const int ex = dir == 0, ey = dir == 1, ez = dir == 2;
  auto at = [&](int o, int m) { return T(A(i + o * ex, j + o * ey, k + o * ez, m)); };
  const int pos = dir == 0 ? i : (dir == 1 ? j : k);
  const int nd = dir == 0 ? nx : (dir == 1 ? ny : nz);
  const int ws = s.weno_scheme;
  const double rgas0 = s.rgas0;
  int ishk = 0;
  for (int o = -ws + 1; o <= ws; ++o)
    if (at(o, 8) > s.sensor_threshold) ishk = 1;
  const int epo = s.ep_ord[dir][pos];
  if (ishk == 0) {
    T ft1 = 0, ft2 = 0, ft3 = 0, ft4 = 0, ft5 = 0, ft6 = 0;
    const int lmax = max(s.ep_order / 2 + epo, 1);
    for (int l = 1; l <= lmax; ++l) {
      T uvs1 = 0, uvs2 = 0, uvs3 = 0, uvs4 = 0, uvs5 = 0, uvs5_i = 0, uvs5_k = 0, uvs5_p = 0, uvs6 = 0;
      for (int m = 0; m <= l - 1; ++m) {
        T rhoi = at(-m, 1), uui = at(-m, 2), vvi = at(-m, 3), wwi = at(-m, 4), enti = at(-m, 5),
               tti = at(-m, 6);
        T ppi = tti * rhoi * rgas0;
        T rhoip = at(-m + l, 1), uuip = at(-m + l, 2), vvip = at(-m + l, 3), wwip = at(-m + l, 4),
               entip = at(-m + l, 5), ttip = at(-m + l, 6);
        T ppip = ttip * rhoip * rgas0;
        const T vni = dir == 0 ? uui : (dir == 1 ? vvi : wwi);
        const T vnip = dir == 0 ? uuip : (dir == 1 ? vvip : wwip);
        T rhom = rhoi + rhoip;
        if (s.nkeep >= 0) {
          T eei = enti - ppi / rhoi - 0.5 * (uui * uui + vvi * vvi + wwi * wwi);
          T eeip = entip - ppip / rhoip - 0.5 * (uuip * uuip + vvip * vvip + wwip * wwip);
          T eem = eei + eeip;
          T drhof = 1.0, deef = 1.0;
          if (s.nkeep != 0) {
            T sumnumrho = 1.0;
            T drho = 2.0 * (rhoip - rhoi) / rhom;
            T dee = 2.0 * (eeip - eei) / eem;
            T t_sumdenrho = (0.5 * drho) * (0.5 * drho);
            T t_sumdenee = (0.5 * dee) * (0.5 * dee);
            T t2_sumdenrho = t_sumdenrho, t2_sumdenee = t_sumdenee;
            T sumdenrho = 1.0 + t_sumdenrho / 3.0;
            T sumdenee = 1.0 + t_sumdenee;
            T sumnumee = 1.0 + t_sumdenee / 3.0;
            for (int n = 2; n <= s.nkeep; ++n) {
              int n2 = 2 * n;
              t_sumdenrho = t2_sumdenrho * t_sumdenrho;
              t_sumdenee = t2_sumdenee * t_sumdenee;
              sumdenrho = sumdenrho + t_sumdenrho / (1.0 + n2);
              sumdenee = sumdenee + t_sumdenee;
              sumnumee = sumnumee + t_sumdenee / (1.0 + n2);
            }
            drhof = sumnumrho / sumdenrho;
            deef = sumnumee / sumdenee;
          }
          T uv_part = (vni + vnip) * rhom * drhof;
          uvs1 = uvs1 + uv_part * 2.0;
          uvs2 = uvs2 + uv_part * (uui + uuip);
          uvs3 = uvs3 + uv_part * (vvi + vvip);
          uvs4 = uvs4 + uv_part * (wwi + wwip);
          uvs5_i = uvs5_i + uv_part * eem * deef;
          uvs5_k = uvs5_k + uv_part * (uui * uuip + vvi * vvip + wwi * wwip);
          uvs5_p = uvs5_p + 4.0 * (vni * ppip + vnip * ppi);
          uvs6 = uvs6 + 2.0 * (ppi + ppip);
        } else {
          T uv_part = (vni + vnip) * rhom;
          uvs1 = uvs1 + uv_part * 2.0;
          uvs2 = uvs2 + uv_part * (uui + uuip);
          uvs3 = uvs3 + uv_part * (vvi + vvip);
          uvs4 = uvs4 + uv_part * (wwi + wwip);
          uvs5 = uvs5 + uv_part * (enti + entip);
          uvs6 = uvs6 + 2.0 * (ppi + ppip);
        }
      }
      const double cl = s.coeff_deriv1[lmax - 1][l - 1];
      ft1 = ft1 + cl * uvs1;
      ft2 = ft2 + cl * uvs2;
      ft3 = ft3 + cl * uvs3;
      ft4 = ft4 + cl * uvs4;
      if (s.nkeep >= 0)
        ft5 = ft5 + cl * (uvs5_i + uvs5_k + uvs5_p);
      else
        ft5 = ft5 + cl * uvs5;
      ft6 = ft6 + cl * uvs6;
    }
    fh[0] = 0.25 * ft1;
    fh[1] = 0.25 * ft2;
    fh[2] = 0.25 * ft3;
    fh[3] = 0.25 * ft4;
    fh[4] = 0.25 * ft5;
    if ((pos == 0 && s.force_zero_flux[2 * dir] == 1) || (pos == nd && s.force_zero_flux[2 * dir + 1] == 1))
      for (int m = 0; m < 5; ++m) fh[m] = 0.0;
    fh[1 + dir] = fh[1 + dir] + 0.5 * ft6;
  } else if (s.flux_splitting == 1) {
    // Rusanov (component-wise local Lax-Friedrichs) WENO branch of the *_hybrid_rusanov kernels
    // (kernels_cpu.F90:692-941 for x): stencil maximum of |u_n -+ c|, split of the conserved
    // fluxes, wenorec_1d_rusanov
    T evmax = -1.0;
    for (int l = 1; l <= 2 * ws; ++l) {
      const int o = l - ws;
      const T un = at(o, 2 + dir), tt = at(o, 6);
      const T c = sqrt(T(gamloc_at(static_cast<double>(tt))) * rgas0 * tt);
      const T evm = max(fabs(un - c), fabs(un + c));
      evmax = max(evm, evmax);
    }
    T gp[5][8], gm[5][8];
    for (int l = 1; l <= 2 * ws; ++l) {
      const int o = l - ws;
      const T rho = at(o, 1), h = at(o, 5);
      const T vel[3] = {at(o, 2), at(o, 3), at(o, 4)};
      const T rhou = rho * vel[dir];
      const T pp = rho * at(o, 6) * rgas0;
      const T rhoevm = rho * evmax;
      T evm = rhou;
      T c = 0.5 * (evm + rhoevm);
      gp[0][l - 1] = c;
      gm[0][l - 1] = evm - c;
      for (int d = 0; d < 3; ++d) {
        evm = vel[d] * rhou;
        if (d == dir) evm = evm + pp;
        c = 0.5 * (evm + rhoevm * vel[d]);
        gp[1 + d][l - 1] = c;
        gm[1 + d][l - 1] = evm - c;
      }
      evm = h * rhou;
      c = 0.5 * (evm + evmax * (rho * h - pp));
      gp[4][l - 1] = c;
      gm[4][l - 1] = evm - c;
    }
    const int ord = max(ws + epo, 1);
    wenorec_1d(gp, gm, fh, ws, ord, s.weno_version, s.rho0, s.u0, true);
  } else {
    // compute_roe_average (kernels_cpu.F90:3013-3089)
    T uu = at(0, 2), vv = at(0, 3), ww = at(0, 4);
    T h = at(0, 5);
    T up = at(1, 2), vp = at(1, 3), wp = at(1, 4);
    T hp = at(1, 5);
    T r = at(1, 1) / at(0, 1);
    r = sqrt(r);
    T rho = r * at(0, 1);
    T rp1 = 1.0 / (r + 1.0);
    uu = (r * up + uu) * rp1;
    vv = (r * vp + vv) * rp1;
    ww = (r * wp + ww) * rp1;
    h = (r * hp + h) * rp1;
    T qq = 0.5 * (uu * uu + vv * vv + ww * ww);
    T hbar = h - qq - cp(s.indx_cp_r + 1) * s.t0;
    T tt, gamloc;
    if (s.calorically_perfect == 1) {
      tt = s.t0 + hbar / T(cp(0));
      gamloc = cp(0) / (cp(0) - rgas0);
    } else {
      tt = at(0, 6);
      const T ttp = at(1, 6);
      tt = (r * ttp + tt) * rp1;
      T told = tt;
      for (int iter = 1; iter <= 50; ++iter) {
        T num = 0.0, den = 0.0;
        for (int ll = s.indx_cp_l; ll <= s.indx_cp_r; ++ll) {
          const T tpow = pow(told / s.t0, ll);
          if (ll == -1) {
            den = den + cp(ll) * tpow;
            num = num + cp(ll) * log(told / s.t0);
          } else {
            const T tpowp = (told / s.t0) * tpow;
            den = den + cp(ll) * tpow;
            num = num + cp(ll) * (tpowp - 1.0) / (ll + 1.0);
          }
        }
        num = num * s.t0;
        tt = told + (hbar - num) / den;
        if (fabs(tt - told) < 1e-12) break;
        told = tt;
      }
      gamloc = T(gamloc_at(static_cast<double>(tt)));
    }
    T cc = gamloc * tt * rgas0;
    T gm1loc = gamloc - 1.0;
    T c = sqrt(cc);
    T ci = 1.0 / c;
    T p_rho = tt * rgas0;
    T p_e = rho * gm1loc;
    T etot = h - tt * rgas0;
    T b3 = etot - rho * p_rho / p_e;
    T b2 = p_e / (rho * cc);
    T b1 = p_rho / cc - b2 * (etot - 2.0 * qq);
    T el[5][5], er[5][5];
    eigenvectors(dir, b1, b2, b3, uu, vv, ww, c, ci, h, el, er);
    T evmax[5];
    for (int m = 0; m < 5; ++m) evmax[m] = -1.0;
    const int wsz = 2 * ws;
    for (int l = 1; l <= wsz; ++l) {
      const int o = l - ws;
      T vn = at(o, 2 + dir);
      T t = at(o, 6);
      T gl = T(gamloc_at(static_cast<double>(t)));
      T cs = sqrt(gl * rgas0 * t);
      evmax[0] = max(fabs(vn - cs), evmax[0]);
      evmax[1] = max(fabs(vn), evmax[1]);
      evmax[2] = evmax[1];
      evmax[3] = evmax[1];
      evmax[4] = max(fabs(vn + cs), evmax[4]);
    }
    T gp[5][8], gm[5][8];
    for (int l = 1; l <= wsz; ++l) {
      const int o = l - ws;
      T rr = at(o, 1), u1 = at(o, 2), v1 = at(o, 3), w1 = at(o, 4), h1 = at(o, 5);
      T vn = dir == 0 ? u1 : (dir == 1 ? v1 : w1);
      T rhovn = rr * vn;
      T pp = rr * at(o, 6) * rgas0;
      T fi[5];
      fi[0] = rhovn;
      fi[1] = u1 * rhovn;
      fi[2] = v1 * rhovn;
      fi[3] = w1 * rhovn;
      fi[1 + dir] = fi[1 + dir] + pp;
      fi[4] = h1 * rhovn;
      for (int m = 0; m < 5; ++m) {
        T wc = 0.0, gc = 0.0;
        wc = wc + el[0][m] * rr;
        gc = gc + el[0][m] * fi[0];
        wc = wc + el[1][m] * rr * u1;
        gc = gc + el[1][m] * fi[1];
        wc = wc + el[2][m] * rr * v1;
        gc = gc + el[2][m] * fi[2];
        wc = wc + el[3][m] * rr * w1;
        gc = gc + el[3][m] * fi[3];
        wc = wc + el[4][m] * (rr * h1 - pp);
        gc = gc + el[4][m] * fi[4];
        T cm = 0.5 * (gc + evmax[m] * wc);
        gp[m][l - 1] = cm;
        gm[m][l - 1] = gc - cm;
      }
    }
    const int ord = max(ws + epo, 1);
    T fi[5];
    wenorec_1d(gp, gm, fi, ws, ord, s.weno_version, s.rho0, s.u0);
    for (int m = 0; m < 5; ++m) {
      T acc = 0.0;
      for (int mm = 0; mm < 5; ++mm) acc = acc + er[mm][m] * fi[mm];
      fh[m] = acc;
    }
  }
}

void Solver::face_flux(int dir, int i, int j, int k, double fh[5]) const { face_flux_t<double>(dir, i, j, k, fh); }

template void Solver::face_flux_t<Counted>(int, int, int, int, Counted*) const;

// euler_x / euler_y / euler_z (singleideal_cpu.F90:674-843) = hybrid flux kernel + update
// (euler_{x,y,z}_update_subroutine, kernels_cpu.F90:944-963, 991-1010, 1039-1058)
void Solver::euler(int dir) {
  int f0, f1;
  if (dir == 0) { f0 = s.eul_imin - 1; f1 = s.eul_imax; }
  else if (dir == 1) { f0 = s.eul_jmin - 1; f1 = s.eul_jmax; }
  else { f0 = s.eul_kmin - 1; f1 = s.eul_kmax; }
  if (f1 - (f0 + 1) < 0) return;
  const int i0 = dir == 0 ? f0 : 1, i1 = dir == 0 ? f1 : nx;
  const int j0 = dir == 1 ? f0 : 1, j1 = dir == 1 ? f1 : ny;
  const int k0 = dir == 2 ? f0 : 1, k1 = dir == 2 ? f1 : nz;
  par_for(k0, k1, [&](int k) {
    for (int j = j0; j <= j1; ++j)
      for (int i = i0; i <= i1; ++i) {
        double fh[5];
        face_flux(dir, i, j, k, fh);
        for (int m = 0; m < 5; ++m) FH(i, j, k, m + 1) = fh[m];
      }
  });
  const int ex = dir == 0, ey = dir == 1, ez = dir == 2;
  const int u0i = dir == 0 ? f0 + 1 : 1, u1i = dir == 0 ? f1 : nx;
  const int u0j = dir == 1 ? f0 + 1 : 1, u1j = dir == 1 ? f1 : ny;
  const int u0k = dir == 2 ? f0 + 1 : 1, u1k = dir == 2 ? f1 : nz;
  par_for(u0k, u1k, [&](int k) {
    for (int j = u0j; j <= u1j; ++j)
      for (int i = u0i; i <= u1i; ++i) {
        const double met = dir == 0 ? s.dcsidx[i - 1] : (dir == 1 ? s.detady[j - 1] : s.dzitdz[k - 1]);
        for (int iv = 1; iv <= 5; ++iv)
          FL(i, j, k, iv) = FL(i, j, k, iv) + (FH(i, j, k, iv) - FH(i - ex, j - ey, k - ez, iv)) * met;
      }
  });
}

// visflx_reduced_ord2_subroutine (kernels_cpu.F90:4623-4721)
void Solver::visflx_reduced_ord2(int update_sensor) {
  const double prandtl = s.prandtl, u0 = s.u0, l0 = s.l0;
  par_for(1, nz, [&](int k) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double uu = A(i, j, k, 2), vv = A(i, j, k, 3), ww = A(i, j, k, 4), mu = A(i, j, k, 7);
        double dxl = 1.0 / (X(i + 1) - X(i - 1));
        double dyl = 1.0 / (Y(j + 1) - Y(j - 1));
        double dzl = 1.0 / (Z(k + 1) - Z(k - 1));
        double ux = dxl * (A(i + 1, j, k, 2) - A(i - 1, j, k, 2));
        double vx = dxl * (A(i + 1, j, k, 3) - A(i - 1, j, k, 3));
        double wx = dxl * (A(i + 1, j, k, 4) - A(i - 1, j, k, 4));
        double mux = dxl * (A(i + 1, j, k, 7) - A(i - 1, j, k, 7));
        double uy = dyl * (A(i, j + 1, k, 2) - A(i, j - 1, k, 2));
        double vy = dyl * (A(i, j + 1, k, 3) - A(i, j - 1, k, 3));
        double wy = dyl * (A(i, j + 1, k, 4) - A(i, j - 1, k, 4));
        double ty = dyl * (A(i, j + 1, k, 6) - A(i, j - 1, k, 6));
        double muy = dyl * (A(i, j + 1, k, 7) - A(i, j - 1, k, 7));
        double uz = dzl * (A(i, j, k + 1, 2) - A(i, j, k - 1, 2));
        double vz = dzl * (A(i, j, k + 1, 3) - A(i, j, k - 1, 3));
        double wz = dzl * (A(i, j, k + 1, 4) - A(i, j, k - 1, 4));
        double muz = dzl * (A(i, j, k + 1, 7) - A(i, j, k - 1, 7));
        if (j == 1) {
          wallprop[(0 * sz + k + ng - 1) * sx + i + ng - 1] = mu * uy;
          wallprop[(1 * sz + k + ng - 1) * sx + i + ng - 1] = mu * wy;
          wallprop[(2 * sz + k + ng - 1) * sx + i + ng - 1] = mu * ty * cploc_at(A(i, j, k, 6)) / prandtl;
        }
        double div = ux + vy + wz;
        double div3l = div / 3.0;
        A(i, j, k, 10) = div3l;
        double omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
        double omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
        A(i, j, k, 9) = std::sqrt(omod2);
        if (update_sensor == 1) {
          double t = std::max(-div / std::sqrt(omod2 + div * div + (u0 / l0) * (u0 / l0)), 0.0);
          A(i, j, k, 8) = t * t;
        }
        double sig11 = ux - 2.0 * div3l, sig12 = vx, sig13 = wx;
        double sig21 = uy, sig22 = vy - 2.0 * div3l, sig23 = wy;
        double sig31 = uz, sig32 = vz, sig33 = wz - 2.0 * div3l;
        double sigx = mux * sig11 + muy * sig12 + muz * sig13;
        double sigy = mux * sig21 + muy * sig22 + muz * sig23;
        double sigz = mux * sig31 + muy * sig32 + muz * sig33;
        double sigah = (sig11 * ux + sig12 * uy + sig13 * uz + sig21 * vx + sig22 * vy + sig23 * vz + sig31 * wx +
                        sig32 * wy + sig33 * wz) *
                       mu;
        double sigq = sigx * uu + sigy * vv + sigz * ww + sigah;
        FL(i, j, k, 2) = FL(i, j, k, 2) - sigx;
        FL(i, j, k, 3) = FL(i, j, k, 3) - sigy;
        FL(i, j, k, 4) = FL(i, j, k, 4) - sigz;
        FL(i, j, k, 5) = FL(i, j, k, 5) - sigq;
      }
  });
}

// visflx_x / _y / _z_subroutine (kernels_cpu.F90:4779-4999): conservative face Laplacian
void Solver::visflx_faces() {
  const double prandtl = s.prandtl;
  // x: face fluxes into fhat(2:5), then the divergence
  par_for(1, nz, [&](int k) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        double uu = A(i, j, k, 2), uup = A(i + 1, j, k, 2), vv = A(i, j, k, 3), vvp = A(i + 1, j, k, 3);
        double ww = A(i, j, k, 4), wwp = A(i + 1, j, k, 4), tt = A(i, j, k, 6), ttp = A(i + 1, j, k, 6);
        double mu = A(i, j, k, 7), mup = A(i + 1, j, k, 7);
        double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        double qqp = 0.5 * (uup * uup + vvp * vvp + wwp * wwp);
        double sigx = uup - uu, sigy = vvp - vv, sigz = wwp - ww, sigq_tt = ttp - tt, sigq_qq = qqp - qq;
        double muf = mu + mup;
        muf = 0.5 * muf / (X(i + 1) - X(i));
        sigx = sigx * muf;
        sigy = sigy * muf;
        sigz = sigz * muf;
        double sigq = (sigq_tt * cploc_at(0.5 * (tt + ttp)) / prandtl + sigq_qq) * muf;
        FH(i, j, k, 2) = -sigx;
        FH(i, j, k, 3) = -sigy;
        FH(i, j, k, 4) = -sigz;
        FH(i, j, k, 5) = -sigq;
      }
  });
  par_for(1, nz, [&](int k) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double dxhl = 2.0 / (X(i + 1) - X(i - 1));
        for (int iv = 2; iv <= 5; ++iv) FL(i, j, k, iv) = FL(i, j, k, iv) + dxhl * (FH(i, j, k, iv) - FH(i - 1, j, k, iv));
      }
  });
  // y: carried face flux along j
  par_for(1, nz, [&](int k) {
    for (int i = 1; i <= nx; ++i) {
      double dyhl = 0, fl2o = 0, fl3o = 0, fl4o = 0, fl5o = 0;
      for (int j = 0; j <= ny; ++j) {
        double uu = A(i, j, k, 2), uup = A(i, j + 1, k, 2), vv = A(i, j, k, 3), vvp = A(i, j + 1, k, 3);
        double ww = A(i, j, k, 4), wwp = A(i, j + 1, k, 4), tt = A(i, j, k, 6), ttp = A(i, j + 1, k, 6);
        double mu = A(i, j, k, 7), mup = A(i, j + 1, k, 7);
        double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        double qqp = 0.5 * (uup * uup + vvp * vvp + wwp * wwp);
        double sigx = uup - uu, sigy = vvp - vv, sigz = wwp - ww, sigq_tt = ttp - tt, sigq_qq = qqp - qq;
        double muf = mu + mup;
        muf = 0.5 * muf / (Y(j + 1) - Y(j));
        sigx = sigx * muf;
        sigy = sigy * muf;
        sigz = sigz * muf;
        double sigq = (sigq_tt * cploc_at(0.5 * (tt + ttp)) / prandtl + sigq_qq) * muf;
        if (j > 0) {
          FL(i, j, k, 2) = FL(i, j, k, 2) + fl2o - sigx * dyhl;
          FL(i, j, k, 3) = FL(i, j, k, 3) + fl3o - sigy * dyhl;
          FL(i, j, k, 4) = FL(i, j, k, 4) + fl4o - sigz * dyhl;
          FL(i, j, k, 5) = FL(i, j, k, 5) + fl5o - sigq * dyhl;
        }
        if (j < ny) {
          dyhl = 2.0 / (Y(j + 2) - Y(j));
          fl2o = sigx * dyhl;
          fl3o = sigy * dyhl;
          fl4o = sigz * dyhl;
          fl5o = sigq * dyhl;
        }
      }
    }
  });
  // z: carried face flux along k
  par_for(1, ny, [&](int j) {
    for (int i = 1; i <= nx; ++i) {
      double dzhl = 0, fl2o = 0, fl3o = 0, fl4o = 0, fl5o = 0;
      for (int k = 0; k <= nz; ++k) {
        double uu = A(i, j, k, 2), uup = A(i, j, k + 1, 2), vv = A(i, j, k, 3), vvp = A(i, j, k + 1, 3);
        double ww = A(i, j, k, 4), wwp = A(i, j, k + 1, 4), tt = A(i, j, k, 6), ttp = A(i, j, k + 1, 6);
        double mu = A(i, j, k, 7), mup = A(i, j, k + 1, 7);
        double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        double qqp = 0.5 * (uup * uup + vvp * vvp + wwp * wwp);
        double sigx = uup - uu, sigy = vvp - vv, sigz = wwp - ww, sigq_tt = ttp - tt, sigq_qq = qqp - qq;
        double muf = mu + mup;
        muf = 0.5 * muf / (Z(k + 1) - Z(k));
        sigx = sigx * muf;
        sigy = sigy * muf;
        sigz = sigz * muf;
        double sigq = (sigq_tt * cploc_at(0.5 * (tt + ttp)) / prandtl + sigq_qq) * muf;
        if (k > 0) {
          FL(i, j, k, 2) = FL(i, j, k, 2) + fl2o - sigx * dzhl;
          FL(i, j, k, 3) = FL(i, j, k, 3) + fl3o - sigy * dzhl;
          FL(i, j, k, 4) = FL(i, j, k, 4) + fl4o - sigz * dzhl;
          FL(i, j, k, 5) = FL(i, j, k, 5) + fl5o - sigq * dzhl;
        }
        if (k < nz) {
          dzhl = 2.0 / (Z(k + 2) - Z(k));
          fl2o = sigx * dzhl;
          fl3o = sigy * dzhl;
          fl4o = sigz * dzhl;
          fl5o = sigq * dzhl;
        }
      }
    }
  });
}

// sensor_subroutine (kernels_cpu.F90:4726-4744)
void Solver::sensor() {
  const double u0 = s.u0, l0 = s.l0;
  par_for(1, nz, [&](int k) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double omod2 = A(i, j, k, 9) * A(i, j, k, 9);
        double div = 3.0 * A(i, j, k, 10);
        double t = std::max(-div / std::sqrt(omod2 + div * div + (u0 / l0) * (u0 / l0)), 0.0);
        A(i, j, k, 8) = t * t;
      }
  });
}

// bcextr_var_subroutine (kernels_cpu.F90:6199-6254)
void Solver::bcextr_var(int m) {
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int l = 1; l <= ng; ++l) A(1 - l, j, k, m) = A(1, j, k, m);
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int l = 1; l <= ng; ++l) A(nx + l, j, k, m) = A(nx, j, k, m);
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i)
      for (int l = 1; l <= ng; ++l) A(i, 1 - l, k, m) = A(i, 1, k, m);
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i)
      for (int l = 1; l <= ng; ++l) A(i, ny + l, k, m) = A(i, ny, k, m);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int l = 1; l <= ng; ++l) A(i, j, 1 - l, m) = A(i, j, 1, m);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int l = 1; l <= ng; ++l) A(i, j, nz + l, m) = A(i, j, nz, m);
}

// visflx_div_ord2_subroutine (kernels_cpu.F90:3446-3480)
void Solver::visflx_div_ord2() {
  par_for(1, nz, [&](int k) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double uu = A(i, j, k, 2), vv = A(i, j, k, 3), ww = A(i, j, k, 4), mu = A(i, j, k, 7);
        double dxl = mu / (X(i + 1) - X(i - 1));
        double dyl = mu / (Y(j + 1) - Y(j - 1));
        double dzl = mu / (Z(k + 1) - Z(k - 1));
        double sigx = dxl * (A(i + 1, j, k, 10) - A(i - 1, j, k, 10));
        double sigy = dyl * (A(i, j + 1, k, 10) - A(i, j - 1, k, 10));
        double sigz = dzl * (A(i, j, k + 1, 10) - A(i, j, k - 1, 10));
        double sigq = sigx * uu + sigy * vv + sigz * ww;
        FL(i, j, k, 2) = FL(i, j, k, 2) - sigx;
        FL(i, j, k, 3) = FL(i, j, k, 3) - sigy;
        FL(i, j, k, 4) = FL(i, j, k, 4) - sigz;
        FL(i, j, k, 5) = FL(i, j, k, 5) - sigq;
      }
  });
}

// visflx_nosensor_subroutine (kernels_cpu.F90:3996-4180): non-conservative viscous form
// (conservative_viscous = 0, calorically perfect gas)
void Solver::visflx_nosensor() {
  const int lmax = s.visc_order / 2;
  const double prandtl = s.prandtl;
  const double* c1 = s.coeff_deriv1[lmax - 1];
  const double* c2 = s.coeff_deriv2[lmax - 1];
  par_for(1, nz, [&](int k) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double uu = A(i, j, k, 2), vv = A(i, j, k, 3), ww = A(i, j, k, 4), tt = A(i, j, k, 6),
                     mu = A(i, j, k, 7);
        double ux = 0, vx = 0, wx = 0, tx = 0, mux = 0;
        double uy = 0, vy = 0, wy = 0, ty = 0, muy = 0;
        double uz = 0, vz = 0, wz = 0, tz = 0, muz = 0;
        double ulapx = c2[0] * uu, ulapy = ulapx, ulapz = ulapx;
        double vlapx = c2[0] * vv, vlapy = vlapx, vlapz = vlapx;
        double wlapx = c2[0] * ww, wlapy = wlapx, wlapz = wlapx;
        double tlapx = c2[0] * tt, tlapy = tlapx, tlapz = tlapx;
        for (int l = 1; l <= lmax; ++l) {
          const double ccl = c1[l - 1], clapl = c2[l];
          ux = ux + ccl * (A(i + l, j, k, 2) - A(i - l, j, k, 2));
          ulapx = ulapx + clapl * (A(i + l, j, k, 2) + A(i - l, j, k, 2));
          vx = vx + ccl * (A(i + l, j, k, 3) - A(i - l, j, k, 3));
          vlapx = vlapx + clapl * (A(i + l, j, k, 3) + A(i - l, j, k, 3));
          wx = wx + ccl * (A(i + l, j, k, 4) - A(i - l, j, k, 4));
          wlapx = wlapx + clapl * (A(i + l, j, k, 4) + A(i - l, j, k, 4));
          tx = tx + ccl * (A(i + l, j, k, 6) - A(i - l, j, k, 6));
          tlapx = tlapx + clapl * (A(i + l, j, k, 6) + A(i - l, j, k, 6));
          mux = mux + ccl * (A(i + l, j, k, 7) - A(i - l, j, k, 7));
        }
        for (int l = 1; l <= lmax; ++l) {
          const double ccl = c1[l - 1], clapl = c2[l];
          uy = uy + ccl * (A(i, j + l, k, 2) - A(i, j - l, k, 2));
          ulapy = ulapy + clapl * (A(i, j + l, k, 2) + A(i, j - l, k, 2));
          vy = vy + ccl * (A(i, j + l, k, 3) - A(i, j - l, k, 3));
          vlapy = vlapy + clapl * (A(i, j + l, k, 3) + A(i, j - l, k, 3));
          wy = wy + ccl * (A(i, j + l, k, 4) - A(i, j - l, k, 4));
          wlapy = wlapy + clapl * (A(i, j + l, k, 4) + A(i, j - l, k, 4));
          ty = ty + ccl * (A(i, j + l, k, 6) - A(i, j - l, k, 6));
          tlapy = tlapy + clapl * (A(i, j + l, k, 6) + A(i, j - l, k, 6));
          muy = muy + ccl * (A(i, j + l, k, 7) - A(i, j - l, k, 7));
        }
        for (int l = 1; l <= lmax; ++l) {
          const double ccl = c1[l - 1], clapl = c2[l];
          uz = uz + ccl * (A(i, j, k + l, 2) - A(i, j, k - l, 2));
          ulapz = ulapz + clapl * (A(i, j, k + l, 2) + A(i, j, k - l, 2));
          vz = vz + ccl * (A(i, j, k + l, 3) - A(i, j, k - l, 3));
          vlapz = vlapz + clapl * (A(i, j, k + l, 3) + A(i, j, k - l, 3));
          wz = wz + ccl * (A(i, j, k + l, 4) - A(i, j, k - l, 4));
          wlapz = wlapz + clapl * (A(i, j, k + l, 4) + A(i, j, k - l, 4));
          tz = tz + ccl * (A(i, j, k + l, 6) - A(i, j, k - l, 6));
          tlapz = tlapz + clapl * (A(i, j, k + l, 6) + A(i, j, k - l, 6));
          muz = muz + ccl * (A(i, j, k + l, 7) - A(i, j, k - l, 7));
        }
        const double dx = s.dcsidx[i - 1], dy = s.detady[j - 1], dz = s.dzitdz[k - 1];
        ux = ux * dx; vx = vx * dx; wx = wx * dx; tx = tx * dx; mux = mux * dx;
        uy = uy * dy; vy = vy * dy; wy = wy * dy; ty = ty * dy; muy = muy * dy;
        uz = uz * dz; vz = vz * dz; wz = wz * dz; tz = tz * dz; muz = muz * dz;
        const double sx2 = s.dcsidxs[i - 1], sy2 = s.detadys[j - 1], sz2 = s.dzitdzs[k - 1];
        const double x2 = s.dcsidx2[i - 1], y2 = s.detady2[j - 1], z2 = s.dzitdz2[k - 1];
        ulapx = ulapx * sx2 + ux * x2; vlapx = vlapx * sx2 + vx * x2;
        wlapx = wlapx * sx2 + wx * x2; tlapx = tlapx * sx2 + tx * x2;
        ulapy = ulapy * sy2 + uy * y2; vlapy = vlapy * sy2 + vy * y2;
        wlapy = wlapy * sy2 + wy * y2; tlapy = tlapy * sy2 + ty * y2;
        ulapz = ulapz * sz2 + uz * z2; vlapz = vlapz * sz2 + vz * z2;
        wlapz = wlapz * sz2 + wz * z2; tlapz = tlapz * sz2 + tz * z2;
        const double ulap = ulapx + ulapy + ulapz, vlap = vlapx + vlapy + vlapz;
        const double wlap = wlapx + wlapy + wlapz, tlap = tlapx + tlapy + tlapz;
        const double div = ux + vy + wz;
        const double div3l = div / 3.0;
        A(i, j, k, 10) = div3l;
        const double omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
        const double omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
        A(i, j, k, 9) = std::sqrt(omod2);
        const double sig11 = 2.0 * (ux - div3l), sig12 = uy + vx, sig13 = uz + wx;
        const double sig22 = 2.0 * (vy - div3l), sig23 = vz + wy, sig33 = 2.0 * (wz - div3l);
        const double sigx = mux * sig11 + muy * sig12 + muz * sig13 + mu * ulap;
        const double sigy = mux * sig12 + muy * sig22 + muz * sig23 + mu * vlap;
        const double sigz = mux * sig13 + muy * sig23 + muz * sig33 + mu * wlap;
        const double cploc = cploc_at(tt);
        const double sigqt = (mux * tx + muy * ty + muz * tz + mu * tlap) * cploc / prandtl;
        const double sigah = (sig11 * ux + sig12 * uy + sig13 * uz + sig12 * vx + sig22 * vy + sig23 * vz +
                              sig13 * wx + sig23 * wy + sig33 * wz) * mu;
        const double sigq = sigx * uu + sigy * vv + sigz * ww + sigah + sigqt;
        FL(i, j, k, 2) = FL(i, j, k, 2) - sigx;
        FL(i, j, k, 3) = FL(i, j, k, 3) - sigy;
        FL(i, j, k, 4) = FL(i, j, k, 4) - sigz;
        FL(i, j, k, 5) = FL(i, j, k, 5) - sigq;
        if (j == 1) {
          wallprop[(0 * sz + k + ng - 1) * sx + i + ng - 1] = mu * uy;
          wallprop[(1 * sz + k + ng - 1) * sx + i + ng - 1] = mu * wy;
          wallprop[(2 * sz + k + ng - 1) * sx + i + ng - 1] = mu * ty * cploc / prandtl;
        }
      }
  });
}

// The Ducros sensor that visflx_subroutine (kernels_cpu.F90:3598-3777) stores at run()'s start for
// conservative_viscous = 0 (its flux contribution is discarded by zero_flux): visc_order
// derivatives, theta from div and omega directly.
void Solver::sensor_visc_order() {
  const int lmax = s.visc_order / 2;
  const double* c1 = s.coeff_deriv1[lmax - 1];
  const double u0 = s.u0, l0 = s.l0;
  par_for(1, nz, [&](int k) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double ux = 0, vx = 0, wx = 0, uy = 0, vy = 0, wy = 0, uz = 0, vz = 0, wz = 0;
        for (int l = 1; l <= lmax; ++l) {
          const double ccl = c1[l - 1];
          ux = ux + ccl * (A(i + l, j, k, 2) - A(i - l, j, k, 2));
          vx = vx + ccl * (A(i + l, j, k, 3) - A(i - l, j, k, 3));
          wx = wx + ccl * (A(i + l, j, k, 4) - A(i - l, j, k, 4));
          uy = uy + ccl * (A(i, j + l, k, 2) - A(i, j - l, k, 2));
          vy = vy + ccl * (A(i, j + l, k, 3) - A(i, j - l, k, 3));
          wy = wy + ccl * (A(i, j + l, k, 4) - A(i, j - l, k, 4));
          uz = uz + ccl * (A(i, j, k + l, 2) - A(i, j, k - l, 2));
          vz = vz + ccl * (A(i, j, k + l, 3) - A(i, j, k - l, 3));
          wz = wz + ccl * (A(i, j, k + l, 4) - A(i, j, k - l, 4));
        }
        const double dx = s.dcsidx[i - 1], dy = s.detady[j - 1], dz = s.dzitdz[k - 1];
        ux = ux * dx; vx = vx * dx; wx = wx * dx;
        uy = uy * dy; vy = vy * dy; wy = wy * dy;
        uz = uz * dz; vz = vz * dz; wz = wz * dz;
        const double div = ux + vy + wz;
        const double omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
        const double omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
        const double t = std::max(-div / std::sqrt(omod2 + div * div + (u0 / l0) * (u0 / l0)), 0.0);
        A(i, j, k, 8) = t * t;
      }
  });
}

// visflx_div_subroutine (kernels_cpu.F90:3484-3532)
void Solver::visflx_div() {
  const int lmax = s.visc_order / 2;
  const double* c1 = s.coeff_deriv1[lmax - 1];
  par_for(1, nz, [&](int k) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double uu = A(i, j, k, 2), vv = A(i, j, k, 3), ww = A(i, j, k, 4), mu = A(i, j, k, 7);
        double divx3l = 0, divy3l = 0, divz3l = 0;
        for (int l = 1; l <= lmax; ++l) {
          const double ccl = c1[l - 1];
          divx3l = divx3l + ccl * (A(i + l, j, k, 10) - A(i - l, j, k, 10));
          divy3l = divy3l + ccl * (A(i, j + l, k, 10) - A(i, j - l, k, 10));
          divz3l = divz3l + ccl * (A(i, j, k + l, 10) - A(i, j, k - l, 10));
        }
        divx3l = divx3l * s.dcsidx[i - 1];
        divy3l = divy3l * s.detady[j - 1];
        divz3l = divz3l * s.dzitdz[k - 1];
        const double sigx = mu * divx3l, sigy = mu * divy3l, sigz = mu * divz3l;
        const double sigq = sigx * uu + sigy * vv + sigz * ww;
        FL(i, j, k, 2) = FL(i, j, k, 2) - sigx;
        FL(i, j, k, 3) = FL(i, j, k, 3) - sigy;
        FL(i, j, k, 4) = FL(i, j, k, 4) - sigz;
        FL(i, j, k, 5) = FL(i, j, k, 5) - sigq;
      }
  });
}

// bc_nr (singleideal_cpu.F90:1001-1062) with bc_nr_lat_x_kernel / bc_nr_lat_y_kernel
// (kernels_cpu.F90:5169-5283, 5420-5540): characteristic correction of fl at the boundary
// points of the faces with a non-reflecting type (1: outgoing waves only; 2: incoming waves from
// the ghost point; 3: incoming waves towards the free stream; 6: the acoustic reflection of
// type-6), one-sided second-order normal derivatives of w.
void Solver::bc_nr() {
  const double rgas0 = s.rgas0;
  for (int ilat = 1; ilat <= 4; ++ilat) {
    const int nr_type = s.bctags_nr[ilat - 1];
    if (nr_type <= 0) continue;
    const int dir = (ilat - 1) / 2;            // 0 x, 1 y
    const int start_or_end = (ilat - 1) % 2 + 1;
    const int sgn = start_or_end == 1 ? 1 : -1;
    const int n1 = dir == 0 ? ny : nx;
    for (int k = 1; k <= nz; ++k)
      for (int t = 1; t <= n1; ++t) {
        const int i = dir == 0 ? (start_or_end == 1 ? 1 : nx) : t;
        const int j = dir == 1 ? (start_or_end == 1 ? 1 : ny) : t;
        const double c_one[3] = {-1.5, 2.0, -0.5};
        double dw_dn[5], dw_dn_outer[5];
        for (int m = 0; m < 5; ++m) {
          dw_dn[m] = 0.0;
          for (int l = 1; l <= 3; ++l) {
            const int o = sgn * (l - 1);
            dw_dn[m] = dw_dn[m] + sgn * c_one[l - 1] * W(i + (dir == 0 ? o : 0), j + (dir == 1 ? o : 0), k, m);
          }
          double w_target = 0.0;
          if (nr_type == 2) w_target = W(i - (dir == 0 ? sgn : 0), j - (dir == 1 ? sgn : 0), k, m);
          else if (nr_type == 3) w_target = s.winf[m];
          dw_dn_outer[m] = sgn * (W(i, j, k, m) - w_target);
        }
        const double rho = A(i, j, k, 1), uu = A(i, j, k, 2), vv = A(i, j, k, 3), ww = A(i, j, k, 4);
        const double h = A(i, j, k, 5), tt = A(i, j, k, 6);
        const double gamloc = gamloc_at(tt);
        const double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        const double cc = gamloc * tt * rgas0;
        const double c = std::sqrt(cc);
        const double ci = 1.0 / c;
        const double p_rho = tt * rgas0;
        const double p_e = rho * (gamloc - 1.0);
        const double etot = h - tt * rgas0;
        const double b3 = etot - rho * p_rho / p_e;
        const double b2 = p_e / (rho * cc);
        const double b1 = p_rho / cc - b2 * (etot - 2.0 * qq);
        // eigenvectors_x / eigenvectors_y (kernels_cpu.F90:2728-2782, 2842-2896): el(var, char), er(char, var)
        double el[5][5], er[5][5];
        const double vn = dir == 0 ? uu : vv;
        const double vt1 = dir == 0 ? vv : uu;  // first tangential velocity (v for x, u for y)
        const int t1 = dir == 0 ? 2 : 1;        // its conserved slot
        const int nslot = dir == 0 ? 1 : 2;
        for (int a = 0; a < 5; ++a)
          for (int b = 0; b < 5; ++b) el[a][b] = er[a][b] = 0.0;
        const double vel[3] = {uu, vv, ww};
        el[0][0] = 0.5 * (b1 + vn * ci);
        for (int d = 0; d < 3; ++d) el[1 + d][0] = -0.5 * (b2 * vel[d] + (1 + d == nslot ? ci : 0.0));
        el[4][0] = 0.5 * b2;
        el[0][1] = 1.0 - b1;
        for (int d = 0; d < 3; ++d) el[1 + d][1] = b2 * vel[d];
        el[4][1] = -b2;
        el[0][2] = -vt1; el[t1][2] = 1.0;
        el[0][3] = -ww; el[3][3] = 1.0;
        el[0][4] = 0.5 * (b1 - vn * ci);
        for (int d = 0; d < 3; ++d) el[1 + d][4] = -0.5 * (b2 * vel[d] - (1 + d == nslot ? ci : 0.0));
        el[4][4] = 0.5 * b2;
        er[0][0] = 1.0; er[1][0] = 1.0; er[4][0] = 1.0;
        for (int d = 0; d < 3; ++d) {
          er[0][1 + d] = vel[d] - (1 + d == nslot ? c : 0.0);
          er[1][1 + d] = vel[d];
          er[4][1 + d] = vel[d] + (1 + d == nslot ? c : 0.0);
        }
        er[2][1] = er[2][2] = er[2][3] = 0.0;
        er[3][1] = er[3][2] = er[3][3] = 0.0;
        er[2][t1] = 1.0;
        er[3][3] = 1.0;
        er[0][4] = h - vn * c;
        er[1][4] = b3;
        er[2][4] = vt1;
        er[3][4] = ww;
        er[4][4] = h + vn * c;
        double dwc_dn[5], dwc_dn_outer[5], ev[5];
        for (int m = 0; m < 5; ++m) {
          dwc_dn[m] = 0.0;
          dwc_dn_outer[m] = 0.0;
          for (int mm = 0; mm < 5; ++mm) {
            dwc_dn[m] = dwc_dn[m] + el[mm][m] * dw_dn[mm];
            dwc_dn_outer[m] = dwc_dn_outer[m] + el[mm][m] * dw_dn_outer[mm];
          }
        }
        ev[0] = vn - c; ev[1] = vn; ev[2] = ev[1]; ev[3] = ev[1]; ev[4] = vn + c;
        if (nr_type == 1)
          for (int l = 0; l < 5; ++l) ev[l] = start_or_end == 1 ? std::min(ev[l], 0.0) : std::max(ev[l], 0.0);
        if (nr_type == 2 || nr_type == 3)
          for (int m = 0; m < 5; ++m)
            if (sgn * ev[m] > 0.0) dwc_dn[m] = dwc_dn_outer[m];
        for (int m = 0; m < 5; ++m) dwc_dn[m] = ev[m] * dwc_dn[m];
        if (nr_type == 6) {
          dwc_dn[1] = dwc_dn[2] = dwc_dn[3] = 0.0;
          if (start_or_end == 1) dwc_dn[4] = dwc_dn[0]; else dwc_dn[0] = dwc_dn[4];
        }
        const double met = dir == 0 ? s.dcsidx[i - 1] : s.detady[j - 1];
        for (int m = 0; m < 5; ++m) {
          double df = 0.0;
          for (int mm = 0; mm < 5; ++mm) df = df + er[mm][m] * dwc_dn[mm];
          FL(i, j, k, m + 1) = FL(i, j, k, m + 1) + df * met;
        }
      }
  }
}

// force_rhs (singleideal_cpu.F90:845-889) with force_rhs_1/2 (kernels_cpu.F90:3157-3193, 3092-3116).
// The oracle sums each k-plane sequentially and then the planes in k order.
void Solver::force_rhs() {
  std::vector<double> part(static_cast<size_t>(nz) * 5, 0.0);
  par_for(1, nz, [&](int k) {
    double b1 = 0, b2 = 0, b3 = 0, b4 = 0, b5 = 0;
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double dy = s.ynl[j] - s.ynl[j - 1];
        b1 = b1 + FLN(i, j, k, 1) * dy;
        b2 = b2 + FLN(i, j, k, 2) * dy;
        b3 = b3 + W(i, j, k, 0) * dy;
        b4 = b4 + W(i, j, k, 1) * dy;
        b5 = b5 + W(i, j, k, 1) * dy * A(i, j, k, 6);
      }
    double* p = &part[(k - 1) * 5];
    p[0] = b1; p[1] = b2; p[2] = b3; p[3] = b4; p[4] = b5;
  });
  double bulk[5] = {0, 0, 0, 0, 0};
  for (int k = 0; k < nz; ++k)
    for (int m = 0; m < 5; ++m) bulk[m] = bulk[m] + part[k * 5 + m];
  for (int m = 0; m < 5; ++m) bulk[m] = bulk[m] / s.volchan;
  dpdx = dpdx + bulk[1];
  rhobulk = bulk[2];
  ubulk = bulk[3] / rhobulk;
  tbulk = bulk[4] / rhobulk / ubulk;
  const double bulk_1 = bulk[0], bulk_2 = bulk[1];
  par_for(1, nz, [&](int k) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double uu = A(i, j, k, 2);
        FLN(i, j, k, 1) = FLN(i, j, k, 1) - bulk_1;
        FLN(i, j, k, 2) = FLN(i, j, k, 2) - bulk_2;
        FLN(i, j, k, 5) = FLN(i, j, k, 5) - uu * bulk_2;
      }
  });
}

// force_var (singleideal_cpu.F90:890-933) with force_var_1/2 (kernels_cpu.F90:3241-3314)
void Solver::force_var() {
  if (!(s.theta_wall >= -1.0)) return;
  std::vector<double> part(static_cast<size_t>(nz), 0.0);
  par_for(1, nz, [&](int k) {
    double b5 = 0;
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double dy = s.ynl[j] - s.ynl[j - 1];
        double rho = W(i, j, k, 0), rhou = W(i, j, k, 1), rhov = W(i, j, k, 2), rhow = W(i, j, k, 3),
               rhoe = W(i, j, k, 4);
        double ri = 1.0 / rho;
        double uu = rhou * ri, vv = rhov * ri, ww = rhow * ri;
        double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        double ee = rhoe / rho - qq;
        double tt = temp_from_e(ee, A(i, j, k, 6));
        A(i, j, k, 6) = tt;
        b5 = b5 + rhou * tt * dy;
      }
    part[k - 1] = b5;
  });
  double bulkt = 0;
  for (int k = 0; k < nz; ++k) bulkt = bulkt + part[k];
  double bulktg = bulkt / s.volchan;
  bulktg = bulktg / rhobulk / ubulk;
  double tbdiff = s.t_bulk_target - bulktg;
  par_for(1, nz, [&](int k) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double rho = W(i, j, k, 0), rhou = W(i, j, k, 1), rhov = W(i, j, k, 2), rhow = W(i, j, k, 3);
        double tt = A(i, j, k, 6);
        double ttnew = tt + tbdiff;
        double ee = e_from_temp(ttnew);
        W(i, j, k, 4) = rho * ee + 0.5 * (rhou * rhou + rhov * rhov + rhow * rhow) / rho;
      }
  });
}

// rk_sync (singleideal_cpu.F90:332-409), mode_async = 0
void Solver::rk_sync() {
  if (s.channel_case) dpdx = 0.0;
  for (int istep = 1; istep <= s.nrk; ++istep) {
    const double rhodt = s.rhork[istep - 1] * dt;
    const double gamdt = s.gamrk[istep - 1] * dt;
    // init_flux_subroutine (kernels_cpu.F90:29-47)
    for (size_t q = 0; q < fl.size(); ++q) {
      fln[q] = -rhodt * fl[q];
      fl[q] = 0.0;
    }
    bcswap();
    compute_aux(1, 1);
    euler(0);
    if (s.conservative_viscous == 1) {
      visflx_reduced_ord2(0);
      visflx_faces();
    } else {
      visflx_nosensor();
    }
    bcextr_var(10);
    bcswap_var(10);
    euler(1);
    euler(2);
    if (s.recyc) draw_random_plane();
    if (istep == 3) {
      sensor();
      bcswap_var(8);
    }
    if (s.conservative_viscous == 1)
      visflx_div_ord2();
    else
      visflx_div();
    bc_nr();
    // update_flux_subroutine (kernels_cpu.F90:3400-3418)
    for (size_t q = 0; q < fl.size(); ++q) fln[q] = fln[q] - gamdt * fl[q];
    if (s.channel_case) force_rhs();
    // update_field_subroutine (kernels_cpu.F90:3422-3442)
    par_for(1, nz, [&](int k) {
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i)
          for (int m = 0; m < 5; ++m) W(i, j, k, m) = W(i, j, k, m) + FLN(i, j, k, m + 1);
    });
    if (s.channel_case) force_var();
    update_ghost(0);
  }
}

// compute_dt (singleideal_cpu.F90:1476-1517), compute_dt_subroutine (kernels_cpu.F90:6814-6880)
void Solver::compute_dt() {
  if (s.cfl < 0) {
    dt = -s.cfl;
    return;
  }
  std::vector<double> part(static_cast<size_t>(nz) * 9, 0.0);
  const double rgas0 = s.rgas0, prandtl = s.prandtl;
  par_for(1, nz, [&](int k) {
    double mx[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double rho = W(i, j, k, 0);
        double ri = 1.0 / rho;
        double uu = A(i, j, k, 2), vv = A(i, j, k, 3), ww = A(i, j, k, 4), tt = A(i, j, k, 6), mu = A(i, j, k, 7);
        double nu = ri * mu;
        double k_over_rhocp = nu / prandtl;
        double c = std::sqrt(gamloc_at(tt) * rgas0 * tt);
        double v[9] = {(std::fabs(uu) + c) * s.dcsidx[i - 1], (std::fabs(vv) + c) * s.detady[j - 1],
                       (std::fabs(ww) + c) * s.dzitdz[k - 1], nu * s.dcsidxs[i - 1],
                       nu * s.detadys[j - 1], nu * s.dzitdzs[k - 1],
                       k_over_rhocp * s.dcsidxs[i - 1], k_over_rhocp * s.detadys[j - 1],
                       k_over_rhocp * s.dzitdzs[k - 1]};
        for (int q = 0; q < 9; ++q) mx[q] = std::max(mx[q], v[q]);
      }
    for (int q = 0; q < 9; ++q) part[(k - 1) * 9 + q] = mx[q];
  });
  double dtinv_max = 0.0;
  for (size_t q = 0; q < part.size(); ++q) dtinv_max = std::max(dtinv_max, part[q]);
  double dt_min = 1.0 / dtinv_max;
  dt = s.cfl * dt_min;
}

// compute_residual (singleideal_cpu.F90:1339-1364), kernels_cpu.F90:6682-6701, 6765-6810
void Solver::compute_residual() {
  std::vector<double> part(static_cast<size_t>(nz), 0.0);
  par_for(1, nz, [&](int k) {
    double r = 0;
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double q = FLN(i, j, k, 2) / dt;
        r = r + q * q;
      }
    part[k - 1] = r;
  });
  double res = 0;
  for (int k = 0; k < nz; ++k) res = res + part[k];
  double restemp = static_cast<double>(nx) * static_cast<double>(ny) * static_cast<double>(nz);
  residual_rhou = std::sqrt(res / restemp);
  rhomin = std::numeric_limits<double>::max();
  rhomax = -100.0;
  tmin = rhomin; tmax = -100.0; pmin = rhomin; pmax = -100.0;
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double rho = A(i, j, k, 1), tt = A(i, j, k, 6);
        double pp = rho * tt * s.rgas0;
        rhomin = std::min(rhomin, rho); rhomax = std::max(rhomax, rho);
        tmin = std::min(tmin, tt); tmax = std::max(tmax, tt);
        pmin = std::min(pmin, pp); pmax = std::max(pmax, pp);
      }
}

void Solver::init_run() {
  update_ghost(1);
  compute_aux(1, 1);
  if (s.conservative_viscous == 1)
    visflx_reduced_ord2(1);
  else
    sensor_visc_order();
  bcswap_var(8);
  std::fill(fl.begin(), fl.end(), 0.0);
  compute_dt();
}

void Solver::step() {
  icyc = icyc + 1;
  if (s.cfl > 0 && (icyc - s.icyc0) % s.iter_dt_recompute == 0) {
    compute_aux(1, 0);
    compute_dt();
  }
  rk_sync();
  const bool print = ((icyc - s.icyc0) % s.print_control) == 0;
  if (print) compute_residual();
  time = time + dt;
  if (print) rows.push_back(progress_row());
}

void Solver::run(int nsteps) {
  for (int n = 0; n < nsteps; ++n) step();
}

// print_progress (singleideal_cpu.F90:1695-1732), channel row
// compute_stats (singleideal.F90:2003-2179) on one block (the z all-reduce is the identity):
// visc_order velocity derivatives from w including its ghost layers as the step left them, T and
// mu from w_aux(6), w_aux(7); the 70 per-point quantities are summed over k for every (i,j), divided
// by nzmax and averaged in time with the itav samples already in w_stat.
void Solver::compute_stats(int itav) {
  const int nv = NV_STAT;
  const int lmax = s.visc_order / 2;
  if (w_stat.empty()) w_stat.assign(static_cast<size_t>(nv) * nx * ny, 0.0);
  w_stat_z.assign(static_cast<size_t>(nv) * nx * ny, 0.0);
  const double rgas0 = s.rgas0;
  par_for(1, ny, [&](int j) {
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i) {
        double ux = 0, vx = 0, wx = 0, uy = 0, vy = 0, wy = 0, uz = 0, vz = 0, wz = 0;
        for (int l = 1; l <= lmax; ++l) {
          const double ccl = s.coeff_deriv1[lmax - 1][l - 1];
          ux = ux + ccl * (W(i + l, j, k, 1) / W(i + l, j, k, 0) - W(i - l, j, k, 1) / W(i - l, j, k, 0));
          vx = vx + ccl * (W(i + l, j, k, 2) / W(i + l, j, k, 0) - W(i - l, j, k, 2) / W(i - l, j, k, 0));
          wx = wx + ccl * (W(i + l, j, k, 3) / W(i + l, j, k, 0) - W(i - l, j, k, 3) / W(i - l, j, k, 0));
          uy = uy + ccl * (W(i, j + l, k, 1) / W(i, j + l, k, 0) - W(i, j - l, k, 1) / W(i, j - l, k, 0));
          vy = vy + ccl * (W(i, j + l, k, 2) / W(i, j + l, k, 0) - W(i, j - l, k, 2) / W(i, j - l, k, 0));
          wy = wy + ccl * (W(i, j + l, k, 3) / W(i, j + l, k, 0) - W(i, j - l, k, 3) / W(i, j - l, k, 0));
          uz = uz + ccl * (W(i, j, k + l, 1) / W(i, j, k + l, 0) - W(i, j, k - l, 1) / W(i, j, k - l, 0));
          vz = vz + ccl * (W(i, j, k + l, 2) / W(i, j, k + l, 0) - W(i, j, k - l, 2) / W(i, j, k - l, 0));
          wz = wz + ccl * (W(i, j, k + l, 3) / W(i, j, k + l, 0) - W(i, j, k - l, 3) / W(i, j, k - l, 0));
        }
        const double dx = s.dcsidx[i - 1], dy = s.detady[j - 1], dz = s.dzitdz[k - 1];
        ux = ux * dx; vx = vx * dx; wx = wx * dx;
        uy = uy * dy; vy = vy * dy; wy = wy * dy;
        uz = uz * dz; vz = vz * dz; wz = wz * dz;
        const double omx = wy - vz, omy = uz - wx, omz = vx - uy;
        const double rho = W(i, j, k, 0), rhou = W(i, j, k, 1), rhov = W(i, j, k, 2), rhow = W(i, j, k, 3);
        const double ri = 1.0 / rho;
        const double uu = rhou * ri, vv = rhov * ri, ww = rhow * ri;
        const double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        const double tt = A(i, j, k, 6);
        const double pp = rho * rgas0 * tt;
        const double mu = A(i, j, k, 7);
        const double nu = mu / rho;
        // get_gamloc (singleideal.F90:4752-4771)
        const double gamloc = gamloc_at(tt);
        const double cploc = gamloc / (gamloc - 1.0) * rgas0;
        const double c = std::sqrt(gamloc * rgas0 * tt);
        const double machlocal = std::sqrt(2.0 * qq) / c;
        const double t_tot = tt + qq * (gamloc - 1.0) / gamloc;
        const double rho2 = rho * rho, uu2 = uu * uu, vv2 = vv * vv, ww2 = ww * ww, pp2 = pp * pp, tt2 = tt * tt;
        const double divl = ux + vy + wz;
        const double div3l = divl / 3.0;
        double sg[3][3];
        sg[0][0] = 2.0 * (ux - div3l);
        sg[0][1] = uy + vx;
        sg[0][2] = uz + wx;
        sg[1][0] = sg[0][1];
        sg[1][1] = 2.0 * (vy - div3l);
        sg[1][2] = vz + wy;
        sg[2][0] = sg[0][2];
        sg[2][1] = sg[1][2];
        sg[2][2] = 2.0 * (wz - div3l);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) sg[a][b] = sg[a][b] * mu;
        const double v[NV_STAT] = {
            rho, uu, vv, ww, pp, tt, rho2, uu2, vv2, ww2, pp2, tt2, rhou, rhov, rhow,
            rhou * uu, rhov * vv, rhow * ww, rhou * vv, mu, nu, omx * omx, omy * omy, omz * omz,
            rho * tt, rho * tt2, t_tot, rho * t_tot, t_tot * t_tot, rhou * tt, rhov * tt, rhow * tt,
            machlocal, machlocal * machlocal, rhou * uu2, rhov * uu2, rhou * vv2, rhov * vv2, rhou * ww2,
            rhov * ww2, pp * uu, pp * vv, sg[0][0], sg[0][1], sg[0][2], sg[1][1], sg[1][2], sg[2][2],
            sg[0][0] * uu, sg[0][1] * uu, sg[1][0] * vv, sg[1][1] * vv, sg[2][0] * ww, sg[2][1] * ww,
            sg[0][0] * vv, sg[0][1] * vv, sg[0][0] * ux, sg[1][0] * vx, sg[2][0] * wx, sg[0][0] * vx,
            pp * ux, pp * vy, pp * wz, pp * (uy + vx), divl * divl, rho * tt2 * tt, rho * tt2 * tt2,
            rhou * uu2 * uu, cploc, gamloc};
        double* acc = &w_stat_z[(static_cast<size_t>(j - 1) * nx + (i - 1)) * nv];
        for (int l = 0; l < nv; ++l) acc[l] = acc[l] + v[l];
        // statistics 55-60 add several terms, left to right as the source line reads
        acc[54] = acc[54] + sg[1][0] * uu;
        acc[55] = acc[55] + sg[1][1] * uu;
        acc[56] = acc[56] + sg[0][1] * uy;
        acc[56] = acc[56] + sg[0][2] * uz;
        acc[57] = acc[57] + sg[1][1] * vy;
        acc[57] = acc[57] + sg[1][2] * vz;
        acc[58] = acc[58] + sg[2][1] * wy;
        acc[58] = acc[58] + sg[2][2] * wz;
        acc[59] = acc[59] + sg[0][1] * (ux + vy);
        acc[59] = acc[59] + sg[1][1] * uy;
        acc[59] = acc[59] + sg[0][2] * vz;
        acc[59] = acc[59] + sg[1][2] * uz;
      }
  });
  const double nzmax = static_cast<double>(s.nzmax);
  const double rav = static_cast<double>(itav);
  for (size_t q = 0; q < w_stat_z.size(); ++q) {
    w_stat_z[q] = w_stat_z[q] / nzmax;
    w_stat[q] = w_stat[q] * rav + w_stat_z[q];
    w_stat[q] = w_stat[q] / (rav + 1.0);
  }
}

// compute_stats_3d (singleideal.F90:2513-2543): 14 point statistics averaged in time
void Solver::compute_stats_3d(int itav) {
  const int nv = NV_STAT_3D;
  if (w_stat_3d.empty()) w_stat_3d.assign(static_cast<size_t>(nv) * nint_(), 0.0);
  const double rav = static_cast<double>(itav);
  par_for(1, nz, [&](int k) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double r = W(i, j, k, 0), ru = W(i, j, k, 1), rv = W(i, j, k, 2), rw = W(i, j, k, 3);
        const double t = A(i, j, k, 6);
        const double v[NV_STAT_3D] = {r,           ru,          rv,          rw,          r * t,
                                      r * r,       ru * ru / r, rv * rv / r, rw * rw / r, ru * rv / r,
                                      ru * rw / r, rv * rw / r, r * (t * t), (r * t) * (r * t)};
        double* o = &w_stat_3d[ii(i, j, k) * nv];
        for (int l = 0; l < nv; ++l) o[l] = o[l] * rav + v[l];
      }
  });
  for (double& x : w_stat_3d) x = x / (rav + 1.0);
}

ProgressRow Solver::progress_row() const {
  ProgressRow r;
  r.icyc = icyc;
  r.dt = dt;
  r.time = time;
  double res = residual_rhou / (s.u0 * s.u0) / s.rho0 * s.l0;
  double dp = dpdx / (s.u0 * s.u0) / s.rho0 * s.l0;
  r.residual_rhou = res;
  r.dpdx_over_dt = -dp / dt;
  r.rhobulk = rhobulk; r.ubulk = ubulk; r.tbulk = tbulk;
  r.rhomin = rhomin; r.rhomax = rhomax; r.tmin = tmin; r.tmax = tmax; r.pmin = pmin; r.pmax = pmax;
  return r;
}

}  // namespace streams_oracle
