// Shared device-side definitions of the B200 backend: the per-context geometry and parameter
// block (passed by value to every kernel), array indexing, thermodynamics of the calorically
// perfect gas, and deterministic block reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sb200 {

constexpr int NV = 5;
constexpr int MAX_CP = 12;           // cp(T) polynomial coefficients (STREAMS_B200_MAX_CP)
constexpr double TOL_ITER_NR = 1e-12;  // Newton tolerance of the temperature (tol_iter_nr)

// Number of FP64 reduction slots produced per block by the stage kernels.
constexpr int NRED_RHS = 5;   // force_rhs: sum fln1*dy, fln2*dy, rho*dy, rhou*dy, rhou*T*dy
constexpr int NRED_UPD = 8;   // force_var sum rhou*T*dy, residual sum, rho/T/p min and max
// running statistics per (i,j) column and per cell (nv_stat, nv_stat_3d of singleideal.F90:474-478)
constexpr int NV_STAT = 70;
constexpr int NV_STAT_3D = 14;
constexpr int WSAMPLE = 16;  // WENO face sample: every 16th plane

struct Geom {
  // block sizes and padded strides (ghosted arrays: index (i,j,k), i in 1-ng..nx+ng)
  int nx, ny, nz, ng;
  int sx, sy, sz;
  long long nvol;  // sx*sy*sz: stride between variables of a ghosted array
  long long nint;  // nx*ny*nz: stride between variables of an interior array
  // one-dimensional grid (device pointers, already offset so that x[i] is x(i) of the reference)
  const double* x;
  // per line of each direction, index 1..n: 1/(x(i+1)-x(i-1)) in FP64 and in FP32 and
  // 2/(x(i+1)-x(i-1)) in FP64, the grid divisions of the viscous pass (the same IEEE quotients)
  const double* vrl[3];
  const float* vrlf[3];
  const double* vhl[3];
  const double* y;
  const double* z;
  const double* yn;       // yn[j], j = 1..ny+1
  const double* dcsidx;   // [i], i = 1..nx
  const double* detady;
  const double* dzitdz;
  const double* dcsidxs;
  const double* detadys;
  const double* dzitdzs;
  const int* epx;         // ep_ord_change along x, [i] for faces i = 0..nx
  const int* epy;
  const int* epz;
  double coeff[4][4];     // coeff_deriv1(l, lmax) at [lmax-1][l-1]
  // non-conservative viscous form (conservative_viscous = 0)
  int conservative_viscous;
  const double* dcsidx2;  // [i], i = 1..nx (second-derivative metric terms)
  const double* detady2;
  const double* dzitdz2;
  double coeff2[4][5];    // coeff_deriv2(l, lmax) at [lmax-1][l], l = 0..4
  // boundary handling
  int periodic[3];
  int wall_ymin, wall_ymax;  // staggered isothermal walls (ghosts mirrored on the fly)
  int bctag[6], nr[6];       // boundary tags and non-reflecting types per face
  double winf[5], p0;        // free stream (non-reflecting type 3), reference pressure
  double xshock_imp, shock_angle, tanhfacs, winf_past_shock[5];  // impinging shock (bctag[3] = 7)
  // recycling-rescaling inflow (bctag[0] = 10)
  int recyc, i_recyc, jbl_inflow;
  double betarecyc, rand_scale;
  const double* wmean_inflow;  // [(m-1)*ny + (j-1)]*ng + (i-1), wmean(1-i, j, m)
  const double* yplus_inflow;  // [j], j = 1-ng..ny+ng
  const double* eta_inflow;
  const double* yplus_recyc;
  const double* eta_recyc;
  const double* weta_inflow;   // [j], j = 1..ny
  const int* map_j_inn;        // [j], j = 1..ny
  const int* map_j_out;
  int fzf[6];                // force_zero_flux
  int eul_imin, eul_imax, eul_jmin, eul_jmax, eul_kmin, eul_kmax;
  // numerics
  int lmax_base, nkeep, weno_scheme, weno_version;
  int flux_splitting;  // 0: characteristic WENO, 1: component-wise (Rusanov) WENO
  double sensor_threshold;
  // fluid
  int visc_model;
  double mu0, t0, rgas0, rho0, u0, l0, sutherland_s, t_ref_dim, vtexp, prandtl;
  double cp0, cv0, cp_last, cv_last, gamloc;
  // constants of the WENO faces formed once on the host: gamma - 1 and 1/(gamma - 1) of the
  // calorically perfect gas, the smoothness-indicator scales 1/(rho0^2 u0^2) and
  // 1/(rho0^2 u0^4) of wenorec_1d (kernels_cpu.F90:2539-2546) and 1/(rho0^2 u0^6)
  double gm1, rgm1, wbs_a, wbs_b, wbs_c;
  // thermally perfect gas (calorically_perfect = 0): cp(T) = sum of cpc[l - cp_l] (T/t0)^l for
  // l = cp_l..cp_r, cv likewise (set_fluid_prop's cp_coeff / cv_coeff, times rgas0)
  int calorically_perfect, cp_l, cp_r;
  const double* cpc;  // device arrays of MAX_CP values (a kernel-parameter array indexed at run
  const double* cvc;  // time would be copied to local memory)
  double t_wall;
  // channel forcing
  int channel_case, force_var;
  double volchan, t_bulk_target;
  // arithmetic of the flux and viscous passes: 0 FP64, 1 mixed (FP32 fluxes, FP64 state)
  int precision;
  // WENO faces computed apart from the hybrid passes: per direction the list of the faces whose
  // stencil sees the sensor (rebuilt at stage 1, the sensor being fixed for a step) and one face
  // buffer of their fluxes (planes of nwface values: 5 in FP64, 5 high + 5 low parts in FP32)
  void* wface;
  long long nwface;
  unsigned int* wlist[3];
  unsigned int* wcount;  // [3]
  // ghosted flags sensor > threshold of the step (periodic ghosts copied, other ghosts 0)
  unsigned char* wbits;
  // a direction's hybrid pass reads the buffer when its list holds at most wthr[d] faces and
  // computes its WENO faces itself otherwise (wthr = weno_split_frac x the direction's faces)
  unsigned int wthr[3];
  // the lists are built only when a sample of the faces (every WSAMPLE-th plane of the list
  // kernels' third grid index) holds at most wthr_s[d] WENO faces (wcount[4 + d] on the device)
  unsigned int wthr_s[3];
  int wsplit_on;  // weno_split_frac > 0: the lists, face kernels and split forms are launched
  double weno_split_frac;  // host side
  // launch shape of the y/z march passes (host side only): the lines are cut into segments so
  // that about march_threads threads run, each segment at least march_minseg cells long
  long long march_threads;
  int march_minseg;
};
// State of the crandom sequence on the device (glibc's additive feedback generator, continued
// from the host set-up's draws): the 34-word ring and the position of the next word.
struct RngState {
  unsigned int ring[34];
  long long pos;
};

// smallest march segment length a context may be tuned to (sizes the reduction scratch)
constexpr int MARCH_MINSEG_MIN = 4;

__host__ __device__ __forceinline__ long long gidx(const Geom& g, int i, int j, int k) {
  return ((long long)(k + g.ng - 1) * g.sy + (j + g.ng - 1)) * g.sx + (i + g.ng - 1);
}
__host__ __device__ __forceinline__ long long iidx(const Geom& g, int i, int j, int k) {
  return ((long long)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1);
}
// Interior cell (i, j, k) of the interior index q (i fastest).  Interior counts stay below 2^32
// (no direction may have 2^32 faces, checked at context creation), so the divisions are 32-bit
// rather than the emulated 64-bit ones.
__device__ __forceinline__ void cell_of(const Geom& g, long long q, int& i, int& j, int& k) {
  const unsigned u = (unsigned)q, nx = (unsigned)g.nx, ny = (unsigned)g.ny;
  const unsigned r = u / nx;
  i = (int)(u - r * nx) + 1;
  const unsigned kk = r / ny;
  j = (int)(r - kk * ny) + 1;
  k = (int)kk + 1;
}

// Device-resident scalars of a context (one cache line group).
struct Scalars {
  double dt;
  double time;
  double dpdx;
  double rhobulk, ubulk, tbulk;
  double tbdiff;       // pending force_var energy shift (applied by the next aux pass)
  double bulk[5];      // last force_rhs bulk values (divided by volchan)
  double residual_sum; // sum of (fln_2/dt)^2 of the last stage 3
  double rhomin, rhomax, tmin, tmax, pmin, pmax;
  int pending_shift;   // 1 when tbdiff has not been applied to w yet
  int nan_flag;
  int err_flag;
  int pad;
};

// x^l for an integer exponent (Fortran's ** with an integer power)
__host__ __device__ __forceinline__ double ipow_d(double x, int l) {
  double r = 1.0;
  for (int q = 0; q < (l < 0 ? -l : l); ++q) r = r * x;
  return l < 0 ? 1.0 / r : r;
}

// Newton iteration for the temperature of a thermally perfect gas, as get_temperature_from_e_dev
// (kernels_cpu.F90:7116-7152, coefficients cv, ebar = e - cv(r+1) t0) and compute_roe_average
// (:3049-3069, coefficients cp, hbar = h - q - cp(r+1) t0) do it: at most 50 steps, stop when the
// step is below tol_iter_nr
__device__ __forceinline__ double tp_newton(const Geom& g, const double* c, double ebar, double t_start) {
  const double t0 = g.t0;
  // a start that is not a temperature (aux before its first pass holds zeros) becomes t0, the
  // value initial_conditions gives w_aux(6)
  if (!(t_start > 0.0)) t_start = t0;
  double t_old = t_start, tt = t_start;
  for (int iter = 0; iter < 50; ++iter) {
    const double tr = t_old / t0;
    double den = 0.0, num = 0.0, tp = ipow_d(tr, g.cp_l);
    for (int l = g.cp_l; l <= g.cp_r; ++l) {
      const double cl = c[l - g.cp_l];
      den = den + cl * tp;
      if (l == -1) num = num + cl * log(tr);
      else num = num + cl * (tr * tp - 1.0) / (l + 1.0);
      tp = tp * tr;
    }
    num = num * t0;
    tt = t_old + (ebar - num) / den;
    if (fabs(tt - t_old) < TOL_ITER_NR) break;
    t_old = tt;
  }
  return tt;
}

// get_temperature_from_e_dev / get_e_from_temperature_dev (kernels_cpu.F90:7116-7176): closed
// form for the calorically perfect gas, Newton from t_start (the caller's previous temperature of
// the point) for the thermally perfect one.  TPA = false compiles the thermally perfect branch
// out (kernel instantiations that never run it keep their registers).
template <bool TPA = true>
__device__ __forceinline__ double t_from_e(const Geom& g, double ee, double t_start) {
  double ebar = ee - g.cv_last * g.t0;
  if (!TPA || g.calorically_perfect) return g.t0 + ebar / g.cv0;
  return tp_newton(g, g.cvc, ebar, t_start);
}
template <bool TPA = true>
__device__ __forceinline__ double e_from_t(const Geom& g, double tt) {
  double ee = g.cv_last;
  if (!TPA || g.calorically_perfect) {
    ee = ee + g.cv0 * (tt / g.t0 - 1.0);
  } else {
    const double tr = tt / g.t0;
    double tp = ipow_d(tr, g.cp_l + 1);  // (T/t0)^(l+1)
    for (int l = g.cp_l; l <= g.cp_r; ++l) {
      const double cl = g.cvc[l - g.cp_l];
      if (l == -1) ee = ee + cl * log(tr);
      else ee = ee + cl / (l + 1.0) * (tp - 1.0);
      tp = tp * tr;
    }
  }
  return ee * g.t0;
}
// cp(T) and gamma(T) (get_gamloc_dev, kernels_cpu.F90:7096-7113; the cploc of the viscous terms)
__device__ __forceinline__ double cp_of_t(const Geom& g, double tt) {
  if (g.calorically_perfect) return g.cp0;
  const double tr = tt / g.t0;
  double cploc = 0.0, tp = ipow_d(tr, g.cp_l);
  for (int l = g.cp_l; l <= g.cp_r; ++l) {
    cploc = cploc + g.cpc[l - g.cp_l] * tp;
    tp = tp * tr;
  }
  return cploc;
}
__device__ __forceinline__ double gamloc_of_t(const Geom& g, double tt) {
  if (g.calorically_perfect) return g.gamloc;
  const double cploc = cp_of_t(g, tt);
  return cploc / (cploc - g.rgas0);
}

// Apply force_var_2 (kernels_cpu.F90:3285-3314) to the conserved values of one interior point:
// temperature from the (unshifted) state as force_var_1 computes it (:3241-3282), shifted by tbdiff.
template <bool TPA = true>
__device__ __forceinline__ double shifted_rhoe(const Geom& g, double rho, double rhou, double rhov, double rhow,
                                               double rhoe, double tbdiff, double t_start) {
  double ri = 1.0 / rho;
  double uu = rhou * ri, vv = rhov * ri, ww = rhow * ri;
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = rhoe / rho - qq;
  double tt = t_from_e<TPA>(g, ee, t_start);
  double ttnew = tt + tbdiff;
  double en = e_from_t<TPA>(g, ttnew);
  return rho * en + 0.5 * (rhou * rhou + rhov * rhov + rhow * rhow) / rho;
}

// viscosity law of eval_aux_subroutine (kernels_cpu.F90:6995-7002)
__device__ __forceinline__ double viscosity(const Geom& g, double tt) {
  if (g.visc_model == 1) return g.mu0 * pow(tt / g.t0, g.vtexp);
  if (g.visc_model == 2) {
    double tr = tt / g.t0;
    double st = g.sutherland_s / g.t_ref_dim;
    return g.mu0 * pow(tr, 1.5) * (1.0 + st) / (tr + st);
  }
  return 0.0;
}

// the same law in FP32 (the mixed form's stored viscosity)
__device__ __forceinline__ float viscosity_f(const Geom& g, float tt) {
  const float tr = tt / float(g.t0);
  if (g.visc_model == 1) return float(g.mu0) * powf(tr, float(g.vtexp));
  if (g.visc_model == 2) {
    const float st = float(g.sutherland_s / g.t_ref_dim);
    return float(g.mu0) * (tr * sqrtf(tr)) * (1.0f + st) / (tr + st);
  }
  return 0.0f;
}

// Index of a stencil point along one axis of the sensor / div arrays (stored interior only):
// periodic directions wrap; otherwise the caller decides (sensor: 0, div: clamp).
__device__ __forceinline__ int wrap(int i, int n) { return i < 1 ? i + n : (i > n ? i - n : i); }

// Deterministic block reduction of NR values per thread (sum), fixed tree order.  Every thread
// of the block must call it; thread 0 of the block receives the totals.
template <int NR, int NT>
__device__ __forceinline__ void block_reduce_sum(double (&v)[NR], double* smem /* NR * NT/32 */) {
#pragma unroll
  for (int r = 0; r < NR; ++r)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[r] += __shfl_down_sync(0xffffffffu, v[r], o);
  // linear thread index: the helper is also called from 2-D blocks
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int lane = tid & 31, warp = tid >> 5;
  if (lane == 0)
#pragma unroll
    for (int r = 0; r < NR; ++r) smem[r * (NT / 32) + warp] = v[r];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      double a = lane < NT / 32 ? smem[r * (NT / 32) + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
      v[r] = a;
    }
  }
}

}  // namespace sb200
