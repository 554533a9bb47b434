// Stage kernels of the B200 backend (FP64 and mixed forms).
//
// One Runge-Kutta stage (rk_sync, code/src/singleideal/singleideal_cpu.F90:332-409) runs as:
//   k_apply_shift  the pending force_var energy shift of the previous stage, on interior w
//   k_aux      w -> primitive/thermo fields at interior and face-ghost points; ghost values are
//              produced on the fly (periodic wrap, staggered isothermal wall mirror)
//   k_xflux    x-face hybrid fluxes + divergence (fl = ...); a warp holds 32 consecutive faces of
//              the rows' face sequence, shuffles between lanes
//   k_visc     reduced 2nd-order viscous terms, conservative face Laplacian in x, y, z,
//              div/3, stage-3 Ducros sensor, wall shear
//   k_march<1> y-face fluxes + divergence (fl += ...); register-window march along y lines
//   k_march<2> z-face fluxes + divergence + grad(mu div/3) term; block partials of force_rhs
//   k_finish_rhs  bulk quantities and the forcing correction (deterministic order)
//   k_update   RK register fln, forcing correction, w += fln, force_var / residual partials
//   k_finish_upd  bulk temperature -> pending energy shift; residual and min/max
// No face flux array is stored.  All reductions are block partials summed in a fixed order, so
// results do not depend on scheduling.
//
// Precision: template parameter R is the arithmetic type of the fluxes and viscous terms and the
// storage type of the primitive fields (aux) and div/3.  R = double is the FP64 form; R = float
// the mixed form, where w, the RK registers fl, the temperature recovery from the total energy,
// the Ducros sensor, the time step and all reductions stay FP64 and the face fluxes are carried
// as float-float pairs whose differences are formed in FP64.
#pragma once

#include <algorithm>
#include <cfloat>

#include "flux.cuh"
#include "kernels.hpp"

namespace sb200 {

namespace {

constexpr int AUX_NT = 256;
constexpr int XF_TX = 32, XF_TY = 4, XF_NT = XF_TX * XF_TY;  // x faces: 4 row-warps per block
constexpr int MT_NT = 128;                                     // march kernels
// Resident blocks per SM asked of the register allocator for the FP64 and FP32 instantiations
// of the flux kernels (measured on the 1024x256x192 boundary layer; the kernels are FP64-latency
// bound, so resident warps pay).  FP64 x pass: 4 blocks of 128 threads (128 registers, no
// spills; 16.5 against 18.6 ms per step at 3 blocks), which the WENO scratch of 2WS-1 values a
// side allows (51 KB a block).  FP64 march passes: 3 blocks (the y pass without a register
// window: at 4 blocks its reloads miss L1, 18.8 against 17.3 ms; the windowed passes spill
// 176-228 bytes at 4 blocks).  FP32, with the Newton-refined quotients: 6 blocks for the x pass
// (12.31 against 12.89 ms per step at 5, the same at 7) and 5 for the march passes (y 12.11,
// z 14.72 against 12.36, 15.33 at 4; z 17.1 at 6).
#ifndef XF_MINB_D
#define XF_MINB_D 4
#endif
#ifndef XF_MINB_F
#define XF_MINB_F 6
#endif
#ifndef MT_MINB_D
#define MT_MINB_D 3
#endif
// y / z passes: the stencil window slides along the line in registers (1), or every face loads
// its stencil afresh (0: no window held across the WENO branch, fewer registers).  Measured on
// the boundary layer: y 17.3 (reload) against 18.2 ms per step (window), z 21.9 (reload)
// against 21.3 (window): the z planes are a plane apart, so the reloads leave L1.
#ifndef SB_MARCH_WINDOW_Y
#define SB_MARCH_WINDOW_Y 0
#endif
#ifndef SB_MARCH_WINDOW_Z
#define SB_MARCH_WINDOW_Z 1
#endif
// the viscous pass with its operands staged in shared memory (1) or read per use (0)
#ifndef SB_VISC_TILED
#define SB_VISC_TILED 1
#endif
// shared-memory carve-out (percent) preferred by the WENO face kernels: their listed faces'
// stencil loads are scattered and live on L1 hits (developed boundary layer 1024x256x192: 5.0
// against 8.1 ms per step of face kernels with the largest carve-out, which fits a fourth block)
#ifndef SB_WF_CARVEOUT
#define SB_WF_CARVEOUT 72
#endif
#ifndef MT_MINB_F
#define MT_MINB_F 5
#endif
// the channel's FP32 z pass (force_rhs partials) keeps 4: at 5 it spills 244 bytes
#ifndef MT_MINB_F_CH
#define MT_MINB_F_CH 4
#endif
// the viscous pass: the staged FP64 pass at 3 blocks of 256 threads per SM (80 registers; 7.42
// against 7.57 ms per step at 4 blocks and 64 registers on the 1024x256x192 boundary layer), the
// FP32 one at 4 (5.02 against 5.62 ms at 3); the direct pass at 4 blocks measured faster than 2
// blocks at 128 registers
#ifndef VISC_MINB
#define VISC_MINB 3
#endif
// resident threads per SM asked of the register allocator for the memory-bound pointwise passes:
// 2048 (32 registers, a little spilling in the update pass), for more loads in flight
// (1024x256x192 boundary layer, ms per step against the allocator's own choice: update 4.24
// against 5.02 at 60 registers, 4.51 at 1536 threads; aux 3.01 against 3.23; dt 1.12 against
// 1.27).  The update pass's blocks are 1024 threads (UPD_MINB of them), the others 256.
#ifndef UPD_MINB
#define UPD_MINB 2
#endif
#ifndef AUX_MINB
#define AUX_MINB 8
#endif
#ifndef DT_MINB
#define DT_MINB 8
#endif
#ifndef VISC_MINB_F
#define VISC_MINB_F 4
#endif
constexpr int FIN_NT = 1024;
// cells per block of the update and time-step passes: 1024 (the time-step pass: 4 per thread of
// 256), a quarter of the block partials for their one-block finishing reductions (1024x256x192:
// 0.43 -> 0.13 and 0.17 -> 0.05 ms per step)
#ifndef SB_PT_CELLS
#define SB_PT_CELLS 4
#endif
constexpr int PT_CELLS = SB_PT_CELLS;
// the update pass: one cell per thread in blocks of 1024 (the same count of block partials)
constexpr int UPD_NT = 256 * PT_CELLS;
inline unsigned pt_blocks(long long nint) { return (unsigned)((nint + 256 * PT_CELLS - 1) / (256 * PT_CELLS)); }

// Block coordinates seen by a kernel body (d_*): the hardware block index in a plain launch
// (k_*), the block's place in its own box's grid in a launch over a box table (kb_*)
struct Blk {
  unsigned x, y, z;
};

// Primitive state of an interior point recomputed from w in FP64, with the operations of
// eval_aux_subroutine (kernels_cpu.F90:6960-7011).
struct Prim {
  double rho, uu, vv, ww, tt;
};
template <bool TPA = true>
__device__ __forceinline__ Prim prim_from_w(const Geom& g, const double* __restrict__ w, long long c,
                                            double t_start) {
  const long long n = g.nvol;
  Prim p;
  p.rho = w[c];
  const double ri = 1.0 / p.rho;
  p.uu = w[n + c] * ri;
  p.vv = w[2 * n + c] * ri;
  p.ww = w[3 * n + c] * ri;
  const double qq = 0.5 * (p.uu * p.uu + p.vv * p.vv + p.ww * p.ww);
  p.tt = t_from_e<TPA>(g, w[4 * n + c] / p.rho - qq, t_start);
  return p;
}

// Conserved state at an interior or face-ghost point (i,j,k): the stored value, a periodic copy
// (bcswap, code/src/base_cpu.F90:1326-1435) or the staggered-wall mirror of
// bcwall_staggered_subroutine (kernels_cpu.F90:6612-6678); t_src is the start of the Newton
// iteration for the mirrored point's temperature (thermally perfect gas).
template <bool TPA = true>
__device__ __forceinline__ void point_state(const Geom& g, const double* __restrict__ w, int i, int j, int k,
                                            double (&st)[5], double t_src) {
  const long long n = g.nvol;
  const int ox = (i < 1 || i > g.nx), oy = (j < 1 || j > g.ny), oz = (k < 1 || k > g.nz);
  int si = i, sj = j, sk = k;
  int wall = 0;
  // periodic faces wrap, staggered walls mirror; any other face reads its stored ghost
  if (ox && g.periodic[0]) si = wrap(i, g.nx);
  if (oz && g.periodic[2]) sk = wrap(k, g.nz);
  if (oy) {
    if (j < 1) {
      if (g.periodic[1]) sj = j + g.ny;
      else if (g.wall_ymin) { sj = 1 - j; wall = 1; }
    } else {
      if (g.periodic[1]) sj = j - g.ny;
      else if (g.wall_ymax) { sj = 2 * g.ny + 1 - j; wall = 1; }
    }
  }
  const long long src = gidx(g, si, sj, sk);
  double rho = w[src], rhou = w[n + src], rhov = w[2 * n + src], rhow = w[3 * n + src], rhoe = w[4 * n + src];
  if (wall) {
    // mirror about the wall, T_g = 2 T_w - T, p_g = p, velocity reversed
    double uu = rhou / rho, vv = rhov / rho, ww = rhow / rho;
    double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
    double ee = rhoe / rho - qq;
    double tt = t_from_e<TPA>(g, ee, t_src);
    double pp = rho * tt * g.rgas0;
    tt = 2.0 * g.t_wall - tt;
    ee = e_from_t<TPA>(g, tt);
    rho = pp / tt / g.rgas0;
    rhou = -rho * uu;
    rhov = -rho * vv;
    rhow = -rho * ww;
    rhoe = rho * (ee + qq);
  }
  st[0] = rho; st[1] = rhou; st[2] = rhov; st[3] = rhow; st[4] = rhoe;
}

// w -> aux at all interior and face-ghost points (eval_aux_subroutine, kernels_cpu.F90:6960-7011),
// computed in FP64 and stored as A; with write_ghost_w = 1 the ghost states are also stored into
// w, with write_ghost_w = 2 only they are (aux is left as it is).  With vel non-null the FP64
// velocities are stored too (the mixed form's stage-3 sensor reads them).
template <class A, bool TP = false>
__device__ __forceinline__ void d_aux(const Geom& g, double* __restrict__ w, A* __restrict__ aux,
                                                int write_ghost_w, double* __restrict__ vel, const Blk blk) {
  const long long n = g.nvol;
  const long long q = (long long)blk.x * AUX_NT + threadIdx.x;
  if (q >= n) return;
  const int ii = (int)(q % g.sx);
  const int jj = (int)((q / g.sx) % g.sy);
  const int kk = (int)(q / ((long long)g.sx * g.sy));
  const int i = ii - g.ng + 1, j = jj - g.ng + 1, k = kk - g.ng + 1;
  const int ox = (i < 1 || i > g.nx), oy = (j < 1 || j > g.ny), oz = (k < 1 || k > g.nz);
  if (ox + oy + oz > 1) return;  // halo edges and corners are never read
  if (write_ghost_w == 2 && !(ox | oy | oz)) return;
  const long long dst = gidx(g, i, j, k);
  // Newton starts (thermally perfect gas): the point's previous temperature, as eval_aux starts
  // from w_aux(6); for a wall ghost the mirror of it estimates the interior source point's
  double t_old = g.t0, t_src = g.t0;
  if constexpr (TP) {
    t_old = double(aux[5 * n + dst]);
    if (!(t_old > 0.0)) t_old = g.t0;
    t_src = 2.0 * g.t_wall - t_old;
    if (!(t_src > 0.0)) t_src = g.t0;
  }
  double st[5];
  point_state<TP>(g, w, i, j, k, st, t_src);
  double rho = st[0], rhou = st[1], rhov = st[2], rhow = st[3], rhoe = st[4];
  if (write_ghost_w && (ox | oy | oz)) {
    w[dst] = rho; w[n + dst] = rhou; w[2 * n + dst] = rhov; w[3 * n + dst] = rhow; w[4 * n + dst] = rhoe;
  }
  if (write_ghost_w == 2) return;  // ghost layers of w only; aux keeps its values
  double ri = 1.0 / rho;
  double uu = rhou * ri, vv = rhov * ri, ww = rhow * ri;
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = rhoe / rho - qq;
  double tt = t_from_e<TP>(g, ee, t_old);
  double pp = rho * tt * g.rgas0;
  if (vel) {  // FP64 velocities, as the sensor forms them from w
    vel[dst] = uu;
    vel[n + dst] = vv;
    vel[2 * n + dst] = ww;
  }
  aux[dst] = A(rho);
  aux[n + dst] = A(uu);
  aux[2 * n + dst] = A(vv);
  aux[3 * n + dst] = A(ww);
  aux[4 * n + dst] = A((rhoe + pp) / rho);
  aux[5 * n + dst] = A(tt);
  // the mixed form's viscous arithmetic is FP32, and so is its viscosity law (with SB_FP32_FAST)
  if constexpr (sizeof(A) == sizeof(float) && SB_FP32_FAST != 0)
    aux[6 * n + dst] = viscosity_f(g, float(tt));
  else
    aux[6 * n + dst] = A(viscosity(g, tt));
  // FP64 form: the sound speed, which the WENO eigenvalue bound of every face reads at its
  // stencil points (the same expression the flux would form)
  if constexpr (sizeof(A) == sizeof(double)) {
    const double gq = TP ? gamloc_of_t(g, tt) : g.gamloc;
    aux[7 * n + dst] = sqrt(gq * g.rgas0 * tt);
  }
}
template <class A, bool TP = false>
__global__ void __launch_bounds__(AUX_NT, AUX_MINB) k_aux(Geom g, double* __restrict__ w, A* __restrict__ aux,
                                                int write_ghost_w, double* __restrict__ vel) {
  d_aux<A, TP>(g, w, aux, write_ghost_w, vel, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

// Ducros sensor in FP64 from w for the mixed form, so that the central/WENO switch is taken
// on the same values as in the FP64 form.  mode 0: initial sensor of run() (visflx(mode=2),
// kernels_cpu.F90:4680-4682); mode 1: sensor_subroutine of stage 3 (:4726-4744), which works
// from the stored |omega| and div/3 of visflx_reduced_ord2; mode 2: the same from the
// visc_order derivatives of visflx_nosensor_subroutine (conservative_viscous = 0); mode 3: the
// initial sensor of run() for conservative_viscous = 0 (visflx(mode=0), visflx_subroutine,
// kernels_cpu.F90:3598-3777: visc_order derivatives, theta from div and omega directly).
__device__ __forceinline__ void d_sensor64(const Geom& g, const double* __restrict__ w, double* __restrict__ out,
                                                  int mode, const Blk blk) {
  const long long q = (long long)blk.x * 256 + threadIdx.x;
  if (q >= g.nint) return;
  int i, j, k;
  cell_of(g, q, i, j, k);
  auto vel = [&](int a, int b, int c, double (&v)[3]) {
    double st[5];
    point_state(g, w, a, b, c, st, g.t_wall);
    const double ri = 1.0 / st[0];
    v[0] = st[1] * ri; v[1] = st[2] * ri; v[2] = st[3] * ri;
  };
  double ux, vx, wx, uy, vy, wy, uz, vz, wz;
  if (mode < 2) {
    double xp[3], xm[3], yp[3], ym[3], zp[3], zm[3];
    vel(i + 1, j, k, xp); vel(i - 1, j, k, xm);
    vel(i, j + 1, k, yp); vel(i, j - 1, k, ym);
    vel(i, j, k + 1, zp); vel(i, j, k - 1, zm);
    double dxl = 1.0 / (g.x[i + 1] - g.x[i - 1]);
    double dyl = 1.0 / (g.y[j + 1] - g.y[j - 1]);
    double dzl = 1.0 / (g.z[k + 1] - g.z[k - 1]);
    ux = dxl * (xp[0] - xm[0]); vx = dxl * (xp[1] - xm[1]); wx = dxl * (xp[2] - xm[2]);
    uy = dyl * (yp[0] - ym[0]); vy = dyl * (yp[1] - ym[1]); wy = dyl * (yp[2] - ym[2]);
    uz = dzl * (zp[0] - zm[0]); vz = dzl * (zp[1] - zm[1]); wz = dzl * (zp[2] - zm[2]);
  } else {
    // the derivatives of visflx_nosensor_subroutine (order visc_order, metric after the sum)
    const int lv = g.lmax_base;
    double d[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int l = 1; l <= lv; ++l) {
      const double ccl = g.coeff[lv - 1][l - 1];
      double p[3], m[3];
      vel(i + l, j, k, p); vel(i - l, j, k, m);
      for (int v = 0; v < 3; ++v) d[0][v] = d[0][v] + ccl * (p[v] - m[v]);
      vel(i, j + l, k, p); vel(i, j - l, k, m);
      for (int v = 0; v < 3; ++v) d[1][v] = d[1][v] + ccl * (p[v] - m[v]);
      vel(i, j, k + l, p); vel(i, j, k - l, m);
      for (int v = 0; v < 3; ++v) d[2][v] = d[2][v] + ccl * (p[v] - m[v]);
    }
    ux = d[0][0] * g.dcsidx[i]; vx = d[0][1] * g.dcsidx[i]; wx = d[0][2] * g.dcsidx[i];
    uy = d[1][0] * g.detady[j]; vy = d[1][1] * g.detady[j]; wy = d[1][2] * g.detady[j];
    uz = d[2][0] * g.dzitdz[k]; vz = d[2][1] * g.dzitdz[k]; wz = d[2][2] * g.dzitdz[k];
  }
  double div = ux + vy + wz;
  double omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
  double omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
  double u0l0 = g.u0 / g.l0;
  if (mode == 1 || mode == 2) {
    double div3l = div / 3.0;
    double om = sqrt(omod2);
    omod2 = om * om;
    div = 3.0 * div3l;
  }
  double t = fmax(-div / sqrt(omod2 + div * div + u0l0 * u0l0), 0.0);
  out[q] = t * t;
}
__global__ void __launch_bounds__(256) k_sensor64(Geom g, const double* __restrict__ w, double* __restrict__ out,
                                                  int mode) {
  d_sensor64(g, w, out, mode, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}
// The stage-3 Ducros sensor of the mixed form (k_sensor64 modes 1 and 2) from the FP64 velocities
// that the stage's aux pass stored at the interior and face-ghost points: the same quotients and
// the same arithmetic, without re-forming six neighbours' states per point.
__device__ __forceinline__ void d_sensor_vel(const Geom& g, const double* __restrict__ vel, double* __restrict__ out,
                                                    int mode, const Blk blk) {
  const long long q = (long long)blk.x * 256 + threadIdx.x;
  if (q >= g.nint) return;
  int i, j, k;
  cell_of(g, q, i, j, k);
  const long long n = g.nvol, c = gidx(g, i, j, k), sY = g.sx, sZ = (long long)g.sx * g.sy;
  auto V = [&](long long a, int m) { return vel[m * n + a]; };
  double ux, vx, wx, uy, vy, wy, uz, vz, wz;
  if (mode == 1) {
    double dxl = 1.0 / (g.x[i + 1] - g.x[i - 1]);
    double dyl = 1.0 / (g.y[j + 1] - g.y[j - 1]);
    double dzl = 1.0 / (g.z[k + 1] - g.z[k - 1]);
    ux = dxl * (V(c + 1, 0) - V(c - 1, 0)); vx = dxl * (V(c + 1, 1) - V(c - 1, 1)); wx = dxl * (V(c + 1, 2) - V(c - 1, 2));
    uy = dyl * (V(c + sY, 0) - V(c - sY, 0)); vy = dyl * (V(c + sY, 1) - V(c - sY, 1));
    wy = dyl * (V(c + sY, 2) - V(c - sY, 2));
    uz = dzl * (V(c + sZ, 0) - V(c - sZ, 0)); vz = dzl * (V(c + sZ, 1) - V(c - sZ, 1));
    wz = dzl * (V(c + sZ, 2) - V(c - sZ, 2));
  } else {
    const int lv = g.lmax_base;
    double d[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int l = 1; l <= lv; ++l) {
      const double ccl = g.coeff[lv - 1][l - 1];
      for (int v = 0; v < 3; ++v) d[0][v] = d[0][v] + ccl * (V(c + l, v) - V(c - l, v));
      for (int v = 0; v < 3; ++v) d[1][v] = d[1][v] + ccl * (V(c + l * sY, v) - V(c - l * sY, v));
      for (int v = 0; v < 3; ++v) d[2][v] = d[2][v] + ccl * (V(c + l * sZ, v) - V(c - l * sZ, v));
    }
    ux = d[0][0] * g.dcsidx[i]; vx = d[0][1] * g.dcsidx[i]; wx = d[0][2] * g.dcsidx[i];
    uy = d[1][0] * g.detady[j]; vy = d[1][1] * g.detady[j]; wy = d[1][2] * g.detady[j];
    uz = d[2][0] * g.dzitdz[k]; vz = d[2][1] * g.dzitdz[k]; wz = d[2][2] * g.dzitdz[k];
  }
  double div = ux + vy + wz;
  double omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
  double omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
  double u0l0 = g.u0 / g.l0;
  double div3l = div / 3.0;
  double om = sqrt(omod2);
  omod2 = om * om;
  div = 3.0 * div3l;
  double t = fmax(-div / sqrt(omod2 + div * div + u0l0 * u0l0), 0.0);
  out[q] = t * t;
}
__global__ void __launch_bounds__(256) k_sensor_vel(Geom g, const double* __restrict__ vel, double* __restrict__ out,
                                                    int mode) {
  d_sensor_vel(g, vel, out, mode, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

// Pending energy shift on interior points only (before a download).  The Newton start of the
// thermally perfect gas is the point's temperature in aux, as force_var_1 starts from w_aux(6).
template <class A, bool TP = false>
__device__ __forceinline__ void d_apply_shift(const Geom& g, double* __restrict__ w, const A* __restrict__ aux,
                                                        const Scalars* __restrict__ sc, const Blk blk) {
  const long long q = (long long)blk.x * AUX_NT + threadIdx.x;
  if (q >= g.nint) return;
  int i, j, k;
  cell_of(g, q, i, j, k);
  const long long n = g.nvol, s = gidx(g, i, j, k);
  const double t_start = TP ? double(aux[5 * n + s]) : g.t0;
  w[4 * n + s] = shifted_rhoe<TP>(g, w[s], w[n + s], w[2 * n + s], w[3 * n + s], w[4 * n + s], sc->tbdiff, t_start);
}
template <class A, bool TP = false>
__global__ void __launch_bounds__(AUX_NT) k_apply_shift(Geom g, double* __restrict__ w, const A* __restrict__ aux,
                                                        const Scalars* __restrict__ sc) {
  d_apply_shift<A, TP>(g, w, aux, sc, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

// Readers of the interior-only sensor and div/3 arrays at a stencil point that may be a ghost.
template <class R>
__device__ __forceinline__ R sensor_at(const Geom& g, const R* __restrict__ s, int i, int j, int k) {
  if (i < 1 || i > g.nx) { if (!g.periodic[0]) return R(0); i = wrap(i, g.nx); }
  if (j < 1 || j > g.ny) { if (!g.periodic[1]) return R(0); j = wrap(j, g.ny); }
  if (k < 1 || k > g.nz) { if (!g.periodic[2]) return R(0); k = wrap(k, g.nz); }
  return s[iidx(g, i, j, k)];
}
// bcextr_var (kernels_cpu.F90:6199-6254) then bcswap_var: periodic wrap, otherwise nearest interior
template <class R>
__device__ __forceinline__ R div3_at(const Geom& g, const R* __restrict__ d, int i, int j, int k) {
  if (i < 1 || i > g.nx) i = g.periodic[0] ? wrap(i, g.nx) : (i < 1 ? 1 : g.nx);
  if (j < 1 || j > g.ny) j = g.periodic[1] ? wrap(j, g.ny) : (j < 1 ? 1 : g.ny);
  if (k < 1 || k > g.nz) k = g.periodic[2] ? wrap(k, g.nz) : (k < 1 ? 1 : g.nz);
  return d[iidx(g, i, j, k)];
}

// Per-thread scratch of the WENO characteristic projections (dynamic shared memory of the flux
// kernels, 5 fields x (2WS-1) points x 2 sides per thread, thread-interleaved)
template <class R>
__device__ __forceinline__ R* weno_scratch() {
  extern __shared__ __align__(16) unsigned char sb_dyn_smem[];
  return reinterpret_cast<R*>(sb_dyn_smem);
}
template <class R, int WS>
constexpr size_t weno_scratch_bytes(int nthreads) {
  return (size_t)nthreads * 5 * (2 * WS - 1) * 2 * sizeof(R);
}

template <int DIR>
__device__ __forceinline__ int face_ep(const Geom& g, int p) {
  return DIR == 0 ? g.epx[p] : (DIR == 1 ? g.epy[p] : g.epz[p]);
}

// WENO faces apart (1) or always inside the hybrid passes (0).  Apart, the faces whose stencil
// sees the sensor are listed per direction once per step and computed by their own kernel at
// full occupancy; the hybrid passes read their fluxes from a face buffer.  A warp of the hybrid
// passes otherwise runs both branches whenever one of its faces is a WENO face, which with
// scattered WENO faces costs nearly a full WENO pass.  When most faces are WENO faces the
// buffer's extra traffic and the stencil loads without the passes' sliding window cost more
// than that, so each direction chooses on the device from its list's length (weno_split): the
// x pass holds both branches, the y and z passes are launched in both forms and the one not
// chosen leaves at once (about a thousand blocks; the x pass's grid is too large for that).
// The lists themselves are built only when a sample of every 16th plane is within the
// threshold, so a step that keeps its WENO faces in the hybrid passes pays for the sample only.
#ifndef SB_WENO_SPLIT
#define SB_WENO_SPLIT 1
#endif

// Face index of the WENO face buffer of direction DIR for face p (0..n along DIR) of the line
// (a, b): x faces p fastest (a = j, b = k), y and z faces i fastest (a = i; b = k for y, j for z).
template <int DIR>
__host__ __device__ __forceinline__ long long wface_index(const Geom& g, int p, int a, int b) {
  if (DIR == 0) return ((long long)(b - 1) * g.ny + (a - 1)) * (g.nx + 1) + p;
  if (DIR == 1) return ((long long)(b - 1) * (g.ny + 1) + p) * g.nx + (a - 1);
  return ((long long)p * g.ny + (b - 1)) * g.nx + (a - 1);
}
template <int DIR>
__device__ __forceinline__ void wface_decode(const Geom& g, unsigned f, int& p, int& a, int& b) {
  // face counts per direction stay below 2^32 (checked at context creation)
  if (DIR == 0) {
    const unsigned n0 = g.nx + 1, r = f / n0;
    p = (int)(f - r * n0);
    a = (int)(r % (unsigned)g.ny) + 1;
    b = (int)(r / (unsigned)g.ny) + 1;
  } else if (DIR == 1) {
    const unsigned r = f / (unsigned)g.nx;
    a = (int)(f - r * (unsigned)g.nx) + 1;
    p = (int)(r % (unsigned)(g.ny + 1));
    b = (int)(r / (unsigned)(g.ny + 1)) + 1;
  } else {
    const unsigned r = f / (unsigned)g.nx;
    a = (int)(f - r * (unsigned)g.nx) + 1;
    b = (int)(r % (unsigned)g.ny) + 1;
    p = (int)(r / (unsigned)g.ny);
  }
}
// Whether the hybrid pass of direction DIR reads its WENO faces from the face buffer this step
// (the list, built at stage 1, holds at most wthr[DIR] faces) or computes them itself.
template <int DIR>
__device__ __forceinline__ bool weno_split(const Geom& g) {
  return SB_WENO_SPLIT && g.wsplit_on && *(volatile const unsigned*)(g.wcount + DIR) <= g.wthr[DIR];
}
template <int DIR>
__host__ __device__ __forceinline__ long long wface_count(const Geom& g) {
  return DIR == 0 ? (long long)(g.nx + 1) * g.ny * g.nz
                  : (DIR == 1 ? (long long)g.nx * (g.ny + 1) * g.nz : (long long)g.nx * g.ny * (g.nz + 1));
}

// Flux at a face from a loaded stencil window (points p-(S-1) .. p+S of face p):
// hi + lo is the face flux (lo = 0 in the FP64 form).  FS holds the flux variant flags of a
// kernel instantiation: bit 0 the component-wise (Rusanov) WENO splitting, bit 1 the thermally
// perfect gas, bit 2 a central flux with nkeep != 0 (otherwise nkeep = 0 at compile time), bit 3
// the WENO-Z weights (otherwise WENO-JS).  Options fixed per kernel instantiation keep the code
// of the branches a case does not take out of the register allocation of the ones it does
// (measured: nkeep 10-18 %, the WENO version 3-10 % of the flux passes).
// The WENO flux of face p (characteristic or component-wise splitting), order reduced near
// non-periodic boundaries as ep_ord_change says.
template <class R, int DIR, int LB, int WS, int S, int FS = 0>
__device__ __forceinline__ void weno_face(const Geom& g, const Stencil<R, S>& st, int p, R (&hi)[5], R (&lo)[5],
                                          R* __restrict__ gs, int gstride, const R* __restrict__ cpt, long long cstr) {
  const int ep = face_ep<DIR>(g, p);
  const int ord = max(WS + ep, 1);
  if constexpr ((FS & 1) != 0)
    rusanov_flux<R, DIR, WS, S, (FS & 2) != 0, (FS & 8) != 0>(g, st, ord, hi, lo, cpt, cstr);
  else
    weno_flux<R, DIR, WS, S, (FS & 2) != 0, (FS & 8) != 0>(g, st, ord, hi, lo, gs, gstride, cpt, cstr);
}

template <class R, int DIR, int LB, int WS, int S, int FS = 0>
__device__ __forceinline__ void window_flux(const Geom& g, const Stencil<R, S>& st, bool ishk, int p,
                                            R (&hi)[5], R (&lo)[5], R* __restrict__ gs, int gstride,
                                            const R* __restrict__ cpt, long long cstr, bool split, int wa, int wb) {
  const int nd = DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
  if (!ishk) {
    const int ep = face_ep<DIR>(g, p);
    const int lmax = max(g.lmax_base + ep, 1);
    const bool zf = (p == 0 && g.fzf[2 * DIR] == 1) || (p == nd && g.fzf[2 * DIR + 1] == 1);
    central_flux<R, DIR, LB, S, (FS & 4) != 0>(g, st, lmax, g.nkeep, zf, hi, lo);
  } else if (SB_WENO_SPLIT && split) {
    // the WENO faces come from the face buffer
    const R* fb = static_cast<const R*>(g.wface);
    const long long wf = wface_index<DIR>(g, p, wa, wb);
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      hi[m] = __ldg(fb + m * g.nwface + wf);
      lo[m] = sizeof(R) == sizeof(double) ? R(0) : __ldg(fb + (5 + m) * g.nwface + wf);
    }
  } else {
    weno_face<R, DIR, LB, WS, S, FS>(g, st, p, hi, lo, gs, gstride, cpt, cstr);
  }
}

template <class R, int S>
__device__ __forceinline__ void load_point(const Geom& g, Stencil<R, S>& st, int q, const R* __restrict__ aux,
                                           long long n, long long a) {
  st.rho[q] = __ldg(aux + a);
  st.u[q] = __ldg(aux + n + a);
  st.v[q] = __ldg(aux + 2 * n + a);
  st.w[q] = __ldg(aux + 3 * n + a);
  st.h[q] = __ldg(aux + 4 * n + a);
  st.t[q] = __ldg(aux + 5 * n + a);
#if SB_CACHE_C
  st.c[q] = sqrt(R(g.gamloc) * R(g.rgas0) * st.t[q]);
#endif
}

// Divergence of one variable between a face pair, in FP64: (hi_up - hi_lo) + (lo_up - lo_lo).
template <class R>
__device__ __forceinline__ double face_diff(R hup, R lup, R hlo, R llo) {
  if constexpr (sizeof(R) == sizeof(double)) {
    return double(hup) - double(hlo);
  } else {
    return (double(hup) - double(hlo)) + (double(lup) - double(llo));
  }
}

// x faces: each warp owns one (j,k) row segment of 32 faces (i0-1 .. i0+30) and updates the 31
// cells between them; the upper face of a cell comes from the neighbouring lane by a shuffle,
// so no shared memory and no block barrier are needed.  fl is written (first contribution of the
// stage, euler_x after init_flux).
template <class R, int LB, int WS, int FS = 0>
__device__ __forceinline__ void d_xflux(const Geom& g, const R* __restrict__ aux,
                                                 const double* __restrict__ sensor, double* __restrict__ fl, const Blk blk) {
  constexpr int S = LB > WS ? LB : WS;
  const int lane = threadIdx.x;
  // The x faces of all rows form one sequence (row (k-1) ny + (j-1), faces p = 0..nx in a row;
  // fewer than 2^32 faces, checked at create): warp w holds faces 31w .. 31w+31, and forms the
  // cells between its lanes' faces within a row, so no lane idles at a row's end.
  const unsigned nfr = (unsigned)g.nx + 1u;
  const unsigned long long nface = (unsigned long long)nfr * g.ny * g.nz;
  const unsigned long long f0 = (unsigned long long)(blk.x * XF_TY + threadIdx.y) * (XF_TX - 1);
  if (f0 >= nface) return;  // whole warp leaves together
  const bool in = f0 + lane < nface;
  const unsigned fu = in ? (unsigned)(f0 + lane) : 0u;
  const unsigned row = fu / nfr;
  const int p = (int)(fu - row * nfr);  // this lane's face (between p and p+1)
  const int j = (int)(row % (unsigned)g.ny) + 1, k = (int)(row / (unsigned)g.ny) + 1;
  const bool face_ok = in && p >= g.eul_imin - 1 && p <= g.eul_imax;
  R fh[5] = {0, 0, 0, 0, 0}, fo[5] = {0, 0, 0, 0, 0};
  if (face_ok) {
    bool ishk = false;
#pragma unroll
    for (int o = -WS + 1; o <= WS; ++o) ishk = ishk || sensor_at(g, sensor, p + o, j, k) > g.sensor_threshold;
    Stencil<R, S> st;
    const long long base = gidx(g, p, j, k);
#pragma unroll
    for (int q = 0; q < 2 * S; ++q) load_point<R, S>(g, st, q, aux, g.nvol, base + (q - (S - 1)));
    // the FP64 form's aux holds the sound speed of every point (field 8): stencil point 0 onwards
    const R* cpt = sizeof(R) == sizeof(double) ? aux + 7 * g.nvol + base - (S - 1) : nullptr;
    window_flux<R, 0, LB, WS, S, FS>(g, st, ishk, p, fh, fo, weno_scratch<R>() + threadIdx.y * XF_TX + lane, XF_NT,
                                     cpt, 1, weno_split<0>(g), j, k);
  }
  R hu[5], lu[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    hu[m] = __shfl_down_sync(0xffffffffu, fh[m], 1);
    if constexpr (sizeof(R) != sizeof(double)) lu[m] = __shfl_down_sync(0xffffffffu, fo[m], 1);
    else lu[m] = R(0);
  }
  const int i = p + 1;  // cell between faces p and p+1 (the next lane's face, in this row)
  if (lane < XF_TX - 1 && in && i <= g.nx) {
    const bool upd = i >= g.eul_imin && i <= g.eul_imax;
    const double met = g.dcsidx[i];
    const long long ic = iidx(g, i, j, k);
#pragma unroll
    for (int m = 0; m < 5; ++m) fl[m * g.nint + ic] = upd ? face_diff<R>(hu[m], lu[m], fh[m], fo[m]) * met : 0.0;
  }
}
template <class R, int LB, int WS, int FS = 0>
__global__ void __launch_bounds__(XF_NT, sizeof(R) == 8 ? XF_MINB_D : XF_MINB_F) k_xflux(Geom g, const R* __restrict__ aux,
                                                 const double* __restrict__ sensor, double* __restrict__ fl) {
  d_xflux<R, LB, WS, FS>(g, aux, sensor, fl, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

// y or z faces by marching: each thread owns one line (fixed i and the other transverse index)
// over a segment of cells, keeps the stencil window of the current face in registers (one new
// point loaded per face), computes every face of the segment once and adds the divergence to fl.
// The z pass also applies the grad(mu div/3) term of visflx_div_ord2_subroutine
// (kernels_cpu.F90:3446-3480) and emits the force_rhs block partials (:3157-3193).
template <class R, int DIR, int LB, int WS, bool CH = false, int FS = 0, bool SPLIT = false>
__device__ __forceinline__ void d_march(const Geom& g, const R* __restrict__ aux,
                                                 const double* __restrict__ sensor, double* __restrict__ fl,
                                                 const R* __restrict__ div3,
                                                 const double* __restrict__ w, const double* __restrict__ fl_prev,
                                                 const Scalars* __restrict__ sc, double rhork, double gamrk,
                                                 int istep, int seglen, int nseg, double* __restrict__ red, const Blk blk) {
  static_assert(DIR == 1 || DIR == 2, "march kernel handles y and z");
  constexpr int S = LB > WS ? LB : WS;
  constexpr int NP = 2 * S;
  __shared__ double rsh[5 * (MT_NT / 32)];
  const int n1 = g.nx;
  const int n2 = DIR == 1 ? g.nz : g.ny;
  const int nd = DIR == 1 ? g.ny : g.nz;
  const int emin = DIR == 1 ? g.eul_jmin : g.eul_kmin;
  const int emax = DIR == 1 ? g.eul_jmax : g.eul_kmax;
  const long long nlines = (long long)n1 * n2;
  const long long t = (long long)blk.x * MT_NT + threadIdx.x;
  // both forms are launched; the one that the list length does not select leaves at once
  if (weno_split<DIR>(g) != SPLIT) return;
  double part[5] = {0, 0, 0, 0, 0};
  if (t < nlines * nseg) {
    const int i = (int)(t % n1) + 1;
    const int b = (int)((t / n1) % n2) + 1;  // k for y lines, j for z lines
    const int sgi = (int)(t / nlines);
    const int c0 = emin + sgi * seglen;
    const int c1 = min(c0 + seglen - 1, emax);
    const long long n = g.nvol, nI = g.nint;
    const long long sd = DIR == 1 ? (long long)g.sx : (long long)g.sx * g.sy;
    const long long base0 = DIR == 1 ? gidx(g, i, 0, b) : gidx(g, i, b, 0);  // address of c = 0
    // sensor bits of the face p: points p-WS+1 .. p+WS at bits 0 .. 2WS-1
    auto sensor_bit = [&](int c) -> unsigned {
      if (c < 1 || c > nd) {
        if (!g.periodic[DIR]) return 0u;
        c = wrap(c, nd);
      }
      const double th = DIR == 1 ? sensor[iidx(g, i, c, b)] : sensor[iidx(g, i, b, c)];
      return th > g.sensor_threshold ? 1u : 0u;
    };
    // preload the window and sensor bits of the face c0-2; the loop starts at the face c0-1
    Stencil<R, S> st;
    const int p = c0 - 2;
    constexpr bool WIN = DIR == 1 ? SB_MARCH_WINDOW_Y != 0 : SB_MARCH_WINDOW_Z != 0;
    if constexpr (WIN) {
#pragma unroll
      for (int q = 1; q < NP; ++q) load_point<R, S>(g, st, q, aux, n, base0 + (long long)(p - (S - 1) + q) * sd);
    }
    unsigned mask = 0;
#pragma unroll
    for (int bq = 1; bq < 2 * WS; ++bq) mask |= sensor_bit(p - WS + 1 + bq) << bq;
    R hlo[5] = {0, 0, 0, 0, 0}, llo[5] = {0, 0, 0, 0, 0};
    // x(i+1)-x(i-1) and y(j+1)-y(j-1) of the z line (the grad(mu div/3) term)
    R xdiff = R(1), ydiff = R(1);
    if constexpr (DIR == 2) {
      xdiff = R(g.x[i + 1] - g.x[i - 1]);
      ydiff = R(g.y[b + 1] - g.y[b - 1]);
    }
    for (int c = c0 - 1; c <= c1; ++c) {
      if constexpr (WIN) {
        // slide the window to the face c
#pragma unroll
        for (int q = 0; q < NP - 1; ++q) {
          st.rho[q] = st.rho[q + 1]; st.u[q] = st.u[q + 1]; st.v[q] = st.v[q + 1];
          st.w[q] = st.w[q + 1]; st.h[q] = st.h[q + 1]; st.t[q] = st.t[q + 1];
#if SB_CACHE_C
          st.c[q] = st.c[q + 1];
#endif
        }
        load_point<R, S>(g, st, NP - 1, aux, n, base0 + (long long)(c + S) * sd);
      } else {
        // the face's stencil, loaded afresh: the lanes of a warp hold consecutive i, so every
        // load is one coalesced row, and the points shared with the previous face come from L1
#pragma unroll
        for (int q = 0; q < NP; ++q) load_point<R, S>(g, st, q, aux, n, base0 + (long long)(c - (S - 1) + q) * sd);
      }
      mask = (mask >> 1) | (sensor_bit(c + WS) << (2 * WS - 1));
      R hhi[5], lhi[5];
      const R* cpt = sizeof(R) == sizeof(double) ? aux + 7 * n + base0 + (long long)(c - (S - 1)) * sd : nullptr;
      window_flux<R, DIR, LB, WS, S, FS>(g, st, mask != 0u, c, hhi, lhi, weno_scratch<R>() + threadIdx.x, MT_NT, cpt,
                                         sd, SPLIT, i, b);
      if (c >= c0) {
        // cell c lies between the faces c-1 (lo) and c (hi)
        const long long ic = DIR == 1 ? iidx(g, i, c, b) : iidx(g, i, b, c);
        const double met = DIR == 1 ? g.detady[c] : g.dzitdz[c];
        double f[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) f[m] = fl[m * nI + ic] + face_diff<R>(hhi[m], lhi[m], hlo[m], llo[m]) * met;
        if (DIR == 2) {
          const int j = b, k = c;
          const long long a = gidx(g, i, j, k);
          // the cell's velocities are the stencil's point S-1 (the face c's lower point)
          const R uu = st.u[S - 1], vv = st.v[S - 1], ww = st.w[S - 1], mu = aux[6 * n + a];
          R sigx, sigy, sigz;
          if (g.conservative_viscous) {
            const R dxl = mu / xdiff;
            const R dyl = mu / ydiff;
            const R dzl = mu / R(g.z[k + 1] - g.z[k - 1]);
            sigx = dxl * (div3_at(g, div3, i + 1, j, k) - div3_at(g, div3, i - 1, j, k));
            sigy = dyl * (div3_at(g, div3, i, j + 1, k) - div3_at(g, div3, i, j - 1, k));
            sigz = dzl * (div3_at(g, div3, i, j, k + 1) - div3_at(g, div3, i, j, k - 1));
          } else {
            // visflx_div_subroutine (kernels_cpu.F90:3484-3532): order visc_order
            const int lv = g.lmax_base;
            R dx3 = R(0), dy3 = R(0), dz3 = R(0);
            for (int l = 1; l <= lv; ++l) {
              const R ccl = R(g.coeff[lv - 1][l - 1]);
              dx3 = dx3 + ccl * (div3_at(g, div3, i + l, j, k) - div3_at(g, div3, i - l, j, k));
              dy3 = dy3 + ccl * (div3_at(g, div3, i, j + l, k) - div3_at(g, div3, i, j - l, k));
              dz3 = dz3 + ccl * (div3_at(g, div3, i, j, k + l) - div3_at(g, div3, i, j, k - l));
            }
            sigx = mu * (dx3 * R(g.dcsidx[i]));
            sigy = mu * (dy3 * R(g.detady[j]));
            sigz = mu * (dz3 * R(g.dzitdz[k]));
          }
          const R sigq = sigx * uu + sigy * vv + sigz * ww;
          f[1] = f[1] - double(sigx);
          f[2] = f[2] - double(sigy);
          f[3] = f[3] - double(sigz);
          f[4] = f[4] - double(sigq);
          if constexpr (CH) {
            const double dt = sc->dt;
            const double rhodt = rhork * dt, gamdt = gamrk * dt;
            double fln1 = (istep > 1 ? -(rhodt * fl_prev[ic]) : 0.0) - gamdt * f[0];
            double fln2 = (istep > 1 ? -(rhodt * fl_prev[nI + ic]) : 0.0) - gamdt * f[1];
            double dy = g.yn[j + 1] - g.yn[j];
            const Prim pr = prim_from_w<(FS & 2) != 0>(g, w, a, (FS & 2) != 0 ? double(aux[5 * n + a]) : g.t0);
            double rhou = w[n + a];
            part[0] += fln1 * dy;
            part[1] += fln2 * dy;
            part[2] += pr.rho * dy;
            part[3] += rhou * dy;
            part[4] += rhou * dy * pr.tt;
          }
        }
#pragma unroll
        for (int m = 0; m < 5; ++m) fl[m * nI + ic] = f[m];
      }
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        hlo[m] = hhi[m];
        llo[m] = lhi[m];
      }
    }
  }
  if constexpr (DIR == 2 && CH) {
    block_reduce_sum<5, MT_NT>(part, rsh);
    if (threadIdx.x == 0)
#pragma unroll
      for (int r = 0; r < 5; ++r) red[(long long)blk.x * 5 + r] = part[r];
  }
}
template <class R, int DIR, int LB, int WS, bool CH = false, int FS = 0, bool SPLIT = false>
__global__ void __launch_bounds__(MT_NT, sizeof(R) == 8 ? MT_MINB_D : (CH ? MT_MINB_F_CH : MT_MINB_F)) k_march(Geom g, const R* __restrict__ aux,
                                                 const double* __restrict__ sensor, double* __restrict__ fl,
                                                 const R* __restrict__ div3,
                                                 const double* __restrict__ w, const double* __restrict__ fl_prev,
                                                 const Scalars* __restrict__ sc, double rhork, double gamrk,
                                                 int istep, int seglen, int nseg, double* __restrict__ red) {
  d_march<R, DIR, LB, WS, CH, FS, SPLIT>(g, aux, sensor, fl, div3, w, fl_prev, sc, rhork, gamrk, istep, seglen, nseg, red, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

// visflx_reduced_ord2_subroutine (kernels_cpu.F90:4623-4721, update_sensor = 0) followed by
// visflx_x/y/z_subroutine (:4779-4999), in the reference's accumulation order; at stage 3 also
// sensor_subroutine (:4726-4744) into the next sensor buffer.  Arithmetic in R, accumulation
// into the FP64 register.
template <class R, bool TP = false>
__device__ __forceinline__ void d_visc(const Geom& g, const R* __restrict__ aux, double* __restrict__ fl,
                                              R* __restrict__ div3, double* __restrict__ sensor_next,
                                              double* __restrict__ wallprop, int do_sensor, const Blk blk) {
  const long long q = (long long)blk.x * 256 + threadIdx.x;
  if (q >= g.nint) return;
  int i, j, k;
  cell_of(g, q, i, j, k);
  const long long n = g.nvol, nI = g.nint;
  const long long c = gidx(g, i, j, k);
  const long long sX = 1, sY = g.sx, sZ = (long long)g.sx * g.sy;
  auto A = [&](long long a, int m) -> R { return __ldg(aux + (m - 1) * n + a); };
  const R uu = A(c, 2), vv = A(c, 3), ww = A(c, 4), mu = A(c, 7);
  // cp at the point (visflx_reduced_ord2) and at a face's mean temperature (visflx_x/y/z);
  // a constant for the calorically perfect gas
  const R cploc = TP ? R(cp_of_t(g, double(A(c, 6)))) : R(g.cp0), prandtl = R(g.prandtl);
  // 1/(x(i+1)-x(i-1)) etc. from the per-line tables (the same quotients as a division here)
  R dxl, dyl, dzl;
  if constexpr (sizeof(R) == sizeof(double)) {
    dxl = R(__ldg(g.vrl[0] + i)); dyl = R(__ldg(g.vrl[1] + j)); dzl = R(__ldg(g.vrl[2] + k));
  } else {
    dxl = R(__ldg(g.vrlf[0] + i)); dyl = R(__ldg(g.vrlf[1] + j)); dzl = R(__ldg(g.vrlf[2] + k));
  }
  R ux = dxl * (A(c + sX, 2) - A(c - sX, 2));
  R vx = dxl * (A(c + sX, 3) - A(c - sX, 3));
  R wx = dxl * (A(c + sX, 4) - A(c - sX, 4));
  R mux = dxl * (A(c + sX, 7) - A(c - sX, 7));
  R uy = dyl * (A(c + sY, 2) - A(c - sY, 2));
  R vy = dyl * (A(c + sY, 3) - A(c - sY, 3));
  R wy = dyl * (A(c + sY, 4) - A(c - sY, 4));
  R ty = dyl * (A(c + sY, 6) - A(c - sY, 6));
  R muy = dyl * (A(c + sY, 7) - A(c - sY, 7));
  R uz = dzl * (A(c + sZ, 2) - A(c - sZ, 2));
  R vz = dzl * (A(c + sZ, 3) - A(c - sZ, 3));
  R wz = dzl * (A(c + sZ, 4) - A(c - sZ, 4));
  R muz = dzl * (A(c + sZ, 7) - A(c - sZ, 7));
  if (j == 1) {
    const long long wp = (long long)(k - 1) * g.nx + (i - 1);
    const long long nw = (long long)g.nx * g.nz;
    wallprop[wp] = double(mu * uy);
    wallprop[nw + wp] = double(mu * wy);
    wallprop[2 * nw + wp] = double(mu * ty * cploc / prandtl);
  }
  R div = ux + vy + wz;
  R div3l = div / R(3);
  div3[q] = div3l;
  R omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
  R omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
  if (do_sensor) {
    // sensor_subroutine works from the stored |omega| and div/3
    R om = sqrt(omod2);
    R om2 = om * om;
    R dv = R(3) * div3l;
    R u0l0 = R(g.u0 / g.l0);
    R t = fmax(-dv / sqrt(om2 + dv * dv + u0l0 * u0l0), R(0));
    sensor_next[q] = double(t * t);
  }
  R sig11 = ux - R(2) * div3l, sig12 = vx, sig13 = wx;
  R sig21 = uy, sig22 = vy - R(2) * div3l, sig23 = wy;
  R sig31 = uz, sig32 = vz, sig33 = wz - R(2) * div3l;
  R sigx = mux * sig11 + muy * sig12 + muz * sig13;
  R sigy = mux * sig21 + muy * sig22 + muz * sig23;
  R sigz = mux * sig31 + muy * sig32 + muz * sig33;
  R sigah = (sig11 * ux + sig12 * uy + sig13 * uz + sig21 * vx + sig22 * vy + sig23 * vz + sig31 * wx +
             sig32 * wy + sig33 * wz) * mu;
  R sigq = sigx * uu + sigy * vv + sigz * ww + sigah;
  double f2 = fl[nI + q], f3 = fl[2 * nI + q], f4 = fl[3 * nI + q], f5 = fl[4 * nI + q];
  f2 = f2 - double(sigx);
  f3 = f3 - double(sigy);
  f4 = f4 - double(sigz);
  f5 = f5 - double(sigq);
  // conservative face Laplacian: face sigma between points a (lower) and b (upper)
  auto face = [&](long long a, long long b, double d, double (&s)[4]) {
    R u1 = A(a, 2), u2 = A(b, 2), v1 = A(a, 3), v2 = A(b, 3), w1 = A(a, 4), w2 = A(b, 4);
    R t1 = A(a, 6), t2 = A(b, 6), m1 = A(a, 7), m2 = A(b, 7);
    R qq1 = R(0.5) * (u1 * u1 + v1 * v1 + w1 * w1);
    R qq2 = R(0.5) * (u2 * u2 + v2 * v2 + w2 * w2);
    R muf = m1 + m2;
    muf = R(0.5) * muf / R(d);
    s[0] = double((u2 - u1) * muf);
    s[1] = double((v2 - v1) * muf);
    s[2] = double((w2 - w1) * muf);
    const R cpf = TP ? R(cp_of_t(g, double(R(0.5) * (t1 + t2)))) : R(g.cp0);
    s[3] = double(((t2 - t1) * cpf / prandtl + (qq2 - qq1)) * muf);
  };
  double lo[4], hi[4];
  // x: fl += dxhl*(fhat(i) - fhat(i-1)), fhat = -sigma
  face(c - sX, c, g.x[i] - g.x[i - 1], lo);
  face(c, c + sX, g.x[i + 1] - g.x[i], hi);
  double dxhl = __ldg(g.vhl[0] + i);  // 2/(x(i+1)-x(i-1))
  f2 = f2 + dxhl * (-hi[0] - -lo[0]);
  f3 = f3 + dxhl * (-hi[1] - -lo[1]);
  f4 = f4 + dxhl * (-hi[2] - -lo[2]);
  f5 = f5 + dxhl * (-hi[3] - -lo[3]);
  // y: fl = (fl + sigma(j-1/2)*dyhl) - sigma(j+1/2)*dyhl
  face(c - sY, c, g.y[j] - g.y[j - 1], lo);
  face(c, c + sY, g.y[j + 1] - g.y[j], hi);
  double dyhl = __ldg(g.vhl[1] + j);
  f2 = f2 + lo[0] * dyhl - hi[0] * dyhl;
  f3 = f3 + lo[1] * dyhl - hi[1] * dyhl;
  f4 = f4 + lo[2] * dyhl - hi[2] * dyhl;
  f5 = f5 + lo[3] * dyhl - hi[3] * dyhl;
  face(c - sZ, c, g.z[k] - g.z[k - 1], lo);
  face(c, c + sZ, g.z[k + 1] - g.z[k], hi);
  double dzhl = __ldg(g.vhl[2] + k);
  f2 = f2 + lo[0] * dzhl - hi[0] * dzhl;
  f3 = f3 + lo[1] * dzhl - hi[1] * dzhl;
  f4 = f4 + lo[2] * dzhl - hi[2] * dzhl;
  f5 = f5 + lo[3] * dzhl - hi[3] * dzhl;
  fl[nI + q] = f2;
  fl[2 * nI + q] = f3;
  fl[3 * nI + q] = f4;
  fl[4 * nI + q] = f5;
}
// The same viscous pass with its operands staged in shared memory: a block of 32 x 8 threads
// owns a 32 x 8 column of cells and marches VT_K cells along z; the five fields the pass reads
// (u, v, w, T, mu) of the planes k-1, k, k+1 sit in a ring of three tiles of 34 x 10 points (the
// column and its x / y halo), so that every point is loaded once per block (and its halo once
// more) with coalesced rows instead of once per use, and the x / y / z neighbours come from
// shared memory.  The arithmetic is d_visc's, in its order.
#ifndef SB_VT_K
#define SB_VT_K 16
#endif
constexpr int VT_X = 32, VT_Y = 8, VT_NT = VT_X * VT_Y, VT_K = SB_VT_K;
constexpr int VT_PX = VT_X + 2, VT_PY = VT_Y + 2, VT_PP = VT_PX * VT_PY;
// blocks of the staged viscous pass: 32 x 8 columns x segments of VT_K cells in z
inline unsigned visc_tiled_blocks(const Geom& g) {
  return (unsigned)((g.nx + VT_X - 1) / VT_X) * (unsigned)((g.ny + VT_Y - 1) / VT_Y) *
         (unsigned)((g.nz + VT_K - 1) / VT_K);
}
template <class R, bool TP = false>
__device__ __forceinline__ void d_visc_tiled(const Geom& g, const R* __restrict__ aux, double* __restrict__ fl,
                                             R* __restrict__ div3, double* __restrict__ sensor_next,
                                             double* __restrict__ wallprop, int do_sensor, const Blk blk) {
  __shared__ R pl[3][5][VT_PP];
  const unsigned nbx = (unsigned)(g.nx + VT_X - 1) / VT_X, nby = (unsigned)(g.ny + VT_Y - 1) / VT_Y;
  const unsigned bx = blk.x % nbx, rest = blk.x / nbx, by = rest % nby, bk = rest / nby;
  const int tx = (int)threadIdx.x % VT_X, ty = (int)threadIdx.x / VT_X;
  const int i0 = (int)bx * VT_X, j0 = (int)by * VT_Y;  // the tile's points are i0 .. i0+VT_X+1
  const int i = i0 + 1 + tx, j = j0 + 1 + ty;
  const bool own = i <= g.nx && j <= g.ny;
  const int k0 = (int)bk * VT_K + 1, k1 = min(k0 + VT_K - 1, g.nz);
  const long long n = g.nvol, nI = g.nint;
  // plane k of the tile into slot k % 3 (points beyond the face ghosts are left unread: no cell
  // of the column uses them)
  auto load_plane = [&](int k) {
    R(*dst)[VT_PP] = pl[k % 3];
    for (int t = threadIdx.x; t < VT_PP; t += VT_NT) {
      const int ii = i0 + t % VT_PX, jj = j0 + t / VT_PX;
      if (ii <= g.nx + 1 && jj <= g.ny + 1) {
        const long long a = gidx(g, ii, jj, k);
        dst[0][t] = __ldg(aux + n + a);
        dst[1][t] = __ldg(aux + 2 * n + a);
        dst[2][t] = __ldg(aux + 3 * n + a);
        dst[3][t] = __ldg(aux + 5 * n + a);
        dst[4][t] = __ldg(aux + 6 * n + a);
      }
    }
  };
  load_plane(k0 - 1);
  load_plane(k0);
  const R prandtl = R(g.prandtl);
  R dxl = R(0), dyl = R(0);
  if (own) {
    if constexpr (sizeof(R) == sizeof(double)) {
      dxl = R(__ldg(g.vrl[0] + i)); dyl = R(__ldg(g.vrl[1] + j));
    } else {
      dxl = R(__ldg(g.vrlf[0] + i)); dyl = R(__ldg(g.vrlf[1] + j));
    }
  }
  for (int k = k0; k <= k1; ++k) {
    load_plane(k + 1);
    __syncthreads();
    if (own) {
      const int sm = (k - 1) % 3, s0 = k % 3, sp = (k + 1) % 3;
      const int c0 = (tx + 1) + (ty + 1) * VT_PX;
      // field f (0 u, 1 v, 2 w, 3 T, 4 mu) at the cell's point offset by (di, dj) in plane slot sl
      auto F = [&](int sl, int di, int dj, int f) -> R { return pl[sl][f][c0 + di + dj * VT_PX]; };
      const long long q = iidx(g, i, j, k);
      const R uu = F(s0, 0, 0, 0), vv = F(s0, 0, 0, 1), ww = F(s0, 0, 0, 2), mu = F(s0, 0, 0, 4);
      const R cploc = TP ? R(cp_of_t(g, double(F(s0, 0, 0, 3)))) : R(g.cp0);
      R dzl;
      if constexpr (sizeof(R) == sizeof(double)) dzl = R(__ldg(g.vrl[2] + k));
      else dzl = R(__ldg(g.vrlf[2] + k));
      R ux = dxl * (F(s0, 1, 0, 0) - F(s0, -1, 0, 0));
      R vx = dxl * (F(s0, 1, 0, 1) - F(s0, -1, 0, 1));
      R wx = dxl * (F(s0, 1, 0, 2) - F(s0, -1, 0, 2));
      R mux = dxl * (F(s0, 1, 0, 4) - F(s0, -1, 0, 4));
      R uy = dyl * (F(s0, 0, 1, 0) - F(s0, 0, -1, 0));
      R vy = dyl * (F(s0, 0, 1, 1) - F(s0, 0, -1, 1));
      R wy = dyl * (F(s0, 0, 1, 2) - F(s0, 0, -1, 2));
      R ty_ = dyl * (F(s0, 0, 1, 3) - F(s0, 0, -1, 3));
      R muy = dyl * (F(s0, 0, 1, 4) - F(s0, 0, -1, 4));
      R uz = dzl * (F(sp, 0, 0, 0) - F(sm, 0, 0, 0));
      R vz = dzl * (F(sp, 0, 0, 1) - F(sm, 0, 0, 1));
      R wz = dzl * (F(sp, 0, 0, 2) - F(sm, 0, 0, 2));
      R muz = dzl * (F(sp, 0, 0, 4) - F(sm, 0, 0, 4));
      if (j == 1) {
        const long long wp = (long long)(k - 1) * g.nx + (i - 1);
        const long long nw = (long long)g.nx * g.nz;
        wallprop[wp] = double(mu * uy);
        wallprop[nw + wp] = double(mu * wy);
        wallprop[2 * nw + wp] = double(mu * ty_ * cploc / prandtl);
      }
      R div = ux + vy + wz;
      R div3l = div / R(3);
      div3[q] = div3l;
      R omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
      R omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
      if (do_sensor) {
        R om = sqrt(omod2);
        R om2 = om * om;
        R dv = R(3) * div3l;
        R u0l0 = R(g.u0 / g.l0);
        R t = fmax(-dv / sqrt(om2 + dv * dv + u0l0 * u0l0), R(0));
        sensor_next[q] = double(t * t);
      }
      R sig11 = ux - R(2) * div3l, sig12 = vx, sig13 = wx;
      R sig21 = uy, sig22 = vy - R(2) * div3l, sig23 = wy;
      R sig31 = uz, sig32 = vz, sig33 = wz - R(2) * div3l;
      R sigx = mux * sig11 + muy * sig12 + muz * sig13;
      R sigy = mux * sig21 + muy * sig22 + muz * sig23;
      R sigz = mux * sig31 + muy * sig32 + muz * sig33;
      R sigah = (sig11 * ux + sig12 * uy + sig13 * uz + sig21 * vx + sig22 * vy + sig23 * vz + sig31 * wx +
                 sig32 * wy + sig33 * wz) * mu;
      R sigq = sigx * uu + sigy * vv + sigz * ww + sigah;
      double f2 = fl[nI + q], f3 = fl[2 * nI + q], f4 = fl[3 * nI + q], f5 = fl[4 * nI + q];
      f2 = f2 - double(sigx);
      f3 = f3 - double(sigy);
      f4 = f4 - double(sigz);
      f5 = f5 - double(sigq);
      // conservative face Laplacian: face sigma between points a (lower) and b (upper)
      auto face = [&](int sla, int dia, int dja, int slb, int dib, int djb, double d, double (&sf)[4]) {
        R u1 = F(sla, dia, dja, 0), u2 = F(slb, dib, djb, 0), v1 = F(sla, dia, dja, 1), v2 = F(slb, dib, djb, 1);
        R w1 = F(sla, dia, dja, 2), w2 = F(slb, dib, djb, 2);
        R t1 = F(sla, dia, dja, 3), t2 = F(slb, dib, djb, 3), m1 = F(sla, dia, dja, 4), m2 = F(slb, dib, djb, 4);
        R qq1 = R(0.5) * (u1 * u1 + v1 * v1 + w1 * w1);
        R qq2 = R(0.5) * (u2 * u2 + v2 * v2 + w2 * w2);
        R muf = m1 + m2;
        muf = R(0.5) * muf / R(d);
        sf[0] = double((u2 - u1) * muf);
        sf[1] = double((v2 - v1) * muf);
        sf[2] = double((w2 - w1) * muf);
        const R cpf = TP ? R(cp_of_t(g, double(R(0.5) * (t1 + t2)))) : R(g.cp0);
        sf[3] = double(((t2 - t1) * cpf / prandtl + (qq2 - qq1)) * muf);
      };
      double lo[4], hi[4];
      face(s0, -1, 0, s0, 0, 0, g.x[i] - g.x[i - 1], lo);
      face(s0, 0, 0, s0, 1, 0, g.x[i + 1] - g.x[i], hi);
      double dxhl = __ldg(g.vhl[0] + i);
      f2 = f2 + dxhl * (-hi[0] - -lo[0]);
      f3 = f3 + dxhl * (-hi[1] - -lo[1]);
      f4 = f4 + dxhl * (-hi[2] - -lo[2]);
      f5 = f5 + dxhl * (-hi[3] - -lo[3]);
      face(s0, 0, -1, s0, 0, 0, g.y[j] - g.y[j - 1], lo);
      face(s0, 0, 0, s0, 0, 1, g.y[j + 1] - g.y[j], hi);
      double dyhl = __ldg(g.vhl[1] + j);
      f2 = f2 + lo[0] * dyhl - hi[0] * dyhl;
      f3 = f3 + lo[1] * dyhl - hi[1] * dyhl;
      f4 = f4 + lo[2] * dyhl - hi[2] * dyhl;
      f5 = f5 + lo[3] * dyhl - hi[3] * dyhl;
      face(sm, 0, 0, s0, 0, 0, g.z[k] - g.z[k - 1], lo);
      face(s0, 0, 0, sp, 0, 0, g.z[k + 1] - g.z[k], hi);
      double dzhl = __ldg(g.vhl[2] + k);
      f2 = f2 + lo[0] * dzhl - hi[0] * dzhl;
      f3 = f3 + lo[1] * dzhl - hi[1] * dzhl;
      f4 = f4 + lo[2] * dzhl - hi[2] * dzhl;
      f5 = f5 + lo[3] * dzhl - hi[3] * dzhl;
      fl[nI + q] = f2;
      fl[2 * nI + q] = f3;
      fl[3 * nI + q] = f4;
      fl[4 * nI + q] = f5;
    }
    __syncthreads();  // the slot of plane k-1 is overwritten by plane k+2 next
  }
}
template <class R, bool TP = false>
__global__ void __launch_bounds__(VT_NT, sizeof(R) == 8 ? VISC_MINB : VISC_MINB_F)
    k_visc_tiled(Geom g, const R* __restrict__ aux, double* __restrict__ fl, R* __restrict__ div3,
                 double* __restrict__ sensor_next, double* __restrict__ wallprop, int do_sensor) {
  d_visc_tiled<R, TP>(g, aux, fl, div3, sensor_next, wallprop, do_sensor, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

template <class R, bool TP = false>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? VISC_MINB : VISC_MINB_F) k_visc(Geom g, const R* __restrict__ aux, double* __restrict__ fl,
                                              R* __restrict__ div3, double* __restrict__ sensor_next,
                                              double* __restrict__ wallprop, int do_sensor) {
  d_visc<R, TP>(g, aux, fl, div3, sensor_next, wallprop, do_sensor, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

// visflx_nosensor_subroutine (kernels_cpu.F90:3996-4180), the non-conservative viscous form of
// conservative_viscous = 0: first and second derivatives of u, v, w, T (and first of mu) with the
// central stencil of order visc_order, the full stress divergence and dissipation, heat flux;
// div/3 and |omega| for the div term and the stage-3 sensor (sensor_subroutine,
// kernels_cpu.F90:4726-4744, from |omega| and div/3), wall shear at j = 1.  Arithmetic in R,
// accumulation into the FP64 register.
template <class R, bool TP = false>
__device__ __forceinline__ void d_visc_ns(const Geom& g, const R* __restrict__ aux, double* __restrict__ fl,
                                                 R* __restrict__ div3, double* __restrict__ sensor_next,
                                                 double* __restrict__ wallprop, int do_sensor, const Blk blk) {
  const long long q = (long long)blk.x * 256 + threadIdx.x;
  if (q >= g.nint) return;
  int i, j, k;
  cell_of(g, q, i, j, k);
  const long long n = g.nvol, nI = g.nint;
  const long long c = gidx(g, i, j, k);
  const long long st[3] = {1, g.sx, (long long)g.sx * g.sy};
  auto A = [&](long long a, int m) -> R { return __ldg(aux + (m - 1) * n + a); };
  const int lmax = g.lmax_base;
  const R uu = A(c, 2), vv = A(c, 3), ww = A(c, 4), tt = A(c, 6), mu = A(c, 7);
  // d[dir][var]: first derivative of u, v, w, T, mu; lap[dir][var]: second derivative of u, v, w, T
  R d1[3][5], lap[3][4];
  const R c20 = R(g.coeff2[lmax - 1][0]);
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
#pragma unroll
    for (int v = 0; v < 5; ++v) d1[dir][v] = R(0);
    lap[dir][0] = c20 * uu; lap[dir][1] = c20 * vv; lap[dir][2] = c20 * ww; lap[dir][3] = c20 * tt;
    for (int l = 1; l <= lmax; ++l) {
      const R ccl = R(g.coeff[lmax - 1][l - 1]);
      const R clapl = R(g.coeff2[lmax - 1][l]);
      const long long ap = c + l * st[dir], am = c - l * st[dir];
      const int ms[5] = {2, 3, 4, 6, 7};
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const R fp = A(ap, ms[v]), fm = A(am, ms[v]);
        d1[dir][v] = d1[dir][v] + ccl * (fp - fm);
        if (v < 4) lap[dir][v] = lap[dir][v] + clapl * (fp + fm);
      }
    }
  }
  const R m1[3] = {R(g.dcsidx[i]), R(g.detady[j]), R(g.dzitdz[k])};
  const R ms2[3] = {R(g.dcsidxs[i]), R(g.detadys[j]), R(g.dzitdzs[k])};
  const R m2[3] = {R(g.dcsidx2[i]), R(g.detady2[j]), R(g.dzitdz2[k])};
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
#pragma unroll
    for (int v = 0; v < 5; ++v) d1[dir][v] = d1[dir][v] * m1[dir];
#pragma unroll
    for (int v = 0; v < 4; ++v) lap[dir][v] = lap[dir][v] * ms2[dir] + d1[dir][v] * m2[dir];
  }
  const R ux = d1[0][0], vx = d1[0][1], wx = d1[0][2], tx = d1[0][3], mux = d1[0][4];
  const R uy = d1[1][0], vy = d1[1][1], wy = d1[1][2], ty = d1[1][3], muy = d1[1][4];
  const R uz = d1[2][0], vz = d1[2][1], wz = d1[2][2], tz = d1[2][3], muz = d1[2][4];
  const R ulap = lap[0][0] + lap[1][0] + lap[2][0];
  const R vlap = lap[0][1] + lap[1][1] + lap[2][1];
  const R wlap = lap[0][2] + lap[1][2] + lap[2][2];
  const R tlap = lap[0][3] + lap[1][3] + lap[2][3];
  const R div = ux + vy + wz;
  const R div3l = div / R(3);
  div3[q] = div3l;
  const R omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
  const R omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
  if (do_sensor) {
    const R om = sqrt(omod2);
    const R om2 = om * om;
    const R dv = R(3) * div3l;
    const R u0l0 = R(g.u0 / g.l0);
    const R t = fmax(-dv / sqrt(om2 + dv * dv + u0l0 * u0l0), R(0));
    sensor_next[q] = double(t * t);
  }
  const R cploc = TP ? R(cp_of_t(g, double(A(c, 6)))) : R(g.cp0), prandtl = R(g.prandtl);
  const R sig11 = R(2) * (ux - div3l), sig12 = uy + vx, sig13 = uz + wx;
  const R sig22 = R(2) * (vy - div3l), sig23 = vz + wy, sig33 = R(2) * (wz - div3l);
  const R sigx = mux * sig11 + muy * sig12 + muz * sig13 + mu * ulap;
  const R sigy = mux * sig12 + muy * sig22 + muz * sig23 + mu * vlap;
  const R sigz = mux * sig13 + muy * sig23 + muz * sig33 + mu * wlap;
  const R sigqt = (mux * tx + muy * ty + muz * tz + mu * tlap) * cploc / prandtl;
  const R sigah = (sig11 * ux + sig12 * uy + sig13 * uz + sig12 * vx + sig22 * vy + sig23 * vz + sig13 * wx +
                   sig23 * wy + sig33 * wz) * mu;
  const R sigq = sigx * uu + sigy * vv + sigz * ww + sigah + sigqt;
  fl[nI + q] = fl[nI + q] - double(sigx);
  fl[2 * nI + q] = fl[2 * nI + q] - double(sigy);
  fl[3 * nI + q] = fl[3 * nI + q] - double(sigz);
  fl[4 * nI + q] = fl[4 * nI + q] - double(sigq);
  if (j == 1) {
    const long long wp = (long long)(k - 1) * g.nx + (i - 1);
    const long long nw = (long long)g.nx * g.nz;
    wallprop[wp] = double(mu * uy);
    wallprop[nw + wp] = double(mu * wy);
    wallprop[2 * nw + wp] = double(mu * ty * cploc / prandtl);
  }
}
template <class R, bool TP = false>
__global__ void __launch_bounds__(256) k_visc_ns(Geom g, const R* __restrict__ aux, double* __restrict__ fl,
                                                 R* __restrict__ div3, double* __restrict__ sensor_next,
                                                 double* __restrict__ wallprop, int do_sensor) {
  d_visc_ns<R, TP>(g, aux, fl, div3, sensor_next, wallprop, do_sensor, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

// Initial Ducros sensor of run() (visflx(mode=2), singleideal_cpu.F90:1550-1555):
// visflx_reduced_ord2 with update_sensor = 1 (kernels_cpu.F90:4680-4682)
template <class R>
__device__ __forceinline__ void d_init_sensor(const Geom& g, const R* __restrict__ aux,
                                                     double* __restrict__ sensor, const Blk blk) {
  const long long q = (long long)blk.x * 256 + threadIdx.x;
  if (q >= g.nint) return;
  int i, j, k;
  cell_of(g, q, i, j, k);
  const long long n = g.nvol, c = gidx(g, i, j, k), sY = g.sx, sZ = (long long)g.sx * g.sy;
  auto A = [&](long long a, int m) -> R { return aux[(m - 1) * n + a]; };
  R dxl = R(1) / R(g.x[i + 1] - g.x[i - 1]);
  R dyl = R(1) / R(g.y[j + 1] - g.y[j - 1]);
  R dzl = R(1) / R(g.z[k + 1] - g.z[k - 1]);
  R ux = dxl * (A(c + 1, 2) - A(c - 1, 2));
  R vx = dxl * (A(c + 1, 3) - A(c - 1, 3));
  R wx = dxl * (A(c + 1, 4) - A(c - 1, 4));
  R uy = dyl * (A(c + sY, 2) - A(c - sY, 2));
  R vy = dyl * (A(c + sY, 3) - A(c - sY, 3));
  R wy = dyl * (A(c + sY, 4) - A(c - sY, 4));
  R uz = dzl * (A(c + sZ, 2) - A(c - sZ, 2));
  R vz = dzl * (A(c + sZ, 3) - A(c - sZ, 3));
  R wz = dzl * (A(c + sZ, 4) - A(c - sZ, 4));
  R div = ux + vy + wz;
  R omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
  R omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
  R u0l0 = R(g.u0 / g.l0);
  R t = fmax(-div / sqrt(omod2 + div * div + u0l0 * u0l0), R(0));
  sensor[q] = double(t * t);
}
template <class R>
__global__ void __launch_bounds__(256) k_init_sensor(Geom g, const R* __restrict__ aux,
                                                     double* __restrict__ sensor) {
  d_init_sensor<R>(g, aux, sensor, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

// compute_dt_subroutine (kernels_cpu.F90:6814-6880): block maxima of the 9 inverse time scales.
// The FP64 form reads the primitive fields; the mixed form recomputes them from w in FP64.
template <class R>
__device__ __forceinline__ void d_dt(const Geom& g, const double* __restrict__ w, const R* __restrict__ aux,
                                            double* __restrict__ red, const Blk blk) {
  __shared__ double sm[9 * 8];
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
  for (int cq = 0; cq < PT_CELLS; ++cq) {
    const long long q = (long long)blk.x * (256 * PT_CELLS) + cq * 256 + threadIdx.x;
    if (q >= g.nint) break;
    int i, j, k;
    cell_of(g, q, i, j, k);
    const long long n = g.nvol, c = gidx(g, i, j, k);
    double rho = w[c];
    double ri = 1.0 / rho;
    double uu, vv, ww, tt, mu;
    if constexpr (sizeof(R) == sizeof(double)) {
      uu = aux[n + c]; vv = aux[2 * n + c]; ww = aux[3 * n + c]; tt = aux[5 * n + c]; mu = aux[6 * n + c];
    } else {
      const Prim p = prim_from_w<false>(g, w, c, g.t0);  // mixed form only: calorically perfect
      uu = p.uu; vv = p.vv; ww = p.ww; tt = p.tt; mu = viscosity(g, tt);
    }
    double nu = ri * mu;
    double kr = nu / g.prandtl;
    double cs = sqrt(gamloc_of_t(g, tt) * g.rgas0 * tt);
    v[0] = fmax(v[0], (fabs(uu) + cs) * g.dcsidx[i]);
    v[1] = fmax(v[1], (fabs(vv) + cs) * g.detady[j]);
    v[2] = fmax(v[2], (fabs(ww) + cs) * g.dzitdz[k]);
    v[3] = fmax(v[3], nu * g.dcsidxs[i]);
    v[4] = fmax(v[4], nu * g.detadys[j]);
    v[5] = fmax(v[5], nu * g.dzitdzs[k]);
    v[6] = fmax(v[6], kr * g.dcsidxs[i]);
    v[7] = fmax(v[7], kr * g.detadys[j]);
    v[8] = fmax(v[8], kr * g.dzitdzs[k]);
  }
#pragma unroll
  for (int r = 0; r < 9; ++r)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[r] = fmax(v[r], __shfl_down_sync(0xffffffffu, v[r], o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int r = 0; r < 9; ++r) sm[r * 8 + warp] = v[r];
  __syncthreads();
  if (threadIdx.x < 9) {
    double m = 0.0;
    for (int wq = 0; wq < 8; ++wq) m = fmax(m, sm[threadIdx.x * 8 + wq]);
    red[(long long)blk.x * 9 + threadIdx.x] = m;
  }
}
template <class R>
__global__ void __launch_bounds__(256, DT_MINB) k_dt(Geom g, const double* __restrict__ w, const R* __restrict__ aux,
                                            double* __restrict__ red) {
  d_dt<R>(g, w, aux, red, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

__device__ __forceinline__ void d_dt_finish(const double* __restrict__ red, long long nblk, double cfl,
                                                      Scalars* __restrict__ sc, const Blk blk) {
  __shared__ double sm[FIN_NT / 32];
  double m = 0.0;
  for (long long b = threadIdx.x; b < nblk * 9; b += FIN_NT) m = fmax(m, red[b]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int wq = 0; wq < FIN_NT / 32; ++wq) a = fmax(a, sm[wq]);
    double dt_min = 1.0 / a;
    sc->dt = cfl * dt_min;
  }
}
__global__ void __launch_bounds__(FIN_NT) k_dt_finish(const double* __restrict__ red, long long nblk, double cfl,
                                                      Scalars* __restrict__ sc) {
  d_dt_finish(red, nblk, cfl, sc, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

// Sum NR partials per block in a fixed order (thread-strided, then tree).
template <int NR>
__device__ __forceinline__ void finish_sums(const double* __restrict__ red, long long nblk, double (&out)[NR],
                                            double* sm) {
  double v[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) v[r] = 0.0;
  for (long long b = threadIdx.x; b < nblk; b += FIN_NT)
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = v[r] + red[b * NR + r];
  block_reduce_sum<NR, FIN_NT>(v, sm);
#pragma unroll
  for (int r = 0; r < NR; ++r) out[r] = v[r];
}

// force_rhs (singleideal_cpu.F90:845-889): bulk values from the partials
__device__ __forceinline__ void d_finish_rhs(const Geom& g, const double* __restrict__ red, long long nblk,
                                                       int first_stage, Scalars* __restrict__ sc, const Blk blk) {
  __shared__ double sm[5 * (FIN_NT / 32)];
  double b[5];
  finish_sums<5>(red, nblk, b, sm);
  if (threadIdx.x == 0) {
    for (int r = 0; r < 5; ++r) b[r] = b[r] / g.volchan;
    double dpdx = first_stage ? 0.0 : sc->dpdx;
    sc->dpdx = dpdx + b[1];
    sc->rhobulk = b[2];
    sc->ubulk = b[3] / sc->rhobulk;
    sc->tbulk = b[4] / sc->rhobulk / sc->ubulk;
    for (int r = 0; r < 5; ++r) sc->bulk[r] = b[r];
  }
}
__global__ void __launch_bounds__(FIN_NT) k_finish_rhs(Geom g, const double* __restrict__ red, long long nblk,
                                                       int first_stage, Scalars* __restrict__ sc) {
  d_finish_rhs(g, red, nblk, first_stage, sc, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

// update_flux + force_rhs_2 + update_field (kernels_cpu.F90:3400-3442, 3092-3116) and the
// partials of force_var_1 (:3241-3282) and of compute_residual / minmax (:6682-6810).  All FP64;
// the primitive values of the stage's starting state are recomputed from w as eval_aux does.
template <class R, bool TP = false>
__device__ __forceinline__ void d_update(const Geom& g, double* __restrict__ w, const double* __restrict__ fl_prev,
                                                const double* __restrict__ fl_new, const Scalars* __restrict__ sc,
                                                double rhork, double gamrk, int istep, int stats,
                                                double* __restrict__ red, const double* __restrict__ sensor_next,
                                                double* __restrict__ sensor, R* __restrict__ aux, const Blk blk) {
  constexpr int NW = UPD_NT / 32;
  __shared__ double sm[2 * NW];
  __shared__ double smn[3 * NW];
  __shared__ double smx[3 * NW];
  double s2[2] = {0.0, 0.0};
  double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
  double mx[3] = {-100.0, -100.0, -100.0};
  const long long q = (long long)blk.x * UPD_NT + threadIdx.x;
  if (q < g.nint) {
    int i, j, k;
    cell_of(g, q, i, j, k);
    const long long n = g.nvol, nI = g.nint, c = gidx(g, i, j, k);
    const double dt = sc->dt;
    const double rhodt = rhork * dt, gamdt = gamrk * dt;
    // the stage's starting temperature is in aux (Newton start of the thermally perfect gas)
    const double t_aux = TP ? double(aux[5 * n + c]) : g.t0;
    const Prim old = prim_from_w<TP>(g, w, c, t_aux);
    double fln[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      double a = istep > 1 ? -(rhodt * fl_prev[m * nI + q]) : 0.0;
      fln[m] = a - gamdt * fl_new[m * nI + q];
    }
    if (g.channel_case) {
      const double b1 = sc->bulk[0], b2 = sc->bulk[1];
      fln[0] = fln[0] - b1;
      fln[1] = fln[1] - b2;
      fln[4] = fln[4] - old.uu * b2;
    }
    double wn[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      wn[m] = w[m * n + c] + fln[m];
      w[m * n + c] = wn[m];
    }
    // the stage-3 sensor becomes current once every flux of the stage has used the old one
    if (istep == 3) sensor[q] = sensor_next[q];
    double tstat = old.tt;
    if (g.force_var) {
      double dy = g.yn[j + 1] - g.yn[j];
      double ri = 1.0 / wn[0];
      double uu = wn[1] * ri, vv = wn[2] * ri, ww = wn[3] * ri;
      double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
      double ee = wn[4] / wn[0] - qq;
      double tt = t_from_e<TP>(g, ee, t_aux);
      s2[0] = s2[0] + wn[1] * tt * dy;
      tstat = tt;
      // force_var_1 leaves this temperature in w_aux(6), where the statistics read it
      if (istep == 3) aux[5 * n + c] = R(tt);
    }
    if (stats) {
      double r = fln[1] / dt;
      s2[1] = s2[1] + r * r;
      double rho = old.rho;
      double pp = rho * tstat * g.rgas0;
      mn[0] = fmin(mn[0], rho); mn[1] = fmin(mn[1], tstat); mn[2] = fmin(mn[2], pp);
      mx[0] = fmax(mx[0], rho); mx[1] = fmax(mx[1], tstat); mx[2] = fmax(mx[2], pp);
    }
  }
  // the block partials are read only by the forcing and by a stats sample (the same branch for
  // the whole grid)
  if (!g.force_var && !stats) return;
  block_reduce_sum<2, UPD_NT>(s2, sm);
  // min / max (exact, order independent)
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn[r] = fmin(mn[r], __shfl_down_sync(0xffffffffu, mn[r], o));
      mx[r] = fmax(mx[r], __shfl_down_sync(0xffffffffu, mx[r], o));
    }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int r = 0; r < 3; ++r) { smn[r * NW + warp] = mn[r]; smx[r * NW + warp] = mx[r]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double* o = red + (long long)blk.x * NRED_UPD;
    o[0] = s2[0];
    o[1] = s2[1];
    for (int r = 0; r < 3; ++r) {
      double a = DBL_MAX, b = -100.0;
      for (int wq = 0; wq < NW; ++wq) { a = fmin(a, smn[r * NW + wq]); b = fmax(b, smx[r * NW + wq]); }
      o[2 + r] = a;
      o[5 + r] = b;
    }
  }
}
template <class R, bool TP = false>
__global__ void __launch_bounds__(UPD_NT, UPD_MINB) k_update(Geom g, double* __restrict__ w, const double* __restrict__ fl_prev,
                                                const double* __restrict__ fl_new, const Scalars* __restrict__ sc,
                                                double rhork, double gamrk, int istep, int stats,
                                                double* __restrict__ red, const double* __restrict__ sensor_next,
                                                double* __restrict__ sensor, R* __restrict__ aux) {
  d_update<R, TP>(g, w, fl_prev, fl_new, sc, rhork, gamrk, istep, stats, red, sensor_next, sensor, aux, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

// force_var (singleideal_cpu.F90:890-933): energy shift for the next pass; residual and extrema
__device__ __forceinline__ void d_finish_upd(const Geom& g, const double* __restrict__ red, long long nblk,
                                                       int stats, int add_time, Scalars* __restrict__ sc, const Blk blk) {
  __shared__ double sm[2 * (FIN_NT / 32)];
  __shared__ double smn[3 * (FIN_NT / 32)], smx[3 * (FIN_NT / 32)];
  double v[2] = {0.0, 0.0};
  double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {-100.0, -100.0, -100.0};
  // k_update wrote block partials only for the forcing or a stats sample
  const long long nb = (g.force_var || stats) ? nblk : 0;
  for (long long b = threadIdx.x; b < nb; b += FIN_NT) {
    const double* o = red + b * NRED_UPD;
    v[0] = v[0] + o[0];
    v[1] = v[1] + o[1];
    for (int r = 0; r < 3; ++r) { mn[r] = fmin(mn[r], o[2 + r]); mx[r] = fmax(mx[r], o[5 + r]); }
  }
  block_reduce_sum<2, FIN_NT>(v, sm);
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn[r] = fmin(mn[r], __shfl_down_sync(0xffffffffu, mn[r], o));
      mx[r] = fmax(mx[r], __shfl_down_sync(0xffffffffu, mx[r], o));
    }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int r = 0; r < 3; ++r) { smn[r * (FIN_NT / 32) + warp] = mn[r]; smx[r * (FIN_NT / 32) + warp] = mx[r]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (g.force_var) {
      double bulktg = v[0] / g.volchan;
      bulktg = bulktg / sc->rhobulk / sc->ubulk;
      sc->tbdiff = g.t_bulk_target - bulktg;
      sc->pending_shift = 1;
    }
    if (stats) {
      sc->residual_sum = v[1];
      double a[3], b[3];
      for (int r = 0; r < 3; ++r) {
        a[r] = DBL_MAX; b[r] = -100.0;
        for (int wq = 0; wq < FIN_NT / 32; ++wq) {
          a[r] = fmin(a[r], smn[r * (FIN_NT / 32) + wq]);
          b[r] = fmax(b[r], smx[r * (FIN_NT / 32) + wq]);
        }
      }
      sc->rhomin = a[0]; sc->tmin = a[1]; sc->pmin = a[2];
      sc->rhomax = b[0]; sc->tmax = b[1]; sc->pmax = b[2];
      if (!(v[1] == v[1])) sc->nan_flag = 1;
    }
    if (add_time) sc->time = sc->time + sc->dt;
  }
}
__global__ void __launch_bounds__(FIN_NT) k_finish_upd(Geom g, const double* __restrict__ red, long long nblk,
                                                       int stats, int add_time, Scalars* __restrict__ sc) {
  d_finish_upd(g, red, nblk, stats, add_time, sc, Blk{blockIdx.x, blockIdx.y, blockIdx.z});
}

__global__ void k_add_time(Scalars* sc) { sc->time = sc->time + sc->dt; }

// count_weno_subroutine (kernels_cpu.F90:52-113): number of faces whose stencil sees the sensor
__global__ void __launch_bounds__(256) k_count_weno(Geom g, const double* __restrict__ sensor, double* red) {
  __shared__ double sm[3 * 8];
  const long long q = (long long)blockIdx.x * 256 + threadIdx.x;
  double v[3] = {0.0, 0.0, 0.0};
  if (q < g.nint) {
    int i, j, k;
    cell_of(g, q, i, j, k);
    const int ws = g.weno_scheme;
    const double thr = g.sensor_threshold;
    if (i >= g.eul_imin && i <= g.eul_imax) {
      bool s = false;
      for (int o = -ws + 1; o <= ws; ++o) s = s || sensor_at(g, sensor, i + o, j, k) > thr;
      v[0] = s ? 1.0 : 0.0;
    }
    if (j >= g.eul_jmin && j <= g.eul_jmax) {
      bool s = false;
      for (int o = -ws + 1; o <= ws; ++o) s = s || sensor_at(g, sensor, i, j + o, k) > thr;
      v[1] = s ? 1.0 : 0.0;
    }
    if (k >= g.eul_kmin && k <= g.eul_kmax) {
      bool s = false;
      for (int o = -ws + 1; o <= ws; ++o) s = s || sensor_at(g, sensor, i, j, k + o) > thr;
      v[2] = s ? 1.0 : 0.0;
    }
  }
  block_reduce_sum<3, 256>(v, sm);
  if (threadIdx.x == 0)
    for (int r = 0; r < 3; ++r) red[(long long)blockIdx.x * 3 + r] = v[r];
}

// Face (p, a, b) of direction DIR as wface_index numbers it (x (p, j, k), y (p, i, k), z (p, i, j))
// from the list kernels' thread coordinates: t0 the fastest index of that numbering (x faces: p;
// y and z faces: i), t1 the second, t2 the third.
template <int DIR>
__device__ __forceinline__ void list_face(int t0, int t1, int t2, int& p, int& a, int& b) {
  p = DIR == 0 ? t0 : (DIR == 1 ? t1 : t2);
  a = DIR == 0 ? t1 + 1 : t0 + 1;
  b = DIR == 2 ? t1 + 1 : t2 + 1;
}

// Block-aggregated append: one atomic per block reserves the entries of its faces with shk set
// (the order of a list does not matter, every entry is computed independently).  Returns the
// entry of this thread (any value when !shk).  All threads of the block call it; successive
// calls alternate between the two halves of wsum (2 x warps) and base (2), so that a call
// needs no barrier after its last read.
__device__ __forceinline__ unsigned block_append(bool shk, unsigned* counter, unsigned* wsum, unsigned* base,
                                                 int par) {
  const int nw = (int)(blockDim.x >> 5);
  unsigned* ws = wsum + par * nw;
  const unsigned bal = __ballot_sync(0xffffffffu, shk);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) ws[wid] = (unsigned)__popc(bal);
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned tot = 0;
    for (int q = 0; q < nw; ++q) {
      const unsigned cq = ws[q];
      ws[q] = tot;
      tot += cq;
    }
    base[par] = tot ? atomicAdd(counter, tot) : 0u;
  }
  __syncthreads();
  return base[par] + ws[wid] + (unsigned)__popc(bal & ((1u << lane) - 1u));
}

constexpr int WL_NT = 256;  // list kernels: 32 faces along t0 x 8 along t1

// The sample count of direction DIR: the WENO faces (stencil sees the sensor, eul range) of the
// planes t2 = 0, WSAMPLE, 2 WSAMPLE, ... read from the sensor itself, into wcount[4 + DIR].
template <int DIR, int WS>
__global__ void __launch_bounds__(WL_NT) k_weno_sample(Geom g, const double* __restrict__ sensor) {
  __shared__ unsigned wsum[2 * (WL_NT / 32)];
  __shared__ unsigned base[2];
  const int t0 = blockIdx.x * 32 + (threadIdx.x & 31), t1 = blockIdx.y * 8 + (threadIdx.x >> 5);
  const int t2 = blockIdx.z * WSAMPLE;
  int p, a, b;
  list_face<DIR>(t0, t1, t2, p, a, b);
  const int n0 = DIR == 0 ? g.nx + 1 : g.nx, n1 = DIR == 1 ? g.ny + 1 : g.ny;
  const int emin = DIR == 0 ? g.eul_imin : (DIR == 1 ? g.eul_jmin : g.eul_kmin);
  const int emax = DIR == 0 ? g.eul_imax : (DIR == 1 ? g.eul_jmax : g.eul_kmax);
  bool shk = false;
  if (t0 < n0 && t1 < n1 && p >= emin - 1 && p <= emax) {
#pragma unroll
    for (int o = -WS + 1; o <= WS; ++o) {
      const double th = DIR == 0 ? sensor_at(g, sensor, p + o, a, b)
                                 : (DIR == 1 ? sensor_at(g, sensor, a, p + o, b) : sensor_at(g, sensor, a, b, p + o));
      shk = shk || th > g.sensor_threshold;
    }
  }
  block_append(shk, g.wcount + 4 + DIR, wsum, base, 0);
}

// Whether the lists of direction DIR are built this step (its sample is within the threshold).
template <int DIR>
__device__ __forceinline__ bool list_wanted(const Geom& g) {
  return *(volatile const unsigned*)(g.wcount + 4 + DIR) <= g.wthr_s[DIR];
}

// The sensor flags of a step on the ghosted grid: sensor > threshold at interior points, the
// periodic image at the ghosts of periodic directions and 0 at the others (sensor_at).  Only
// when some direction builds its list; grid-stride over tiles of 32 x 8 points of a z plane.
__global__ void __launch_bounds__(256) k_weno_bits(Geom g, const double* __restrict__ sensor) {
  if (!list_wanted<0>(g) && !list_wanted<1>(g) && !list_wanted<2>(g)) return;
  const unsigned tx = (g.sx + 31) / 32, ty = (g.sy + 7) / 8;
  const unsigned ntile = tx * ty * (unsigned)g.sz;
  for (unsigned tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const unsigned r = tile / tx;
    const int i = (int)(tile - r * tx) * 32 + (threadIdx.x & 31) + 1 - g.ng;
    const int j = (int)(r % ty) * 8 + (threadIdx.x >> 5) + 1 - g.ng;
    const int k = (int)(r / ty) + 1 - g.ng;
    if (i <= g.nx + g.ng && j <= g.ny + g.ng)
      g.wbits[gidx(g, i, j, k)] = sensor_at(g, sensor, i, j, k) > g.sensor_threshold ? 1 : 0;
  }
}

// The WENO faces of direction DIR: the faces the hybrid pass computes (eul range) whose stencil
// sees a sensor flag, appended to the direction's list; grid-stride over tiles of 32 faces along
// t0 x 8 along t1 of one t2 plane.  A direction whose sample is above its threshold builds no
// list and marks its count as above every threshold (its hybrid pass computes the WENO faces).
template <int DIR, int WS>
__global__ void __launch_bounds__(WL_NT) k_weno_list(Geom g) {
  __shared__ unsigned wsum[2 * (WL_NT / 32)];
  __shared__ unsigned base[2];
  if (!list_wanted<DIR>(g)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) g.wcount[DIR] = 0xffffffffu;
    return;
  }
  const int n0 = DIR == 0 ? g.nx + 1 : g.nx, n1 = DIR == 1 ? g.ny + 1 : g.ny;
  const int n2 = DIR == 2 ? g.nz + 1 : g.nz;
  const unsigned tx = (unsigned)(n0 + 31) / 32, ty = (unsigned)(n1 + 7) / 8;
  const unsigned ntile = tx * ty * (unsigned)n2;
  const int emin = DIR == 0 ? g.eul_imin : (DIR == 1 ? g.eul_jmin : g.eul_kmin);
  const int emax = DIR == 0 ? g.eul_imax : (DIR == 1 ? g.eul_jmax : g.eul_kmax);
  const long long sd = DIR == 0 ? 1 : (DIR == 1 ? (long long)g.sx : (long long)g.sx * g.sy);
  int par = 0;
  for (unsigned tile = blockIdx.x; tile < ntile; tile += gridDim.x, par ^= 1) {
    const unsigned r = tile / tx;
    const int t0 = (int)(tile - r * tx) * 32 + (threadIdx.x & 31);
    const int t1 = (int)(r % ty) * 8 + (threadIdx.x >> 5);
    const int t2 = (int)(r / ty);
    int p, a, b;
    list_face<DIR>(t0, t1, t2, p, a, b);
    bool shk = false;
    if (t0 < n0 && t1 < n1 && p >= emin - 1 && p <= emax) {
      // the stencil points p-WS+1 .. p+WS of the face, all inside the ghosted grid (ng >= WS)
      const long long c = DIR == 0 ? gidx(g, p, a, b) : (DIR == 1 ? gidx(g, a, p, b) : gidx(g, a, b, p));
      const unsigned char* f = g.wbits + c;
      unsigned any = 0;
#pragma unroll
      for (int o = -WS + 1; o <= WS; ++o) any |= f[o * sd];
      shk = any != 0;
    }
    const unsigned e = block_append(shk, g.wcount + DIR, wsum, base, par);
    if (shk) g.wlist[DIR][e] = (unsigned)wface_index<DIR>(g, p, a, b);
  }
}

// The fluxes of the listed WENO faces of direction DIR into the face buffer (grid-stride over the
// list; each thread loads its face's stencil as the hybrid pass would hold it).
constexpr int WF_NT = 128;
template <class R, int DIR, int LB, int WS, int FS>
__global__ void __launch_bounds__(WF_NT) k_weno_faces(Geom g, const R* __restrict__ aux) {
  constexpr int S = LB > WS ? LB : WS;
  const unsigned cnt = g.wcount[DIR];
  if (cnt > g.wthr[DIR]) return;  // the hybrid pass computes the WENO faces itself
  const long long n = g.nvol;
  const long long sd = DIR == 0 ? 1 : (DIR == 1 ? (long long)g.sx : (long long)g.sx * g.sy);
  R* fb = static_cast<R*>(g.wface);
  for (unsigned e = blockIdx.x * WF_NT + threadIdx.x; e < cnt; e += gridDim.x * WF_NT) {
    const unsigned f = g.wlist[DIR][e];
    int p, a, b;
    wface_decode<DIR>(g, f, p, a, b);
    const long long base = DIR == 0 ? gidx(g, p, a, b) : (DIR == 1 ? gidx(g, a, p, b) : gidx(g, a, b, p));
    Stencil<R, S> st;
#pragma unroll
    for (int q = 0; q < 2 * S; ++q) load_point<R, S>(g, st, q, aux, n, base + (q - (S - 1)) * sd);
    const R* cpt = sizeof(R) == sizeof(double) ? aux + 7 * n + base - (S - 1) * sd : nullptr;
    R hi[5], lo[5];
    weno_face<R, DIR, LB, WS, S, FS>(g, st, p, hi, lo, weno_scratch<R>() + threadIdx.x, WF_NT, cpt, sd);
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      fb[m * g.nwface + f] = hi[m];
      if constexpr (sizeof(R) != sizeof(double)) fb[(5 + m) * g.nwface + f] = lo[m];
    }
  }
}

inline unsigned nblocks(long long n, int nt) { return (unsigned)((n + nt - 1) / nt); }
// blocks of the x pass: warps of 31 new faces each over the (nx+1) ny nz faces, XF_TY per block
inline unsigned x_blocks(const Geom& g) {
  const long long nface = (long long)(g.nx + 1) * g.ny * g.nz;
  return nblocks((nface + XF_TX - 2) / (XF_TX - 1), XF_TY);
}

// Segments of a march pass: enough threads to fill the device, segments of at least 16 cells
// (one redundant face per segment).
inline void march_split_with(const Geom& g, int dir, long long target, int minseg, int* seglen, int* nseg,
                             long long* nthreads) {
  const int emin = dir == 1 ? g.eul_jmin : g.eul_kmin, emax = dir == 1 ? g.eul_jmax : g.eul_kmax;
  const int ncell = emax - emin + 1;
  const long long lines = (long long)g.nx * (dir == 1 ? g.nz : g.ny);
  long long ns = (target + lines - 1) / lines;
  int sl = (int)((ncell + ns - 1) / ns);
  if (sl < minseg) sl = minseg;
  if (sl > ncell) sl = ncell;
  if (sl < 1) sl = 1;
  *seglen = sl;
  *nseg = ncell > 0 ? (ncell + sl - 1) / sl : 0;
  *nthreads = lines * *nseg;
}

inline void march_split(const Geom& g, int dir, int* seglen, int* nseg, long long* nthreads) {
  march_split_with(g, dir, g.march_threads, g.march_minseg, seglen, nseg, nthreads);
}

// typed views of the precision-dependent buffers
template <class R> R* aux_of(DevState& d);
template <> double* aux_of<double>(DevState& d) { return d.aux; }
template <> float* aux_of<float>(DevState& d) { return d.auxf; }
template <class R> R* div3_of(DevState& d);
template <> double* div3_of<double>(DevState& d) { return d.div3; }
template <> float* div3_of<float>(DevState& d) { return d.div3f; }

}  // namespace

}  // namespace sb200
