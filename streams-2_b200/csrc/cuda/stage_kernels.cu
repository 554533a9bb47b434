// Stage kernels of the B200 backend (FP64 form).
//
// One Runge-Kutta stage (rk_sync, code/src/singleideal/singleideal_cpu.F90:332-409) runs as:
//   k_aux      w -> primitive/thermo fields at interior and face-ghost points; ghost values are
//              produced on the fly (periodic wrap, staggered isothermal wall mirror), and the
//              pending force_var energy shift of the previous stage is applied to w first
//   k_euler<0> x-face hybrid fluxes + divergence (fl = ...)
//   k_visc     reduced 2nd-order viscous terms, conservative face Laplacian in x, y, z,
//              div/3, stage-3 Ducros sensor, wall shear
//   k_euler<1> y-face fluxes + divergence (fl += ...)
//   k_euler<2> z-face fluxes + divergence + grad(mu div/3) term; block partials of force_rhs
//   k_finish_rhs  bulk quantities and the forcing correction (deterministic order)
//   k_update   RK register fln, forcing correction, w += fln, force_var / residual partials
//   k_finish_upd  bulk temperature -> pending energy shift; residual and min/max
// No face flux array is stored: face fluxes live in shared memory between the face and the
// cell phases of each k_euler block.  All reductions are block partials summed in a fixed
// order, so results do not depend on scheduling.
#include <cfloat>

#include "flux.cuh"
#include "kernels.hpp"

namespace sb200 {

namespace {

constexpr int AUX_NT = 256;
constexpr int XF_TX = 32, XF_TY = 4, XF_NT = XF_TX * XF_TY;  // x faces: 4 row-warps per block
constexpr int MT_NT = 128;                                     // march kernels
constexpr int FIN_NT = 1024;

// Apply force_var_2 (kernels_cpu.F90:3285-3314) to the conserved values of one interior point:
// temperature from the (unshifted) state as force_var_1 computes it (:3241-3282), shifted by tbdiff.
__device__ __forceinline__ double shifted_rhoe(const Geom& g, double rho, double rhou, double rhov, double rhow,
                                               double rhoe, double tbdiff) {
  double ri = 1.0 / rho;
  double uu = rhou * ri, vv = rhov * ri, ww = rhow * ri;
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = rhoe / rho - qq;
  double tt = t_from_e(g, ee);
  double ttnew = tt + tbdiff;
  double en = e_from_t(g, ttnew);
  return rho * en + 0.5 * (rhou * rhou + rhov * rhov + rhow * rhow) / rho;
}

// w -> aux at all interior and face-ghost points (eval_aux_subroutine, kernels_cpu.F90:6960-7011).
// Ghost states: bcswap periodic copy (code/src/base_cpu.F90:1326-1435) and
// bcwall_staggered_subroutine (kernels_cpu.F90:6612-6678).
__global__ void __launch_bounds__(AUX_NT) k_aux(Geom g, double* __restrict__ w, double* __restrict__ aux,
                                                const Scalars* __restrict__ sc, int apply_shift,
                                                int write_ghost_w) {
  const long long n = g.nvol;
  const long long q = (long long)blockIdx.x * AUX_NT + threadIdx.x;
  if (q >= n) return;
  const int ii = (int)(q % g.sx);
  const int jj = (int)((q / g.sx) % g.sy);
  const int kk = (int)(q / ((long long)g.sx * g.sy));
  const int i = ii - g.ng + 1, j = jj - g.ng + 1, k = kk - g.ng + 1;
  const int ox = (i < 1 || i > g.nx), oy = (j < 1 || j > g.ny), oz = (k < 1 || k > g.nz);
  if (ox + oy + oz > 1) return;  // halo edges and corners are never read
  int si = i, sj = j, sk = k;
  int wall = 0;
  if (ox) si = wrap(i, g.nx);
  if (oz) sk = wrap(k, g.nz);
  if (oy) {
    if (j < 1) {
      if (g.periodic[1]) sj = j + g.ny; else { sj = 1 - j; wall = 1; }
    } else {
      if (g.periodic[1]) sj = j - g.ny; else { sj = 2 * g.ny + 1 - j; wall = 1; }
    }
  }
  const long long src = gidx(g, si, sj, sk);
  double rho = w[src], rhou = w[n + src], rhov = w[2 * n + src], rhow = w[3 * n + src], rhoe = w[4 * n + src];
  if (apply_shift) {
    rhoe = shifted_rhoe(g, rho, rhou, rhov, rhow, rhoe, sc->tbdiff);
    if (!(ox | oy | oz)) w[4 * n + src] = rhoe;
  }
  if (wall) {
    // bcwall_staggered: mirror about the wall, T_g = 2 T_w - T, p_g = p, velocity reversed
    double uu = rhou / rho, vv = rhov / rho, ww = rhow / rho;
    double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
    double ee = rhoe / rho - qq;
    double tt = t_from_e(g, ee);
    double pp = rho * tt * g.rgas0;
    tt = 2.0 * g.t_wall - tt;
    ee = e_from_t(g, tt);
    rho = pp / tt / g.rgas0;
    rhou = -rho * uu;
    rhov = -rho * vv;
    rhow = -rho * ww;
    rhoe = rho * (ee + qq);
  }
  const long long dst = gidx(g, i, j, k);
  if (write_ghost_w && (ox | oy | oz)) {
    w[dst] = rho; w[n + dst] = rhou; w[2 * n + dst] = rhov; w[3 * n + dst] = rhow; w[4 * n + dst] = rhoe;
  }
  double ri = 1.0 / rho;
  double uu = rhou * ri, vv = rhov * ri, ww = rhow * ri;
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = rhoe / rho - qq;
  double tt = t_from_e(g, ee);
  double pp = rho * tt * g.rgas0;
  aux[dst] = rho;
  aux[n + dst] = uu;
  aux[2 * n + dst] = vv;
  aux[3 * n + dst] = ww;
  aux[4 * n + dst] = (rhoe + pp) / rho;
  aux[5 * n + dst] = tt;
  aux[6 * n + dst] = viscosity(g, tt);
}

// Pending energy shift on interior points only (before a download).
__global__ void __launch_bounds__(AUX_NT) k_apply_shift(Geom g, double* __restrict__ w,
                                                        const Scalars* __restrict__ sc) {
  const long long q = (long long)blockIdx.x * AUX_NT + threadIdx.x;
  if (q >= g.nint) return;
  const int i = (int)(q % g.nx) + 1, j = (int)((q / g.nx) % g.ny) + 1, k = (int)(q / ((long long)g.nx * g.ny)) + 1;
  const long long n = g.nvol, s = gidx(g, i, j, k);
  w[4 * n + s] = shifted_rhoe(g, w[s], w[n + s], w[2 * n + s], w[3 * n + s], w[4 * n + s], sc->tbdiff);
}

// Readers of the interior-only sensor and div/3 arrays at a stencil point that may be a ghost.
__device__ __forceinline__ double sensor_at(const Geom& g, const double* __restrict__ s, int i, int j, int k) {
  if (i < 1 || i > g.nx) { if (!g.periodic[0]) return 0.0; i = wrap(i, g.nx); }
  if (j < 1 || j > g.ny) { if (!g.periodic[1]) return 0.0; j = wrap(j, g.ny); }
  if (k < 1 || k > g.nz) { if (!g.periodic[2]) return 0.0; k = wrap(k, g.nz); }
  return s[iidx(g, i, j, k)];
}
// bcextr_var (kernels_cpu.F90:6199-6254) then bcswap_var: periodic wrap, otherwise nearest interior
__device__ __forceinline__ double div3_at(const Geom& g, const double* __restrict__ d, int i, int j, int k) {
  if (i < 1 || i > g.nx) i = g.periodic[0] ? wrap(i, g.nx) : (i < 1 ? 1 : g.nx);
  if (j < 1 || j > g.ny) j = g.periodic[1] ? wrap(j, g.ny) : (j < 1 ? 1 : g.ny);
  if (k < 1 || k > g.nz) k = g.periodic[2] ? wrap(k, g.nz) : (k < 1 ? 1 : g.nz);
  return d[iidx(g, i, j, k)];
}

template <int DIR>
__device__ __forceinline__ int face_ep(const Geom& g, int p) {
  return DIR == 0 ? g.epx[p] : (DIR == 1 ? g.epy[p] : g.epz[p]);
}

// Flux at the face between (i,j,k) and its +1 neighbour along DIR.
template <int DIR, int LB, int WS>
__device__ __forceinline__ void face_flux(const Geom& g, const double* __restrict__ aux,
                                          const double* __restrict__ sensor, int i, int j, int k,
                                          double (&fh)[5]) {
  constexpr int S = LB > WS ? LB : WS;
  const int p = DIR == 0 ? i : (DIR == 1 ? j : k);
  const int nd = DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
  bool ishk = false;
#pragma unroll
  for (int o = -WS + 1; o <= WS; ++o) {
    const double th = sensor_at(g, sensor, i + (DIR == 0) * o, j + (DIR == 1) * o, k + (DIR == 2) * o);
    ishk = ishk || (th > g.sensor_threshold);
  }
  const long long n = g.nvol;
  const long long base = gidx(g, i, j, k);
  const long long stride = DIR == 0 ? 1 : (DIR == 1 ? (long long)g.sx : (long long)g.sx * g.sy);
  Stencil<double, S> st;
#pragma unroll
  for (int q = 0; q < 2 * S; ++q) {
    const long long a = base + (q - (S - 1)) * stride;
    st.rho[q] = __ldg(aux + a);
    st.u[q] = __ldg(aux + n + a);
    st.v[q] = __ldg(aux + 2 * n + a);
    st.w[q] = __ldg(aux + 3 * n + a);
    st.h[q] = __ldg(aux + 4 * n + a);
    st.t[q] = __ldg(aux + 5 * n + a);
  }
  const int ep = face_ep<DIR>(g, p);
  if (!ishk) {
    const int lmax = max(g.lmax_base + ep, 1);
    const bool zf = (p == 0 && g.fzf[2 * DIR] == 1) || (p == nd && g.fzf[2 * DIR + 1] == 1);
    central_flux<double, DIR, LB, S>(g, st, lmax, g.nkeep, zf, fh);
  } else {
    const int ord = max(WS + ep, 1);
    weno_flux<double, DIR, WS, S>(g, st, ord, fh);
  }
}

// Flux at a face from a loaded stencil window (points p-(S-1) .. p+S of face p).
template <int DIR, int LB, int WS, int S>
__device__ __forceinline__ void window_flux(const Geom& g, const Stencil<double, S>& st, bool ishk, int p,
                                            double (&fh)[5]) {
  const int nd = DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
  const int ep = face_ep<DIR>(g, p);
  if (!ishk) {
    const int lmax = max(g.lmax_base + ep, 1);
    const bool zf = (p == 0 && g.fzf[2 * DIR] == 1) || (p == nd && g.fzf[2 * DIR + 1] == 1);
    central_flux<double, DIR, LB, S>(g, st, lmax, g.nkeep, zf, fh);
  } else {
    const int ord = max(WS + ep, 1);
    weno_flux<double, DIR, WS, S>(g, st, ord, fh);
  }
}

template <int S>
__device__ __forceinline__ void load_point(Stencil<double, S>& st, int q, const double* __restrict__ aux, long long n,
                                           long long a) {
  st.rho[q] = __ldg(aux + a);
  st.u[q] = __ldg(aux + n + a);
  st.v[q] = __ldg(aux + 2 * n + a);
  st.w[q] = __ldg(aux + 3 * n + a);
  st.h[q] = __ldg(aux + 4 * n + a);
  st.t[q] = __ldg(aux + 5 * n + a);
}

// x faces: each warp owns one (j,k) row segment of 32 faces (i0-1 .. i0+30) and updates the 31
// cells between them; the upper face of a cell comes from the neighbouring lane by a shuffle,
// so no shared memory and no block barrier are needed.  fl is written (first contribution of the
// stage, euler_x after init_flux).
template <int LB, int WS>
__global__ void __launch_bounds__(XF_NT) k_xflux(Geom g, const double* __restrict__ aux,
                                                 const double* __restrict__ sensor, double* __restrict__ fl) {
  constexpr int S = LB > WS ? LB : WS;
  const int lane = threadIdx.x;
  const int j = blockIdx.y * XF_TY + threadIdx.y + 1, k = blockIdx.z + 1;
  const int i0 = blockIdx.x * (XF_TX - 1) + 1;  // first cell of the segment
  const int p = i0 - 1 + lane;                  // this lane's face (between p and p+1)
  if (j > g.ny) return;                         // whole warp leaves together
  const bool face_ok = p >= g.eul_imin - 1 && p <= g.eul_imax;
  double fh[5] = {0, 0, 0, 0, 0};
  if (face_ok) {
    bool ishk = false;
#pragma unroll
    for (int o = -WS + 1; o <= WS; ++o) ishk = ishk || sensor_at(g, sensor, p + o, j, k) > g.sensor_threshold;
    Stencil<double, S> st;
    const long long base = gidx(g, p, j, k);
#pragma unroll
    for (int q = 0; q < 2 * S; ++q) load_point<S>(st, q, aux, g.nvol, base + (q - (S - 1)));
    window_flux<0, LB, WS, S>(g, st, ishk, p, fh);
  }
  double hi[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) hi[m] = __shfl_down_sync(0xffffffffu, fh[m], 1);
  const int i = i0 + lane;  // cell between faces p and p+1
  if (lane < XF_TX - 1 && i <= g.nx) {
    const bool upd = i >= g.eul_imin && i <= g.eul_imax;
    const double met = g.dcsidx[i];
    const long long ic = iidx(g, i, j, k);
#pragma unroll
    for (int m = 0; m < 5; ++m) fl[m * g.nint + ic] = upd ? (hi[m] - fh[m]) * met : 0.0;
  }
}

// y or z faces by marching: each thread owns one line (fixed i and the other transverse index)
// over a segment of cells, keeps the stencil window of the current face in registers (one new
// point loaded per face), computes every face of the segment once and adds the divergence to fl.
// The z pass also applies the grad(mu div/3) term of visflx_div_ord2_subroutine
// (kernels_cpu.F90:3446-3480) and emits the force_rhs block partials (:3157-3193).
template <int DIR, int LB, int WS>
__global__ void __launch_bounds__(MT_NT) k_march(Geom g, const double* __restrict__ aux,
                                                 const double* __restrict__ sensor, double* __restrict__ fl,
                                                 const double* __restrict__ div3, const double* __restrict__ w,
                                                 const double* __restrict__ fl_prev, const Scalars* __restrict__ sc,
                                                 double rhork, double gamrk, int istep, int seglen, int nseg,
                                                 double* __restrict__ red) {
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
  const long long t = (long long)blockIdx.x * MT_NT + threadIdx.x;
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
    const long long sI = DIR == 1 ? (long long)g.nx : (long long)g.nx * g.ny;  // interior stride
    // sensor bits of the face p: points p-WS+1 .. p+WS at bits 0 .. 2WS-1
    auto sensor_bit = [&](int c) -> unsigned {
      double th;
      if (c < 1 || c > nd) {
        if (!g.periodic[DIR]) return 0u;
        c = wrap(c, nd);
      }
      th = DIR == 1 ? sensor[iidx(g, i, c, b)] : sensor[iidx(g, i, b, c)];
      return th > g.sensor_threshold ? 1u : 0u;
    };
    // preload the window and sensor bits of the face c0-2; the loop starts at the face c0-1
    Stencil<double, S> st;
    const int p = c0 - 2;
#pragma unroll
    for (int q = 1; q < NP; ++q) load_point<S>(st, q, aux, n, base0 + (long long)(p - (S - 1) + q) * sd);
    unsigned mask = 0;
#pragma unroll
    for (int bq = 1; bq < 2 * WS; ++bq) mask |= sensor_bit(p - WS + 1 + bq) << bq;
    double flo[5] = {0, 0, 0, 0, 0};
    for (int c = c0 - 1; c <= c1; ++c) {
      // slide the window to the face c
#pragma unroll
      for (int q = 0; q < NP - 1; ++q) {
        st.rho[q] = st.rho[q + 1]; st.u[q] = st.u[q + 1]; st.v[q] = st.v[q + 1];
        st.w[q] = st.w[q + 1]; st.h[q] = st.h[q + 1]; st.t[q] = st.t[q + 1];
      }
      load_point<S>(st, NP - 1, aux, n, base0 + (long long)(c + S) * sd);
      mask = (mask >> 1) | (sensor_bit(c + WS) << (2 * WS - 1));
      double fhi[5];
      window_flux<DIR, LB, WS, S>(g, st, mask != 0u, c, fhi);
      if (c < c0) {
#pragma unroll
        for (int m = 0; m < 5; ++m) flo[m] = fhi[m];
        continue;
      }
      // cell c lies between the faces c-1 (flo) and c (fhi)
      const long long ic = DIR == 1 ? iidx(g, i, c, b) : iidx(g, i, b, c);
      const double met = DIR == 1 ? g.detady[c] : g.dzitdz[c];
      double f[5];
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        f[m] = fl[m * nI + ic] + (fhi[m] - flo[m]) * met;
        flo[m] = fhi[m];
      }
      if (DIR == 2) {
        const int j = b, k = c;
        const long long a = gidx(g, i, j, k);
        double uu = aux[n + a], vv = aux[2 * n + a], ww = aux[3 * n + a], mu = aux[6 * n + a];
        double dxl = mu / (g.x[i + 1] - g.x[i - 1]);
        double dyl = mu / (g.y[j + 1] - g.y[j - 1]);
        double dzl = mu / (g.z[k + 1] - g.z[k - 1]);
        double sigx = dxl * (div3_at(g, div3, i + 1, j, k) - div3_at(g, div3, i - 1, j, k));
        double sigy = dyl * (div3_at(g, div3, i, j + 1, k) - div3_at(g, div3, i, j - 1, k));
        double sigz = dzl * (div3_at(g, div3, i, j, k + 1) - div3_at(g, div3, i, j, k - 1));
        double sigq = sigx * uu + sigy * vv + sigz * ww;
        f[1] = f[1] - sigx;
        f[2] = f[2] - sigy;
        f[3] = f[3] - sigz;
        f[4] = f[4] - sigq;
        if (g.channel_case) {
          const double dt = sc->dt;
          const double rhodt = rhork * dt, gamdt = gamrk * dt;
          double fln1 = (istep > 1 ? -(rhodt * fl_prev[ic]) : 0.0) - gamdt * f[0];
          double fln2 = (istep > 1 ? -(rhodt * fl_prev[nI + ic]) : 0.0) - gamdt * f[1];
          double dy = g.yn[j + 1] - g.yn[j];
          double rho = w[a], rhou = w[n + a], tt = aux[5 * n + a];
          part[0] += fln1 * dy;
          part[1] += fln2 * dy;
          part[2] += rho * dy;
          part[3] += rhou * dy;
          part[4] += rhou * dy * tt;
        }
      }
#pragma unroll
      for (int m = 0; m < 5; ++m) fl[m * nI + ic] = f[m];
      (void)sI;
    }
  }
  if (DIR == 2 && g.channel_case) {
    block_reduce_sum<5, MT_NT>(part, rsh);
    if (threadIdx.x == 0)
#pragma unroll
      for (int r = 0; r < 5; ++r) red[(long long)blockIdx.x * 5 + r] = part[r];
  }
}

// Cells of the flux passes without a face update (outside eul_[jk]min..max) keep fl unchanged;
// with the channel's staggered walls every cell is inside.

// visflx_reduced_ord2_subroutine (kernels_cpu.F90:4623-4721, update_sensor = 0) followed by
// visflx_x/y/z_subroutine (:4779-4999), in the reference's accumulation order; at stage 3 also
// sensor_subroutine (:4726-4744) into the next sensor buffer.
__global__ void __launch_bounds__(256) k_visc(Geom g, const double* __restrict__ aux, double* __restrict__ fl,
                                              double* __restrict__ div3, double* __restrict__ sensor_next,
                                              double* __restrict__ wallprop, int do_sensor) {
  const long long q = (long long)blockIdx.x * 256 + threadIdx.x;
  if (q >= g.nint) return;
  const int i = (int)(q % g.nx) + 1, j = (int)((q / g.nx) % g.ny) + 1, k = (int)(q / ((long long)g.nx * g.ny)) + 1;
  const long long n = g.nvol, nI = g.nint;
  const long long c = gidx(g, i, j, k);
  const long long sX = 1, sY = g.sx, sZ = (long long)g.sx * g.sy;
  auto A = [&](long long a, int m) { return __ldg(aux + (m - 1) * n + a); };
  const double uu = A(c, 2), vv = A(c, 3), ww = A(c, 4), tt = A(c, 6), mu = A(c, 7);
  const double cploc = g.cp0, prandtl = g.prandtl;
  double dxl = 1.0 / (g.x[i + 1] - g.x[i - 1]);
  double dyl = 1.0 / (g.y[j + 1] - g.y[j - 1]);
  double dzl = 1.0 / (g.z[k + 1] - g.z[k - 1]);
  double ux = dxl * (A(c + sX, 2) - A(c - sX, 2));
  double vx = dxl * (A(c + sX, 3) - A(c - sX, 3));
  double wx = dxl * (A(c + sX, 4) - A(c - sX, 4));
  double mux = dxl * (A(c + sX, 7) - A(c - sX, 7));
  double uy = dyl * (A(c + sY, 2) - A(c - sY, 2));
  double vy = dyl * (A(c + sY, 3) - A(c - sY, 3));
  double wy = dyl * (A(c + sY, 4) - A(c - sY, 4));
  double ty = dyl * (A(c + sY, 6) - A(c - sY, 6));
  double muy = dyl * (A(c + sY, 7) - A(c - sY, 7));
  double uz = dzl * (A(c + sZ, 2) - A(c - sZ, 2));
  double vz = dzl * (A(c + sZ, 3) - A(c - sZ, 3));
  double wz = dzl * (A(c + sZ, 4) - A(c - sZ, 4));
  double muz = dzl * (A(c + sZ, 7) - A(c - sZ, 7));
  if (j == 1) {
    const long long wp = (long long)(k - 1) * g.nx + (i - 1);
    const long long nw = (long long)g.nx * g.nz;
    wallprop[wp] = mu * uy;
    wallprop[nw + wp] = mu * wy;
    wallprop[2 * nw + wp] = mu * ty * cploc / prandtl;
  }
  double div = ux + vy + wz;
  double div3l = div / 3.0;
  div3[q] = div3l;
  double omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
  double omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
  if (do_sensor) {
    // sensor_subroutine works from the stored |omega| and div/3
    double om = sqrt(omod2);
    double om2 = om * om;
    double dv = 3.0 * div3l;
    double u0l0 = g.u0 / g.l0;
    double t = fmax(-dv / sqrt(om2 + dv * dv + u0l0 * u0l0), 0.0);
    sensor_next[q] = t * t;
  }
  double sig11 = ux - 2.0 * div3l, sig12 = vx, sig13 = wx;
  double sig21 = uy, sig22 = vy - 2.0 * div3l, sig23 = wy;
  double sig31 = uz, sig32 = vz, sig33 = wz - 2.0 * div3l;
  double sigx = mux * sig11 + muy * sig12 + muz * sig13;
  double sigy = mux * sig21 + muy * sig22 + muz * sig23;
  double sigz = mux * sig31 + muy * sig32 + muz * sig33;
  double sigah = (sig11 * ux + sig12 * uy + sig13 * uz + sig21 * vx + sig22 * vy + sig23 * vz + sig31 * wx +
                  sig32 * wy + sig33 * wz) * mu;
  double sigq = sigx * uu + sigy * vv + sigz * ww + sigah;
  double f2 = fl[nI + q], f3 = fl[2 * nI + q], f4 = fl[3 * nI + q], f5 = fl[4 * nI + q];
  f2 = f2 - sigx;
  f3 = f3 - sigy;
  f4 = f4 - sigz;
  f5 = f5 - sigq;
  // conservative face Laplacian: face sigma between points a (lower) and b (upper)
  auto face = [&](long long a, long long b, double d, double (&s)[4]) {
    double u1 = A(a, 2), u2 = A(b, 2), v1 = A(a, 3), v2 = A(b, 3), w1 = A(a, 4), w2 = A(b, 4);
    double t1 = A(a, 6), t2 = A(b, 6), m1 = A(a, 7), m2 = A(b, 7);
    double qq1 = 0.5 * (u1 * u1 + v1 * v1 + w1 * w1);
    double qq2 = 0.5 * (u2 * u2 + v2 * v2 + w2 * w2);
    double muf = m1 + m2;
    muf = 0.5 * muf / d;
    s[0] = (u2 - u1) * muf;
    s[1] = (v2 - v1) * muf;
    s[2] = (w2 - w1) * muf;
    s[3] = ((t2 - t1) * cploc / prandtl + (qq2 - qq1)) * muf;
  };
  double lo[4], hi[4];
  // x: fl += dxhl*(fhat(i) - fhat(i-1)), fhat = -sigma
  face(c - sX, c, g.x[i] - g.x[i - 1], lo);
  face(c, c + sX, g.x[i + 1] - g.x[i], hi);
  double dxhl = 2.0 / (g.x[i + 1] - g.x[i - 1]);
  f2 = f2 + dxhl * (-hi[0] - -lo[0]);
  f3 = f3 + dxhl * (-hi[1] - -lo[1]);
  f4 = f4 + dxhl * (-hi[2] - -lo[2]);
  f5 = f5 + dxhl * (-hi[3] - -lo[3]);
  // y: fl = (fl + sigma(j-1/2)*dyhl) - sigma(j+1/2)*dyhl
  face(c - sY, c, g.y[j] - g.y[j - 1], lo);
  face(c, c + sY, g.y[j + 1] - g.y[j], hi);
  double dyhl = 2.0 / (g.y[j + 1] - g.y[j - 1]);
  f2 = f2 + lo[0] * dyhl - hi[0] * dyhl;
  f3 = f3 + lo[1] * dyhl - hi[1] * dyhl;
  f4 = f4 + lo[2] * dyhl - hi[2] * dyhl;
  f5 = f5 + lo[3] * dyhl - hi[3] * dyhl;
  face(c - sZ, c, g.z[k] - g.z[k - 1], lo);
  face(c, c + sZ, g.z[k + 1] - g.z[k], hi);
  double dzhl = 2.0 / (g.z[k + 1] - g.z[k - 1]);
  f2 = f2 + lo[0] * dzhl - hi[0] * dzhl;
  f3 = f3 + lo[1] * dzhl - hi[1] * dzhl;
  f4 = f4 + lo[2] * dzhl - hi[2] * dzhl;
  f5 = f5 + lo[3] * dzhl - hi[3] * dzhl;
  fl[nI + q] = f2;
  fl[2 * nI + q] = f3;
  fl[3 * nI + q] = f4;
  fl[4 * nI + q] = f5;
}

// Initial Ducros sensor of run() (visflx(mode=2), singleideal_cpu.F90:1550-1555):
// visflx_reduced_ord2 with update_sensor = 1 (kernels_cpu.F90:4680-4682)
__global__ void __launch_bounds__(256) k_init_sensor(Geom g, const double* __restrict__ aux,
                                                     double* __restrict__ sensor) {
  const long long q = (long long)blockIdx.x * 256 + threadIdx.x;
  if (q >= g.nint) return;
  const int i = (int)(q % g.nx) + 1, j = (int)((q / g.nx) % g.ny) + 1, k = (int)(q / ((long long)g.nx * g.ny)) + 1;
  const long long n = g.nvol, c = gidx(g, i, j, k), sY = g.sx, sZ = (long long)g.sx * g.sy;
  auto A = [&](long long a, int m) { return aux[(m - 1) * n + a]; };
  double dxl = 1.0 / (g.x[i + 1] - g.x[i - 1]);
  double dyl = 1.0 / (g.y[j + 1] - g.y[j - 1]);
  double dzl = 1.0 / (g.z[k + 1] - g.z[k - 1]);
  double ux = dxl * (A(c + 1, 2) - A(c - 1, 2));
  double vx = dxl * (A(c + 1, 3) - A(c - 1, 3));
  double wx = dxl * (A(c + 1, 4) - A(c - 1, 4));
  double uy = dyl * (A(c + sY, 2) - A(c - sY, 2));
  double vy = dyl * (A(c + sY, 3) - A(c - sY, 3));
  double wy = dyl * (A(c + sY, 4) - A(c - sY, 4));
  double uz = dzl * (A(c + sZ, 2) - A(c - sZ, 2));
  double vz = dzl * (A(c + sZ, 3) - A(c - sZ, 3));
  double wz = dzl * (A(c + sZ, 4) - A(c - sZ, 4));
  double div = ux + vy + wz;
  double omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
  double omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
  double u0l0 = g.u0 / g.l0;
  double t = fmax(-div / sqrt(omod2 + div * div + u0l0 * u0l0), 0.0);
  sensor[q] = t * t;
}

// compute_dt_subroutine (kernels_cpu.F90:6814-6880): block maxima of the 9 inverse time scales
__global__ void __launch_bounds__(256) k_dt(Geom g, const double* __restrict__ w, const double* __restrict__ aux,
                                            double* __restrict__ red) {
  __shared__ double sm[9 * 8];
  const long long q = (long long)blockIdx.x * 256 + threadIdx.x;
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (q < g.nint) {
    const int i = (int)(q % g.nx) + 1, j = (int)((q / g.nx) % g.ny) + 1, k = (int)(q / ((long long)g.nx * g.ny)) + 1;
    const long long n = g.nvol, c = gidx(g, i, j, k);
    double rho = w[c];
    double ri = 1.0 / rho;
    double uu = aux[n + c], vv = aux[2 * n + c], ww = aux[3 * n + c], tt = aux[5 * n + c], mu = aux[6 * n + c];
    double nu = ri * mu;
    double kr = nu / g.prandtl;
    double cs = sqrt(g.gamloc * g.rgas0 * tt);
    v[0] = (fabs(uu) + cs) * g.dcsidx[i];
    v[1] = (fabs(vv) + cs) * g.detady[j];
    v[2] = (fabs(ww) + cs) * g.dzitdz[k];
    v[3] = nu * g.dcsidxs[i];
    v[4] = nu * g.detadys[j];
    v[5] = nu * g.dzitdzs[k];
    v[6] = kr * g.dcsidxs[i];
    v[7] = kr * g.detadys[j];
    v[8] = kr * g.dzitdzs[k];
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
    red[(long long)blockIdx.x * 9 + threadIdx.x] = m;
  }
}

__global__ void __launch_bounds__(FIN_NT) k_dt_finish(const double* __restrict__ red, long long nblk, double cfl,
                                                      Scalars* __restrict__ sc) {
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
__global__ void __launch_bounds__(FIN_NT) k_finish_rhs(Geom g, const double* __restrict__ red, long long nblk,
                                                       int first_stage, Scalars* __restrict__ sc) {
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

// update_flux + force_rhs_2 + update_field (kernels_cpu.F90:3400-3442, 3092-3116) and the
// partials of force_var_1 (:3241-3282) and of compute_residual / minmax (:6682-6810).
__global__ void __launch_bounds__(256) k_update(Geom g, double* __restrict__ w, const double* __restrict__ aux,
                                                const double* __restrict__ fl_prev, const double* __restrict__ fl_new,
                                                const Scalars* __restrict__ sc, double rhork, double gamrk, int istep,
                                                int stats, double* __restrict__ red,
                                                const double* __restrict__ sensor_next, double* __restrict__ sensor) {
  __shared__ double sm[2 * 8];
  __shared__ double smn[3 * 8];
  __shared__ double smx[3 * 8];
  const long long q = (long long)blockIdx.x * 256 + threadIdx.x;
  double s2[2] = {0.0, 0.0};
  double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
  double mx[3] = {-100.0, -100.0, -100.0};
  if (q < g.nint) {
    const int i = (int)(q % g.nx) + 1, j = (int)((q / g.nx) % g.ny) + 1, k = (int)(q / ((long long)g.nx * g.ny)) + 1;
    const long long n = g.nvol, nI = g.nint, c = gidx(g, i, j, k);
    const double dt = sc->dt;
    const double rhodt = rhork * dt, gamdt = gamrk * dt;
    double fln[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      double a = istep > 1 ? -(rhodt * fl_prev[m * nI + q]) : 0.0;
      fln[m] = a - gamdt * fl_new[m * nI + q];
    }
    if (g.channel_case) {
      const double b1 = sc->bulk[0], b2 = sc->bulk[1];
      double uu = aux[n + c];
      fln[0] = fln[0] - b1;
      fln[1] = fln[1] - b2;
      fln[4] = fln[4] - uu * b2;
    }
    double wn[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      wn[m] = w[m * n + c] + fln[m];
      w[m * n + c] = wn[m];
    }
    // the stage-3 sensor becomes current once every flux of the stage has used the old one
    if (istep == 3) sensor[q] = sensor_next[q];
    double tstat = aux[5 * n + c];
    if (g.force_var) {
      double dy = g.yn[j + 1] - g.yn[j];
      double ri = 1.0 / wn[0];
      double uu = wn[1] * ri, vv = wn[2] * ri, ww = wn[3] * ri;
      double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
      double ee = wn[4] / wn[0] - qq;
      double tt = t_from_e(g, ee);
      s2[0] = wn[1] * tt * dy;
      tstat = tt;
    }
    if (stats) {
      double r = fln[1] / dt;
      s2[1] = r * r;
      double rho = aux[c];
      double pp = rho * tstat * g.rgas0;
      mn[0] = rho; mn[1] = tstat; mn[2] = pp;
      mx[0] = rho; mx[1] = tstat; mx[2] = pp;
    }
  }
  block_reduce_sum<2, 256>(s2, sm);
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
    for (int r = 0; r < 3; ++r) { smn[r * 8 + warp] = mn[r]; smx[r * 8 + warp] = mx[r]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double* o = red + (long long)blockIdx.x * NRED_UPD;
    o[0] = s2[0];
    o[1] = s2[1];
    for (int r = 0; r < 3; ++r) {
      double a = DBL_MAX, b = -100.0;
      for (int wq = 0; wq < 8; ++wq) { a = fmin(a, smn[r * 8 + wq]); b = fmax(b, smx[r * 8 + wq]); }
      o[2 + r] = a;
      o[5 + r] = b;
    }
  }
}

// force_var (singleideal_cpu.F90:890-933): energy shift for the next pass; residual and extrema
__global__ void __launch_bounds__(FIN_NT) k_finish_upd(Geom g, const double* __restrict__ red, long long nblk,
                                                       int stats, int add_time, Scalars* __restrict__ sc) {
  __shared__ double sm[2 * (FIN_NT / 32)];
  __shared__ double smn[3 * (FIN_NT / 32)], smx[3 * (FIN_NT / 32)];
  double v[2] = {0.0, 0.0};
  double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {-100.0, -100.0, -100.0};
  for (long long b = threadIdx.x; b < nblk; b += FIN_NT) {
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

__global__ void k_add_time(Scalars* sc) { sc->time = sc->time + sc->dt; }

// count_weno_subroutine (kernels_cpu.F90:52-113): number of faces whose stencil sees the sensor
__global__ void __launch_bounds__(256) k_count_weno(Geom g, const double* __restrict__ sensor, double* red) {
  __shared__ double sm[3 * 8];
  const long long q = (long long)blockIdx.x * 256 + threadIdx.x;
  double v[3] = {0.0, 0.0, 0.0};
  if (q < g.nint) {
    const int i = (int)(q % g.nx) + 1, j = (int)((q / g.nx) % g.ny) + 1, k = (int)(q / ((long long)g.nx * g.ny)) + 1;
    const int ws = g.weno_scheme;
    if (i >= g.eul_imin && i <= g.eul_imax) {
      bool s = false;
      for (int o = -ws + 1; o <= ws; ++o) s = s || sensor_at(g, sensor, i + o, j, k) > g.sensor_threshold;
      v[0] = s ? 1.0 : 0.0;
    }
    if (j >= g.eul_jmin && j <= g.eul_jmax) {
      bool s = false;
      for (int o = -ws + 1; o <= ws; ++o) s = s || sensor_at(g, sensor, i, j + o, k) > g.sensor_threshold;
      v[1] = s ? 1.0 : 0.0;
    }
    if (k >= g.eul_kmin && k <= g.eul_kmax) {
      bool s = false;
      for (int o = -ws + 1; o <= ws; ++o) s = s || sensor_at(g, sensor, i, j, k + o) > g.sensor_threshold;
      v[2] = s ? 1.0 : 0.0;
    }
  }
  block_reduce_sum<3, 256>(v, sm);
  if (threadIdx.x == 0)
    for (int r = 0; r < 3; ++r) red[(long long)blockIdx.x * 3 + r] = v[r];
}

inline unsigned nblocks(long long n, int nt) { return (unsigned)((n + nt - 1) / nt); }

// Wrap one launch with profiler events when profiling is on.
#define SB_LAUNCH(dst, kid, s, ...)                  \
  do {                                               \
    if ((dst).prof && (dst).prof->on) (dst).prof->begin((kid), (s)); \
    __VA_ARGS__;                                     \
    if ((dst).prof && (dst).prof->on) (dst).prof->end((s));          \
  } while (0)

}  // namespace

const char* kernel_name(int kid) {
  static const char* names[K_NUM] = {"k_aux", "k_euler_x", "k_visc", "k_euler_y", "k_euler_z", "k_finish_rhs",
                                     "k_update", "k_finish_upd", "k_dt", "k_dt_finish", "k_init_sensor",
                                     "k_apply_shift", "k_fill_ghosts", "k_count_weno", "k_add_time"};
  return (kid >= 0 && kid < K_NUM) ? names[kid] : "?";
}

void Prof::begin(int kid, cudaStream_t s) {
  Rec r{kid, nullptr, nullptr};
  cudaEventCreate(&r.a);
  cudaEventCreate(&r.b);
  cudaEventRecord(r.a, s);
  pending.push_back(r);
}

void Prof::end(cudaStream_t s) { cudaEventRecord(pending.back().b, s); }

cudaError_t Prof::resolve() {
  cudaError_t err = cudaSuccess;
  for (auto& r : pending) {
    cudaError_t e = cudaEventSynchronize(r.b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, r.a, r.b);
    if (e == cudaSuccess) {
      total_ms[r.kid] += ms;
      count[r.kid] += 1;
    } else {
      err = e;
    }
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  pending.clear();
  return err;
}

void Prof::reset() {
  resolve();
  for (int k = 0; k < K_NUM; ++k) { total_ms[k] = 0; count[k] = 0; }
}

// Segments of a march pass: enough threads to fill the device, segments of at least 16 cells
// (one redundant face per segment).
static void march_split(const Geom& g, int dir, int* seglen, int* nseg, long long* nthreads) {
  const int emin = dir == 1 ? g.eul_jmin : g.eul_kmin, emax = dir == 1 ? g.eul_jmax : g.eul_kmax;
  const int ncell = emax - emin + 1;
  const long long lines = (long long)g.nx * (dir == 1 ? g.nz : g.ny);
  const long long target = 148LL * 1024;
  long long ns = (target + lines - 1) / lines;
  int sl = (int)((ncell + ns - 1) / ns);
  if (sl < 16) sl = 16;
  if (sl > ncell) sl = ncell;
  if (sl < 1) sl = 1;
  *seglen = sl;
  *nseg = ncell > 0 ? (ncell + sl - 1) / sl : 0;
  *nthreads = lines * *nseg;
}

long long reduction_slots(const Geom& g) {
  long long a = (long long)nblocks(g.nint, 256) * (NRED_UPD > 9 ? NRED_UPD : 9);
  int sl, ns;
  long long nt;
  march_split(g, 2, &sl, &ns, &nt);
  long long b = (long long)nblocks(nt, MT_NT) * 5;
  return a > b ? a : b;
}

cudaError_t launch_aux(const Geom& g, DevState& d, int apply_shift, cudaStream_t s, long long* nl) {
  SB_LAUNCH(d, K_AUX, s, k_aux<<<nblocks(g.nvol, AUX_NT), AUX_NT, 0, s>>>(g, d.w, d.aux, d.sc, apply_shift, 0));
  ++*nl;
  return cudaGetLastError();
}

cudaError_t launch_fill_ghosts(const Geom& g, DevState& d, cudaStream_t s, long long* nl) {
  SB_LAUNCH(d, K_FILL_GHOSTS, s, k_aux<<<nblocks(g.nvol, AUX_NT), AUX_NT, 0, s>>>(g, d.w, d.aux, d.sc, 0, 1));
  ++*nl;
  return cudaGetLastError();
}

cudaError_t launch_apply_shift(const Geom& g, DevState& d, cudaStream_t s, long long* nl) {
  SB_LAUNCH(d, K_APPLY_SHIFT, s, k_apply_shift<<<nblocks(g.nint, AUX_NT), AUX_NT, 0, s>>>(g, d.w, d.sc));
  ++*nl;
  return cudaGetLastError();
}

cudaError_t launch_init_sensor(const Geom& g, DevState& d, cudaStream_t s, long long* nl) {
  SB_LAUNCH(d, K_INIT_SENSOR, s, k_init_sensor<<<nblocks(g.nint, 256), 256, 0, s>>>(g, d.aux, d.sensor));
  ++*nl;
  return cudaGetLastError();
}

cudaError_t launch_dt(const Geom& g, DevState& d, double cfl, cudaStream_t s, long long* nl) {
  const unsigned nb = nblocks(g.nint, 256);
  SB_LAUNCH(d, K_DT, s, k_dt<<<nb, 256, 0, s>>>(g, d.w, d.aux, d.red));
  SB_LAUNCH(d, K_DT_FINISH, s, k_dt_finish<<<1, FIN_NT, 0, s>>>(d.red, nb, cfl, d.sc));
  *nl += 2;
  return cudaGetLastError();
}

cudaError_t launch_add_time(DevState& d, cudaStream_t s, long long* nl) {
  SB_LAUNCH(d, K_ADD_TIME, s, k_add_time<<<1, 1, 0, s>>>(d.sc));
  ++*nl;
  return cudaGetLastError();
}

cudaError_t launch_count_weno(const Geom& g, DevState& d, cudaStream_t s, long long* nl) {
  const unsigned nb = nblocks(g.nint, 256);
  SB_LAUNCH(d, K_COUNT_WENO, s, k_count_weno<<<nb, 256, 0, s>>>(g, d.sensor, d.red));
  ++*nl;
  return cudaGetLastError();
}

template <int LB, int WS>
static cudaError_t stage_impl(const Geom& g, DevState& d, const StageArgs& a, double* fl_prev, double* fl_new,
                              cudaStream_t s, long long* nl) {
  const dim3 xb(XF_TX, XF_TY);
  const dim3 xg((g.nx + XF_TX - 2) / (XF_TX - 1), (g.ny + XF_TY - 1) / XF_TY, g.nz);
  int sly, nsy, slz, nsz;
  long long nty, ntz;
  march_split(g, 1, &sly, &nsy, &nty);
  march_split(g, 2, &slz, &nsz, &ntz);
  const unsigned gyb = nblocks(nty, MT_NT), gzb = nblocks(ntz, MT_NT);
  if (a.run_aux) {
    SB_LAUNCH(d, K_AUX, s, k_aux<<<nblocks(g.nvol, AUX_NT), AUX_NT, 0, s>>>(g, d.w, d.aux, d.sc, a.apply_shift, 0));
    ++*nl;
  }
  SB_LAUNCH(d, K_EULER_X, s, k_xflux<LB, WS><<<xg, xb, 0, s>>>(g, d.aux, d.sensor, fl_new));
  SB_LAUNCH(d, K_VISC, s,
            k_visc<<<nblocks(g.nint, 256), 256, 0, s>>>(g, d.aux, fl_new, d.div3, d.sensor_next, d.wallprop,
                                                        a.istep == 3));
  if (gyb > 0)
    SB_LAUNCH(d, K_EULER_Y, s,
              k_march<1, LB, WS><<<gyb, MT_NT, 0, s>>>(g, d.aux, d.sensor, fl_new, d.div3, d.w, fl_prev, d.sc,
                                                       a.rhork, a.gamrk, a.istep, sly, nsy, d.red));
  SB_LAUNCH(d, K_EULER_Z, s,
            k_march<2, LB, WS><<<gzb, MT_NT, 0, s>>>(g, d.aux, d.sensor, fl_new, d.div3, d.w, fl_prev, d.sc,
                                                     a.rhork, a.gamrk, a.istep, slz, nsz, d.red));
  *nl += 4;
  if (g.channel_case) {
    SB_LAUNCH(d, K_FINISH_RHS, s, k_finish_rhs<<<1, FIN_NT, 0, s>>>(g, d.red, (long long)gzb, a.istep == 1, d.sc));
    ++*nl;
  }
  const unsigned nbu = nblocks(g.nint, 256);
  SB_LAUNCH(d, K_UPDATE, s,
            k_update<<<nbu, 256, 0, s>>>(g, d.w, d.aux, fl_prev, fl_new, d.sc, a.rhork, a.gamrk, a.istep,
                                         a.want_stats, d.red, d.sensor_next, d.sensor));
  SB_LAUNCH(d, K_FINISH_UPD, s, k_finish_upd<<<1, FIN_NT, 0, s>>>(g, d.red, nbu, a.want_stats, a.add_time, d.sc));
  *nl += 2;
  return cudaGetLastError();
}

cudaError_t launch_stage(const Geom& g, DevState& d, const StageArgs& a, double* fl_prev, double* fl_new,
                         cudaStream_t s, long long* nl) {
  if (g.lmax_base == 3 && g.weno_scheme == 3) return stage_impl<3, 3>(g, d, a, fl_prev, fl_new, s, nl);
  if (g.lmax_base == 2 && g.weno_scheme == 2) return stage_impl<2, 2>(g, d, a, fl_prev, fl_new, s, nl);
  if (g.lmax_base == 4 && g.weno_scheme == 4) return stage_impl<4, 4>(g, d, a, fl_prev, fl_new, s, nl);
  if (g.lmax_base == 3 && g.weno_scheme == 2) return stage_impl<3, 2>(g, d, a, fl_prev, fl_new, s, nl);
  return cudaErrorInvalidValue;
}

bool stage_supported(int lmax_base, int weno_scheme) {
  return (lmax_base == 3 && weno_scheme == 3) || (lmax_base == 2 && weno_scheme == 2) ||
         (lmax_base == 4 && weno_scheme == 4) || (lmax_base == 3 && weno_scheme == 2);
}

}  // namespace sb200
