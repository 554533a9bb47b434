// Open-boundary kernels of the B200 backend (boundary layer): the ghost fills of update_ghost
// for stored (non-periodic, non-mirrored) faces, the recycling-rescaling inflow with its random
// plane, and the characteristic non-reflecting correction of the right-hand side.
//
// Ghost policy: periodic faces and staggered walls produce their ghost states on the fly where
// they are read (k_aux); every other face keeps its ghosts in w, written here in the order of
// update_ghost (singleideal_cpu.F90:1064-1138): ilat = 1 .. 6.
#include "kernels.hpp"

namespace sb200 {

namespace {

constexpr int BC_NT = 128;

__device__ __forceinline__ double e_of_t(const Geom& g, double tt) { return e_from_t(g, tt); }

// bcextr_subroutine (kernels_cpu.F90:6323-6390): ghosts l = 1..ng copy the boundary node
__global__ void __launch_bounds__(BC_NT) k_bc_extr(Geom g, double* __restrict__ w, int ilat) {
  const int dir = (ilat - 1) / 2;
  const int n1 = dir == 0 ? g.ny : g.nx;           // first index along the face
  const int n2 = dir == 2 ? g.ny : g.nz;           // second index along the face
  const long long q = (long long)blockIdx.x * BC_NT + threadIdx.x;
  if (q >= (long long)n1 * n2) return;
  const int a = (int)(q % n1) + 1, b = (int)(q / n1) + 1;
  const bool lo = (ilat % 2) == 1;
  const long long n = g.nvol;
  for (int l = 1; l <= g.ng; ++l) {
    int i, j, k, is, js, ks;
    if (dir == 0) { j = a; k = b; i = lo ? 1 - l : g.nx + l; is = lo ? 1 : g.nx; js = j; ks = k; }
    else if (dir == 1) { i = a; k = b; j = lo ? 1 - l : g.ny + l; js = lo ? 1 : g.ny; is = i; ks = k; }
    else { i = a; j = b; k = lo ? 1 - l : g.nz + l; ks = lo ? 1 : g.nz; is = i; js = j; }
    const long long dst = gidx(g, i, j, k), src = gidx(g, is, js, ks);
#pragma unroll
    for (int m = 0; m < 5; ++m) w[m * n + dst] = w[m * n + src];
  }
}

// bcwall_subroutine (kernels_cpu.F90:6478-6525), ymin: wall node at rest and at T_wall, ghosts
// mirrored about it (T_g = 2 T_w - T, p_g = p, velocity reversed); the Newton iteration of a
// thermally perfect gas starts from the interior point's temperature in aux, as w_aux(6) there
template <class A>
__global__ void __launch_bounds__(BC_NT) k_bc_wall(Geom g, double* __restrict__ w, const A* __restrict__ aux) {
  const long long q = (long long)blockIdx.x * BC_NT + threadIdx.x;
  if (q >= (long long)g.nx * g.nz) return;
  const int i = (int)(q % g.nx) + 1, k = (int)(q / g.nx) + 1;
  const long long n = g.nvol, c1 = gidx(g, i, 1, k);
  w[n + c1] = 0.0;
  w[2 * n + c1] = 0.0;
  w[3 * n + c1] = 0.0;
  w[4 * n + c1] = w[c1] * e_of_t(g, g.t_wall);
  for (int l = 1; l <= g.ng; ++l) {
    const long long s = gidx(g, i, 1 + l, k), d = gidx(g, i, 1 - l, k);
    double rho = w[s];
    const double uu = w[n + s] / rho, vv = w[2 * n + s] / rho, ww = w[3 * n + s] / rho;
    const double rhoe = w[4 * n + s];
    const double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
    double ee = rhoe / rho - qq;
    double tt = t_from_e(g, ee, double(aux[5 * n + s]));
    const double pp = rho * tt * g.rgas0;
    tt = 2.0 * g.t_wall - tt;
    ee = e_of_t(g, tt);
    rho = pp / tt / g.rgas0;
    w[d] = rho;
    w[n + d] = -rho * uu;
    w[2 * n + d] = -rho * vv;
    w[3 * n + d] = -rho * ww;
    w[4 * n + d] = rho * (ee + qq);
  }
}

// bcshock_subroutine (kernels_cpu.F90:6159-6196), ymax: within 8 tanhfacs of the shock's foot
// the top row and its ghosts take the tanh blend of the free stream and the post-shock state,
// elsewhere the ghosts copy the top row (l = 0 is the row itself)
__global__ void __launch_bounds__(BC_NT) k_bc_shock(Geom g, double* __restrict__ w) {
  const long long q = (long long)blockIdx.x * BC_NT + threadIdx.x;
  if (q >= (long long)g.nx * g.nz) return;
  const int i = (int)(q % g.nx) + 1, k = (int)(q / g.nx) + 1;
  const long long n = g.nvol, top = gidx(g, i, g.ny, k);
  const double tanhlen = 8.0 * g.tanhfacs;
  for (int l = 0; l <= g.ng; ++l) {
    const double xsh = g.xshock_imp - g.y[g.ny + l] / tan(g.shock_angle);
    const double xx = g.x[i] - xsh;
    const long long d = gidx(g, i, g.ny + l, k);
    if (fabs(xx) > tanhlen) {
#pragma unroll
      for (int m = 0; m < 5; ++m) w[m * n + d] = w[m * n + top];
    } else {
      const double tanhf = 0.5 * (1.0 + tanh(xx / g.tanhfacs));
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        const double dwinf = g.winf_past_shock[m] - g.winf[m];
        w[m * n + d] = g.winf[m] + dwinf * tanhf;
      }
    }
  }
}

// z index of the recycling plane that feeds inflow plane k: recyc_exchange shifts by nzmax/2
// (singleideal_cpu.F90:935-999 on one block)
__device__ __forceinline__ int recyc_k(const Geom& g, int k) {
  const int ks = g.nz / 2;
  return ((k - ks - 1) % g.nz + g.nz) % g.nz + 1;
}

// bcrecyc_subroutine_1 (kernels_cpu.F90:5810-5828): spanwise sums of the recycling plane
// i_recyc+1-i, one thread per (i, j, m), summed in k order
__global__ void __launch_bounds__(BC_NT) k_recyc_mean(Geom g, const double* __restrict__ w, double* __restrict__ av) {
  const long long q = (long long)blockIdx.x * BC_NT + threadIdx.x;
  if (q >= (long long)g.ng * g.ny * 5) return;
  const int i = (int)(q % g.ng) + 1;
  const int j = (int)((q / g.ng) % g.ny) + 1;
  const int m = (int)(q / ((long long)g.ng * g.ny));
  const int ir = g.i_recyc + 1 - i;
  double a = 0.0;
  for (int k = 1; k <= g.nz; ++k) a = a + w[m * g.nvol + gidx(g, ir, j, recyc_k(g, k))];
  av[q] = a;  // [(m*ny + j-1)*ng + i-1]
}

// bcrecyc_subroutine_2 and _3 (kernels_cpu.F90:5832-5947): fluctuations of the recycling plane
// about its spanwise (Favre) means, rescaled onto the inflow's inner/outer coordinates, blended,
// damped, with the random plane's perturbation; the inflow ghosts 1-i, i = 1..ng
__global__ void __launch_bounds__(BC_NT) k_recyc_fill(Geom g, double* __restrict__ w, const double* __restrict__ av,
                                                      const double* __restrict__ rplane) {
  const long long q = (long long)blockIdx.x * BC_NT + threadIdx.x;
  if (q >= (long long)g.ny * g.nz) return;
  const int j = (int)(q % g.ny) + 1, k = (int)(q / g.ny) + 1;
  const long long n = g.nvol;
  const int ng = g.ng, ny = g.ny;
  double u0_02 = 0.02 * g.u0 * g.rand_scale;
  const double eta = g.eta_inflow[j];
  const double etamin = fmin(eta, 1.0);
  const double weta = g.weta_inflow[j];
  const double weta1 = 1.0 - weta;
  const double bdamp = 0.5 * (1.0 - tanh(4.0 * (g.eta_inflow[j] - 2.0)));
  const int j_inn = g.map_j_inn[j], j_out = g.map_j_out[j];
  const bool zero = (j == 1 || j_inn >= ny || j_out >= ny);
  double disty_inn = 0.0, disty_out = 0.0;
  if (!zero) {
    disty_inn = (g.yplus_inflow[j] - g.yplus_recyc[j_inn]) / (g.yplus_recyc[j_inn + 1] - g.yplus_recyc[j_inn]);
    disty_out = (g.eta_inflow[j] - g.eta_recyc[j_out]) / (g.eta_recyc[j_out + 1] - g.eta_recyc[j_out]);
  }
  const int kr = recyc_k(g, k);
  for (int i = 1; i <= ng; ++i) {
    auto WMI = [&](int m) { return g.wmean_inflow[((long long)(m - 1) * ny + (j - 1)) * ng + (i - 1)]; };
    const double rhomean = WMI(1);
    const double uumean = WMI(2) / rhomean, vvmean = WMI(3) / rhomean, wwmean = WMI(4) / rhomean;
    double rhofluc = 0.0, ufluc = 0.0, vfluc = 0.0, wfluc = 0.0;
    if (!zero) {
      const int ir = g.i_recyc + 1 - i;
      auto AV = [&](int jj, int m) { return av[((long long)(m - 1) * ny + (jj - 1)) * ng + (i - 1)]; };
      // fluctuation of variable m (1: rho, 2..4: velocity) of the recycling plane at node jj
      auto fl = [&](int jj, int m) {
        const long long a = gidx(g, ir, jj, kr);
        const double rho = w[a];
        if (m == 1) return rho - AV(jj, 1) / (double)g.nz;
        return w[(m - 1) * n + a] / rho - AV(jj, m) / AV(jj, 1);
      };
      auto mix = [&](int m, int jj, double d) { return fl(jj, m) * (1.0 - d) + fl(jj + 1, m) * d; };
      const double rhof_inn = mix(1, j_inn, disty_inn), rhof_out = mix(1, j_out, disty_out);
      const double uf_inn = mix(2, j_inn, disty_inn), uf_out = mix(2, j_out, disty_out);
      const double vf_inn = mix(3, j_inn, disty_inn), vf_out = mix(3, j_out, disty_out);
      const double wf_inn = mix(4, j_inn, disty_inn), wf_out = mix(4, j_out, disty_out);
      rhofluc = rhof_inn * weta1 + rhof_out * weta;
      ufluc = uf_inn * weta1 + uf_out * weta;
      vfluc = vf_inn * weta1 + vf_out * weta;
      wfluc = wf_inn * weta1 + wf_out * weta;
      rhofluc = rhofluc * bdamp;
      ufluc = ufluc * bdamp * g.betarecyc;
      vfluc = vfluc * bdamp * g.betarecyc;
      wfluc = wfluc * bdamp * g.betarecyc;
      const long long pj = (long long)(k - 1) * ny + (j - 1), pn = (long long)ny * g.nz;
      ufluc = ufluc + u0_02 * (rplane[pj] - 0.5) * etamin;
      vfluc = vfluc + u0_02 * (rplane[pn + pj] - 0.5) * etamin;
      wfluc = wfluc + u0_02 * (rplane[2 * pn + pj] - 0.5) * etamin;
    }
    rhofluc = fmax(-0.75 * rhomean, rhofluc);
    rhofluc = fmin(4.0 * rhomean, rhofluc);
    const double rho = rhomean + rhofluc;
    const double tt = g.p0 / rho / g.rgas0;
    const double uu = uumean + ufluc, vv = vvmean + vfluc, ww = wwmean + wfluc;
    const double rhou = rho * uu, rhov = rho * vv, rhow = rho * ww;
    const double ee = e_of_t(g, tt);
    const long long d = gidx(g, 1 - i, j, k);
    w[d] = rho;
    w[n + d] = rhou;
    w[2 * n + d] = rhov;
    w[3 * n + d] = rhow;
    w[4 * n + d] = rho * ee + 0.5 * (rhou * rhou + rhov * rhov + rhow * rhow) / rho;
  }
}

// The random inflow plane of a stage continues the glibc sequence (random(): additive feedback
// x_n = x_(n-31) + x_(n-3) mod 2^32, output x_n >> 1; crandom.c, crandom_f.F90:81-93), but is
// drawn in parallel: the recurrence is linear, so with y_k the 31 words before the stage
// (y_0 .. y_30) every later word is y_m = sum_i c_i y_i, c the coefficients of t^m mod
// (t^31 - t^28 - 1) over the integers mod 2^32.  Thread c starts from the host-made
// coefficients of its chunk's first word and steps them by t (one shift and one addition) for
// each further word of its chunk: every draw is the reference's, bit for bit.  The 32-bit words
// go to `words`; the scatter kernel converts them and advances the ring.
__global__ void __launch_bounds__(128) k_rand_words(const RngState* __restrict__ st, const unsigned int* __restrict__ coef,
                                                    unsigned int* __restrict__ words, long long total) {
  const long long c = (long long)blockIdx.x * 128 + threadIdx.x;
  const long long i0 = c * RAND_CHUNK;
  if (i0 >= total) return;
  const long long pos0 = st->pos;  // >= 344: the generator discards 310 words at seeding
  unsigned int y[31], cv[31];
#pragma unroll
  for (int i = 0; i < 31; ++i) {
    y[i] = st->ring[(pos0 - 31 + i) % 34];
    cv[i] = coef[c * 31 + i];
  }
  const int n = (int)(total - i0 < RAND_CHUNK ? total - i0 : RAND_CHUNK);
  for (int r = 0; r < n; ++r) {
    unsigned int v = 0;
#pragma unroll
    for (int i = 0; i < 31; ++i) v += cv[i] * y[i];
    words[i0 + r] = v;
    // cv <- t cv mod (t^31 - t^28 - 1): the t^31 term becomes t^28 + 1
    const unsigned int top = cv[30];
#pragma unroll
    for (int i = 30; i > 0; --i) cv[i] = cv[i - 1];
    cv[0] = top;
    cv[28] += top;
  }
}

// draw d of the stage: component c = d mod 3, k = (d / 3) mod nz + 1, j = d / (3 nz) + 2
__global__ void __launch_bounds__(256) k_rand_scatter(Geom g, const unsigned int* __restrict__ words,
                                                      double* __restrict__ rplane, long long total) {
  const long long d = (long long)blockIdx.x * 256 + threadIdx.x;
  if (d >= total) return;
  const int c = (int)(d % 3);
  const long long jk = d / 3;
  const int k = (int)(jk % g.nz) + 1, j = (int)(jk / g.nz) + 2;
  const int v = (int)(words[d] >> 1);
  rplane[(long long)c * g.ny * g.nz + (long long)(k - 1) * g.ny + (j - 1)] = g.rand_scale * (double)v / 2147483647.0;
}

// the generator's ring after the stage's draws: the last 34 words at their positions mod 34
__global__ void __launch_bounds__(64) k_rand_advance(RngState* __restrict__ st, const unsigned int* __restrict__ words,
                                                     long long total) {
  const long long pos0 = st->pos;
  __syncthreads();
  if (threadIdx.x < 34) {
    const long long idx = total - 34 + threadIdx.x;
    if (idx >= 0) st->ring[(pos0 + idx) % 34] = words[idx];
  }
  if (threadIdx.x == 0) st->pos = pos0 + total;
}

// bc_nr_lat_x_kernel / bc_nr_lat_y_kernel (kernels_cpu.F90:5169-5283, 5420-5540): characteristic
// correction of fl at the boundary points of face ilat (x or y), one thread per point.
template <class A>
__global__ void __launch_bounds__(BC_NT) k_bc_nr(Geom g, const double* __restrict__ w, const A* __restrict__ aux,
                                                 double* __restrict__ fl, int ilat) {
  const int dir = (ilat - 1) / 2;
  const int n1 = dir == 0 ? g.ny : g.nx;
  const long long q = (long long)blockIdx.x * BC_NT + threadIdx.x;
  if (q >= (long long)n1 * g.nz) return;
  const int t = (int)(q % n1) + 1, k = (int)(q / n1) + 1;
  const int start_or_end = (ilat - 1) % 2 + 1;
  const int sgn = start_or_end == 1 ? 1 : -1;
  const int nr_type = g.nr[ilat - 1];
  const int i = dir == 0 ? (start_or_end == 1 ? 1 : g.nx) : t;
  const int j = dir == 1 ? (start_or_end == 1 ? 1 : g.ny) : t;
  const long long n = g.nvol;
  const long long sd = dir == 0 ? 1 : g.sx;  // address step along the normal
  const long long c0 = gidx(g, i, j, k);
  const double c_one[3] = {-1.5, 2.0, -0.5};
  double dw_dn[5], dw_dn_outer[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    double a = 0.0;
#pragma unroll
    for (int l = 1; l <= 3; ++l) a = a + sgn * c_one[l - 1] * w[m * n + c0 + sgn * (l - 1) * sd];
    dw_dn[m] = a;
    double w_target = 0.0;
    if (nr_type == 2) w_target = w[m * n + c0 - sgn * sd];
    else if (nr_type == 3) w_target = g.winf[m];
    dw_dn_outer[m] = sgn * (w[m * n + c0] - w_target);
  }
  const double rho = double(aux[c0]), uu = double(aux[n + c0]), vv = double(aux[2 * n + c0]);
  const double ww = double(aux[3 * n + c0]), h = double(aux[4 * n + c0]), tt = double(aux[5 * n + c0]);
  const double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  const double gamloc = gamloc_of_t(g, tt), rgas0 = g.rgas0;
  const double cc = gamloc * tt * rgas0;
  const double c = sqrt(cc);
  const double ci = 1.0 / c;
  const double p_rho = tt * rgas0;
  const double p_e = rho * (gamloc - 1.0);
  const double etot = h - tt * rgas0;
  const double b3 = etot - rho * p_rho / p_e;
  const double b2 = p_e / (rho * cc);
  const double b1 = p_rho / cc - b2 * (etot - 2.0 * qq);
  // eigenvectors_x / _y (kernels_cpu.F90:2728-2782, 2842-2896): el[var][char], er[char][var]
  const double vel[3] = {uu, vv, ww};
  const double vn = dir == 0 ? uu : vv;
  const double vt1 = dir == 0 ? vv : uu;
  const int t1 = dir == 0 ? 2 : 1, ns = dir == 0 ? 1 : 2;
  double el[5][5], er[5][5];
#pragma unroll
  for (int a = 0; a < 5; ++a)
#pragma unroll
    for (int b = 0; b < 5; ++b) el[a][b] = er[a][b] = 0.0;
  el[0][0] = 0.5 * (b1 + vn * ci);
  el[0][1] = 1.0 - b1;
  el[0][2] = -vt1;
  el[0][3] = -ww;
  el[0][4] = 0.5 * (b1 - vn * ci);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    el[1 + d][0] = -0.5 * (b2 * vel[d] + (1 + d == ns ? ci : 0.0));
    el[1 + d][1] = b2 * vel[d];
    el[1 + d][4] = -0.5 * (b2 * vel[d] - (1 + d == ns ? ci : 0.0));
    er[0][1 + d] = vel[d] - (1 + d == ns ? c : 0.0);
    er[1][1 + d] = vel[d];
    er[4][1 + d] = vel[d] + (1 + d == ns ? c : 0.0);
  }
  el[4][0] = 0.5 * b2;
  el[4][1] = -b2;
  el[4][4] = 0.5 * b2;
  el[t1][2] = 1.0;
  el[3][3] = 1.0;
  er[0][0] = 1.0; er[1][0] = 1.0; er[4][0] = 1.0;
  er[2][t1] = 1.0;
  er[3][3] = 1.0;
  er[0][4] = h - vn * c;
  er[1][4] = b3;
  er[2][4] = vt1;
  er[3][4] = ww;
  er[4][4] = h + vn * c;
  double dwc[5], dwc_outer[5], ev[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int mm = 0; mm < 5; ++mm) {
      a = a + el[mm][m] * dw_dn[mm];
      b = b + el[mm][m] * dw_dn_outer[mm];
    }
    dwc[m] = a;
    dwc_outer[m] = b;
  }
  ev[0] = vn - c; ev[1] = vn; ev[2] = vn; ev[3] = vn; ev[4] = vn + c;
  if (nr_type == 1)
#pragma unroll
    for (int l = 0; l < 5; ++l) ev[l] = start_or_end == 1 ? fmin(ev[l], 0.0) : fmax(ev[l], 0.0);
  if (nr_type == 2 || nr_type == 3)
#pragma unroll
    for (int m = 0; m < 5; ++m)
      if (sgn * ev[m] > 0.0) dwc[m] = dwc_outer[m];
#pragma unroll
  for (int m = 0; m < 5; ++m) dwc[m] = ev[m] * dwc[m];
  if (nr_type == 6) {
    dwc[1] = dwc[2] = dwc[3] = 0.0;
    if (start_or_end == 1) dwc[4] = dwc[0]; else dwc[0] = dwc[4];
  }
  const double met = dir == 0 ? g.dcsidx[i] : g.detady[j];
  const long long ic = iidx(g, i, j, k);
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    double df = 0.0;
#pragma unroll
    for (int mm = 0; mm < 5; ++mm) df = df + er[mm][m] * dwc[mm];
    fl[m * g.nint + ic] = fl[m * g.nint + ic] + df * met;
  }
}

unsigned nb(long long n) { return (unsigned)((n + BC_NT - 1) / BC_NT); }

}  // namespace

// update_ghost for the stored faces, in ilat order (recycling, extrapolation, node wall)
cudaError_t launch_bc_fill(const Geom& g, DevState& d, cudaStream_t s, long long* nl) {
  for (int ilat = 1; ilat <= 6; ++ilat) {
    const int t = g.bctag[ilat - 1];
    if (t == 10 && ilat == 1) {
      SB_LAUNCH(d, K_BC_FILL, s, k_recyc_mean<<<nb((long long)g.ng * g.ny * 5), BC_NT, 0, s>>>(g, d.w, d.recyc_av));
      SB_LAUNCH(d, K_BC_FILL, s,
                k_recyc_fill<<<nb((long long)g.ny * g.nz), BC_NT, 0, s>>>(g, d.w, d.recyc_av, d.rplane));
      *nl += 2;
    } else if (t == 2) {
      const int dir = (ilat - 1) / 2;
      const long long np = (long long)(dir == 0 ? g.ny : g.nx) * (dir == 2 ? g.ny : g.nz);
      SB_LAUNCH(d, K_BC_FILL, s, k_bc_extr<<<nb(np), BC_NT, 0, s>>>(g, d.w, ilat));
      ++*nl;
    } else if (t == 7 && ilat == 4) {
      SB_LAUNCH(d, K_BC_FILL, s, k_bc_shock<<<nb((long long)g.nx * g.nz), BC_NT, 0, s>>>(g, d.w));
      ++*nl;
    } else if (t == 6 && ilat == 3 && !g.wall_ymin) {
      if (g.precision == 1)
        SB_LAUNCH(d, K_BC_FILL, s, k_bc_wall<float><<<nb((long long)g.nx * g.nz), BC_NT, 0, s>>>(g, d.w, d.auxf));
      else
        SB_LAUNCH(d, K_BC_FILL, s, k_bc_wall<double><<<nb((long long)g.nx * g.nz), BC_NT, 0, s>>>(g, d.w, d.aux));
      ++*nl;
    }
  }
  return cudaGetLastError();
}

bool has_stored_ghosts(const Geom& g) {
  for (int l = 0; l < 6; ++l) {
    const int t = g.bctag[l];
    if (t == 2 || t == 7 || t == 10 || (t == 6 && !(l == 2 ? g.wall_ymin : g.wall_ymax))) return true;
  }
  return false;
}

namespace {
// a b mod (t^31 - t^28 - 1), coefficients mod 2^32 (t^k = t^(k-3) + t^(k-31) for k >= 31)
void polymulmod(const unsigned int* a, const unsigned int* b, unsigned int* out) {
  unsigned int prod[61] = {};
  for (int i = 0; i < 31; ++i)
    for (int j = 0; j < 31; ++j) prod[i + j] += a[i] * b[j];
  for (int k = 60; k >= 31; --k) {
    const unsigned int c = prod[k];
    prod[k] = 0;
    prod[k - 3] += c;
    prod[k - 31] += c;
  }
  for (int i = 0; i < 31; ++i) out[i] = prod[i];
}
}  // namespace

void rand_jump_table(long long total, std::vector<unsigned int>& table) {
  const long long nchunk = (total + RAND_CHUNK - 1) / RAND_CHUNK;
  table.assign((size_t)nchunk * 31, 0u);
  if (nchunk == 0) return;
  // t^RAND_CHUNK by repeated multiplication with t, the first chunk's t^31 = t^28 + 1
  unsigned int step[31] = {}, t1[31] = {}, cur[31] = {};
  step[0] = 1;
  t1[1] = 1;
  for (int q = 0; q < RAND_CHUNK; ++q) {
    unsigned int nx[31];
    polymulmod(step, t1, nx);
    for (int i = 0; i < 31; ++i) step[i] = nx[i];
  }
  cur[0] = 1;
  cur[28] = 1;
  for (long long c = 0; c < nchunk; ++c) {
    for (int i = 0; i < 31; ++i) table[(size_t)c * 31 + i] = cur[i];
    unsigned int nx[31];
    polymulmod(cur, step, nx);
    for (int i = 0; i < 31; ++i) cur[i] = nx[i];
  }
}

cudaError_t launch_rand_plane(const Geom& g, DevState& d, cudaStream_t s, long long* nl) {
  const long long total = (long long)(g.jbl_inflow - 1) * g.nz * 3;
  if (total <= 0) return cudaSuccess;
  const long long nchunk = (total + RAND_CHUNK - 1) / RAND_CHUNK;
  SB_LAUNCH(d, K_RAND_PLANE, s,
            k_rand_words<<<(unsigned)((nchunk + 127) / 128), 128, 0, s>>>(d.rng, d.rcoef, d.rwords, total));
  SB_LAUNCH(d, K_RAND_PLANE, s,
            k_rand_scatter<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(g, d.rwords, d.rplane, total));
  SB_LAUNCH(d, K_RAND_PLANE, s, k_rand_advance<<<1, 64, 0, s>>>(d.rng, d.rwords, total));
  *nl += 3;
  return cudaGetLastError();
}

// bc_nr (singleideal_cpu.F90:1001-1062) on the x and y faces
cudaError_t launch_bc_nr(const Geom& g, DevState& d, double* fl, cudaStream_t s, long long* nl) {
  for (int ilat = 1; ilat <= 4; ++ilat) {
    if (g.nr[ilat - 1] <= 0) continue;
    const long long np = (long long)((ilat <= 2) ? g.ny : g.nx) * g.nz;
    if (g.precision == 1)
      SB_LAUNCH(d, K_BC_NR, s, k_bc_nr<float><<<nb(np), BC_NT, 0, s>>>(g, d.w, d.auxf, fl, ilat));
    else
      SB_LAUNCH(d, K_BC_NR, s, k_bc_nr<double><<<nb(np), BC_NT, 0, s>>>(g, d.w, d.aux, fl, ilat));
    ++*nl;
  }
  return cudaGetLastError();
}

// binaryVersion of this file's kernels as the driver loaded them (architecture check)
int binary_version_bc() {
  cudaFuncAttributes a;
  return cudaFuncGetAttributes(&a, k_bc_extr) == cudaSuccess ? a.binaryVersion : -1;
}

}  // namespace sb200
