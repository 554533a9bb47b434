// Running statistics of the B200 backend.
//
//   k_stats    compute_stats (code/src/singleideal/singleideal.F90:2003-2179): one thread per (i,j)
//              column sums the 70 point quantities over k in order, divides by nzmax and folds the
//              sample into the running time average w_stat = (w_stat*itav + w_stat_z)/(itav+1)
//   k_stats3d  compute_stats_3d (:2513-2543): 14 point quantities averaged in time per cell
// Both arrays use the reference's in-memory layout, statistic index fastest: w_stat(70, nx, ny),
// w_stat_z(70, nx, ny), w_stat_3d(14, nx, ny, nz).
//
// The statistics are sampled where manage_output samples them, right after a step, from the state
// the reference holds at that point:
//   * interior w: the current state;
//   * T and mu: w_aux(6), w_aux(7) of the compute_aux pass at the start of stage 3 (the aux buffer
//     keeps them; with force_var, w_aux(6) holds force_var_1's temperature of the updated state,
//     which the update pass of stage 3 stores);
//   * ghost layers of a periodic direction: the copy made by the bcswap at the start of stage 3
//     (update_ghost(do_swap=0) at the end of a stage does not swap), rebuilt here from the source
//     point's current state minus the stage-3 increment fln = -rhork(3) dt fl(stage 2)
//     - gamrk(3) dt fl(stage 3) (minus the channel forcing of force_rhs), except at interior
//     points that the boundary conditions rewrite with fixed values (node-wall momentum, the
//     shock's window at j = ny), where the copy holds those values;
//   * staggered-wall ghosts: the mirror of the current interior after the force_var energy shift
//     (update_ghost runs after force_var);
//   * any other face: its stored ghosts (update_ghost at the end of stage 3).
#include "kernels.hpp"

namespace sb200 {

namespace {

constexpr int ST_NT = 128;

struct StatStep {
  double rhodt, gamdt;  // stage-3 coefficients times dt
  double b1, b2;        // force_rhs corrections of stage 3 (channel)
  double tbdiff;        // force_var energy shift
  int pending;          // the shift is not applied to w yet
};

// (rho, rho u, rho v, rho w) at a stencil point as described above; the point is interior or lies
// outside the block in one direction only.
template <class A>
__device__ __forceinline__ void stat_point(const Geom& g, const double* __restrict__ w, const A* __restrict__ aux,
                                           const double* __restrict__ fl2, const double* __restrict__ fl3,
                                           const StatStep& a, int i, int j, int k, double (&v)[4]) {
  const long long n = g.nvol, nI = g.nint;
  const bool ox = i < 1 || i > g.nx, oy = j < 1 || j > g.ny, oz = k < 1 || k > g.nz;
  if ((ox && g.periodic[0]) || (oy && g.periodic[1]) || (oz && g.periodic[2])) {
    const int si = ox ? wrap(i, g.nx) : i, sj = oy ? wrap(j, g.ny) : j, sk = oz ? wrap(k, g.nz) : k;
    const long long s = gidx(g, si, sj, sk), qi = iidx(g, si, sj, sk);
    // Interior points that update_ghost rewrites with values that do not depend on the solution
    // hold those values in the copy too: the momentum of the node-based wall's points j = 1
    // (bcwall_subroutine, kernels_cpu.F90:6478-6525) and the points j = ny inside the impinging
    // shock's tanh window (bcshock_subroutine, :6159-6196, loop from l = 0)
    const bool node_wall = sj == 1 && g.bctag[2] == 6 && !g.wall_ymin;
    bool shock_window = false;
    if (sj == g.ny && g.bctag[3] == 7) {
      const double xsh = g.xshock_imp - g.y[g.ny] / tan(g.shock_angle);
      shock_window = !(fabs(g.x[si] - xsh) > 8.0 * g.tanhfacs);
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (shock_window || (node_wall && m > 0)) {
        v[m] = w[m * n + s];
        continue;
      }
      double fln = -(a.rhodt * fl2[m * nI + qi]) - a.gamdt * fl3[m * nI + qi];
      if (g.channel_case) {
        if (m == 0) fln = fln - a.b1;
        if (m == 1) fln = fln - a.b2;
      }
      v[m] = w[m * n + s] - fln;
    }
    return;
  }
  if (oy && ((j < 1 && g.wall_ymin) || (j > g.ny && g.wall_ymax))) {
    // bcwall_staggered_subroutine (kernels_cpu.F90:6612-6678) of the shifted interior
    const int sj = j < 1 ? 1 - j : 2 * g.ny + 1 - j;
    const long long s = gidx(g, i, sj, k);
    const double rho = w[s], rhou = w[n + s], rhov = w[2 * n + s], rhow = w[3 * n + s];
    double rhoe = w[4 * n + s];
    const double ts = double(aux[5 * n + s]);  // Newton start (thermally perfect gas)
    if (a.pending) rhoe = shifted_rhoe(g, rho, rhou, rhov, rhow, rhoe, a.tbdiff, ts);
    const double uu = rhou / rho, vv = rhov / rho, ww = rhow / rho;
    const double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
    const double tt = t_from_e(g, rhoe / rho - qq, ts);
    const double pp = rho * tt * g.rgas0;
    const double tg = 2.0 * g.t_wall - tt;
    const double rg = pp / tg / g.rgas0;
    v[0] = rg; v[1] = -rg * uu; v[2] = -rg * vv; v[3] = -rg * ww;
    return;
  }
  const long long s = gidx(g, i, j, k);
  v[0] = w[s]; v[1] = w[n + s]; v[2] = w[2 * n + s]; v[3] = w[3 * n + s];
}

// Velocities u = (rho u)/rho, ... of every interior and face-ghost point of the sampled state
// (stat_point), each formed once: the derivative stencils of compute_stats divide
// w(.,2:4)/w(.,1) at the neighbour points, the same quotients.
template <class A>
__global__ void __launch_bounds__(256) k_stats_vel(Geom g, const double* __restrict__ w, const A* __restrict__ aux,
                                                   const double* __restrict__ fl2, const double* __restrict__ fl3,
                                                   StatStep a, double* __restrict__ vel) {
  const long long n = g.nvol;
  const long long q = (long long)blockIdx.x * 256 + threadIdx.x;
  if (q >= n) return;
  const int i = (int)(q % g.sx) - g.ng + 1, j = (int)((q / g.sx) % g.sy) - g.ng + 1,
            k = (int)(q / ((long long)g.sx * g.sy)) - g.ng + 1;
  const int ox = (i < 1 || i > g.nx), oy = (j < 1 || j > g.ny), oz = (k < 1 || k > g.nz);
  if (ox + oy + oz > 1) return;  // the derivative stencils use no edge or corner points
  double v[4];
  stat_point(g, w, aux, fl2, fl3, a, i, j, k, v);
  vel[q] = v[1] / v[0];
  vel[n + q] = v[2] / v[0];
  vel[2 * n + q] = v[3] / v[0];
}

template <class A>
__global__ void __launch_bounds__(ST_NT) k_stats(Geom g, const double* __restrict__ w, const A* __restrict__ aux,
                                                 const double* __restrict__ vel, int itav,
                                                 double* __restrict__ wstat_z, double* __restrict__ wstat) {
  const long long q = (long long)blockIdx.x * ST_NT + threadIdx.x;
  if (q >= (long long)g.nx * g.ny) return;
  const int i = (int)(q % g.nx) + 1, j = (int)(q / g.nx) + 1;
  const long long n = g.nvol, sY = g.sx, sZ = (long long)g.sx * g.sy;
  const int lmax = g.lmax_base;  // visc_order / 2 (visc_order = ep_order)
  const double rgas0 = g.rgas0;
  const double dxm = g.dcsidx[i], dym = g.detady[j];
  double acc[NV_STAT];
#pragma unroll
  for (int l = 0; l < NV_STAT; ++l) acc[l] = 0.0;
  for (int k = 1; k <= g.nz; ++k) {
    const long long c = gidx(g, i, j, k);
    double ux = 0, vx = 0, wx = 0, uy = 0, vy = 0, wy = 0, uz = 0, vz = 0, wz = 0;
    for (int l = 1; l <= lmax; ++l) {
      const double ccl = g.coeff[lmax - 1][l - 1];
      const long long ox = l, oy = l * sY, oz = l * sZ;
      ux = ux + ccl * (vel[c + ox] - vel[c - ox]);
      vx = vx + ccl * (vel[n + c + ox] - vel[n + c - ox]);
      wx = wx + ccl * (vel[2 * n + c + ox] - vel[2 * n + c - ox]);
      uy = uy + ccl * (vel[c + oy] - vel[c - oy]);
      vy = vy + ccl * (vel[n + c + oy] - vel[n + c - oy]);
      wy = wy + ccl * (vel[2 * n + c + oy] - vel[2 * n + c - oy]);
      uz = uz + ccl * (vel[c + oz] - vel[c - oz]);
      vz = vz + ccl * (vel[n + c + oz] - vel[n + c - oz]);
      wz = wz + ccl * (vel[2 * n + c + oz] - vel[2 * n + c - oz]);
    }
    const double dzm = g.dzitdz[k];
    ux = ux * dxm; vx = vx * dxm; wx = wx * dxm;
    uy = uy * dym; vy = vy * dym; wy = wy * dym;
    uz = uz * dzm; vz = vz * dzm; wz = wz * dzm;
    const double omx = wy - vz, omy = uz - wx, omz = vx - uy;
    const double rho = w[c], rhou = w[n + c], rhov = w[2 * n + c], rhow = w[3 * n + c];
    const double ri = 1.0 / rho;
    const double uu = rhou * ri, vv = rhov * ri, ww = rhow * ri;
    const double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
    const double tt = double(aux[5 * n + c]);
    const double pp = rho * rgas0 * tt;
    const double mu = double(aux[6 * n + c]);
    const double nu = mu / rho;
    // get_gamloc (singleideal.F90:4752-4771)
    const double gamloc = g.calorically_perfect ? g.cp0 / (g.cp0 - rgas0) : gamloc_of_t(g, tt);
    const double cploc = gamloc / (gamloc - 1.0) * rgas0;
    const double cs = sqrt(gamloc * rgas0 * tt);
    const double mach = sqrt(2.0 * qq) / cs;
    const double t_tot = tt + qq * (gamloc - 1.0) / gamloc;
    const double rho2 = rho * rho, uu2 = uu * uu, vv2 = vv * vv, ww2 = ww * ww, pp2 = pp * pp, tt2 = tt * tt;
    const double divl = ux + vy + wz;
    const double div3l = divl / 3.0;
    const double s11 = 2.0 * (ux - div3l) * mu, s12 = (uy + vx) * mu, s13 = (uz + wx) * mu;
    const double s22 = 2.0 * (vy - div3l) * mu, s23 = (vz + wy) * mu, s33 = 2.0 * (wz - div3l) * mu;
    const double s21 = s12, s31 = s13, s32 = s23;
    // the 70 accumulations in the order of the reference (statistics 55-60 add their terms left
    // to right)
    acc[0] += rho;  acc[1] += uu;  acc[2] += vv;  acc[3] += ww;  acc[4] += pp;  acc[5] += tt;
    acc[6] += rho2; acc[7] += uu2; acc[8] += vv2; acc[9] += ww2; acc[10] += pp2; acc[11] += tt2;
    acc[12] += rhou; acc[13] += rhov; acc[14] += rhow;
    acc[15] += rhou * uu; acc[16] += rhov * vv; acc[17] += rhow * ww; acc[18] += rhou * vv;
    acc[19] += mu; acc[20] += nu;
    acc[21] += omx * omx; acc[22] += omy * omy; acc[23] += omz * omz;
    acc[24] += rho * tt; acc[25] += rho * tt2; acc[26] += t_tot; acc[27] += rho * t_tot; acc[28] += t_tot * t_tot;
    acc[29] += rhou * tt; acc[30] += rhov * tt; acc[31] += rhow * tt;
    acc[32] += mach; acc[33] += mach * mach;
    acc[34] += rhou * uu2; acc[35] += rhov * uu2; acc[36] += rhou * vv2; acc[37] += rhov * vv2;
    acc[38] += rhou * ww2; acc[39] += rhov * ww2;
    acc[40] += pp * uu; acc[41] += pp * vv;
    acc[42] += s11; acc[43] += s12; acc[44] += s13; acc[45] += s22; acc[46] += s23; acc[47] += s33;
    acc[48] += s11 * uu; acc[49] += s12 * uu; acc[50] += s21 * vv; acc[51] += s22 * vv;
    acc[52] += s31 * ww; acc[53] += s32 * ww;
    acc[54] = acc[54] + s11 * vv + s21 * uu;
    acc[55] = acc[55] + s12 * vv + s22 * uu;
    acc[56] = acc[56] + s11 * ux + s12 * uy + s13 * uz;
    acc[57] = acc[57] + s21 * vx + s22 * vy + s23 * vz;
    acc[58] = acc[58] + s31 * wx + s32 * wy + s33 * wz;
    acc[59] = acc[59] + s11 * vx + s12 * (ux + vy) + s22 * uy + s13 * vz + s23 * uz;
    acc[60] += pp * ux; acc[61] += pp * vy; acc[62] += pp * wz; acc[63] += pp * (uy + vx);
    acc[64] += divl * divl;
    acc[65] += rho * tt2 * tt; acc[66] += rho * tt2 * tt2; acc[67] += rhou * uu2 * uu;
    acc[68] += cploc; acc[69] += gamloc;
  }
  // single block: the z all-reduce is the identity and nzmax = nz
  const double nzmax = (double)g.nz, rav = (double)itav;
  double* oz = wstat_z + q * NV_STAT;
  double* os = wstat + q * NV_STAT;
#pragma unroll
  for (int l = 0; l < NV_STAT; ++l) {
    const double z = acc[l] / nzmax;
    oz[l] = z;
    os[l] = (os[l] * rav + z) / (rav + 1.0);
  }
}

// The block's 256 cells own a contiguous run of 14 x 256 statistics: it is staged through shared
// memory so that the reads and writes of w_stat_3d are coalesced.
template <class A>
__global__ void __launch_bounds__(256) k_stats3d(Geom g, const double* __restrict__ w, const A* __restrict__ aux,
                                                 int itav, double* __restrict__ ws3) {
  __shared__ double buf[256 * NV_STAT_3D];
  const long long q0 = (long long)blockIdx.x * 256, q = q0 + threadIdx.x;
  const int cnt = (int)(g.nint - q0 < 256 ? g.nint - q0 : 256);
  double* base = ws3 + q0 * NV_STAT_3D;
  for (int e = threadIdx.x; e < cnt * NV_STAT_3D; e += 256) buf[e] = base[e];
  __syncthreads();
  if (q < g.nint) {
    int i, j, k;
    cell_of(g, q, i, j, k);
    const long long n = g.nvol, c = gidx(g, i, j, k);
    const double r = w[c], ru = w[n + c], rv = w[2 * n + c], rw = w[3 * n + c];
    const double t = double(aux[5 * n + c]);
    const double v[NV_STAT_3D] = {r,           ru,          rv,          rw,          r * t,
                                  r * r,       ru * ru / r, rv * rv / r, rw * rw / r, ru * rv / r,
                                  ru * rw / r, rv * rw / r, r * (t * t), (r * t) * (r * t)};
    const double rav = (double)itav;
    double* o = buf + threadIdx.x * NV_STAT_3D;
#pragma unroll
    for (int l = 0; l < NV_STAT_3D; ++l) o[l] = (o[l] * rav + v[l]) / (rav + 1.0);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < cnt * NV_STAT_3D; e += 256) base[e] = buf[e];
}

inline unsigned nblk(long long n, int nt) { return (unsigned)((n + nt - 1) / nt); }

}  // namespace

cudaError_t launch_stats(const Geom& g, DevState& d, const double* fl2, const double* fl3, double rhork3,
                         double gamrk3, int pending, int itav, cudaStream_t s, long long* nl) {
  Scalars sc{};
  cudaError_t e = cudaMemcpyAsync(&sc, d.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  StatStep a{};
  a.rhodt = rhork3 * sc.dt;
  a.gamdt = gamrk3 * sc.dt;
  a.b1 = sc.bulk[0];
  a.b2 = sc.bulk[1];
  a.tbdiff = sc.tbdiff;
  a.pending = pending;
  const unsigned nv = nblk(g.nvol, 256), nb = nblk((long long)g.nx * g.ny, ST_NT);
  if (g.precision == 1) {
    SB_LAUNCH(d, K_STATS, s, k_stats_vel<float><<<nv, 256, 0, s>>>(g, d.w, d.auxf, fl2, fl3, a, d.wstat_vel));
    SB_LAUNCH(d, K_STATS, s, k_stats<float><<<nb, ST_NT, 0, s>>>(g, d.w, d.auxf, d.wstat_vel, itav, d.wstat_z, d.wstat));
  } else {
    SB_LAUNCH(d, K_STATS, s, k_stats_vel<double><<<nv, 256, 0, s>>>(g, d.w, d.aux, fl2, fl3, a, d.wstat_vel));
    SB_LAUNCH(d, K_STATS, s, k_stats<double><<<nb, ST_NT, 0, s>>>(g, d.w, d.aux, d.wstat_vel, itav, d.wstat_z, d.wstat));
  }
  *nl += 2;
  return cudaGetLastError();
}

cudaError_t launch_stats3d(const Geom& g, DevState& d, int itav, cudaStream_t s, long long* nl) {
  const unsigned nb = nblk(g.nint, 256);
  if (g.precision == 1)
    SB_LAUNCH(d, K_STATS3D, s, k_stats3d<float><<<nb, 256, 0, s>>>(g, d.w, d.auxf, itav, d.wstat3d));
  else
    SB_LAUNCH(d, K_STATS3D, s, k_stats3d<double><<<nb, 256, 0, s>>>(g, d.w, d.aux, itav, d.wstat3d));
  ++*nl;
  return cudaGetLastError();
}

// binaryVersion of this file's kernels as the driver loaded them (architecture check)
int binary_version_stats() {
  cudaFuncAttributes a;
  return cudaFuncGetAttributes(&a, k_stats_vel<double>) == cudaSuccess ? a.binaryVersion : -1;
}

}  // namespace sb200
