// C ABI of the B200 backend: context life cycle, field transfer and the time-advance entry
// points declared in include/streams_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "glibc_rand.hpp"
#include "kernels.hpp"
#include "streams_b200.h"

using namespace sb200;

static_assert(MAX_CP == STREAMS_B200_MAX_CP, "cp polynomial sizes of the ABI and the device differ");

struct streams_b200_ctx {
  streams_b200_params p{};
  Geom g{};
  DevState d{};
  double* fl_a = nullptr;  // RK register written by stages 1 and 3
  double* fl_b = nullptr;  // RK register written by stage 2
  double* last_fl = nullptr;  // register written by the last completed stage
  cudaStream_t stream = nullptr;
  int device = 0;
  bool shift_pending = false;  // force_var energy shift not applied to w yet
  bool aux_current = false;    // aux matches w (no update since the last aux pass)
  bool have_stats = false;
  // the state is the one manage_output samples statistics from: a completed rk_sync and no aux
  // pass or upload since
  bool stats_ready = false;
  long long launches = 0;
  Prof prof;
  std::vector<void*> allocs;
  std::string err;
};

namespace {

thread_local std::string g_global_err;

int set_err(streams_b200_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg; else g_global_err = msg;
  return code;
}

int cuda_err(streams_b200_ctx* c, cudaError_t e, const char* what) {
  return set_err(c, STREAMS_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define SB_CHECK(ctx, call)                                   \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_err((ctx), e_, #call); \
  } while (0)

// Device memory comes from the device's stream-ordered pool (cudaMallocAsync on the context's
// stream, cudaFreeAsync at destroy): creating and destroying contexts while others run, as the
// serving loop does, then neither synchronises the device (cudaFree does) nor returns memory to
// the driver between them (the pool keeps what it has: release threshold raised once per device).
void keep_pool_memory(int device) {
  static std::mutex mu;
  static unsigned long long done = 0;
  std::lock_guard<std::mutex> lk(mu);
  if (device < 0 || device >= 64 || (done & (1ULL << device))) return;
  cudaMemPool_t pool = nullptr;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    unsigned long long keep = ~0ULL;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  done |= 1ULL << device;
}

template <class T>
cudaError_t dev_alloc(streams_b200_ctx* c, T** p, size_t count) {
  void* v = nullptr;
  cudaError_t e = cudaMallocAsync(&v, count * sizeof(T) > 0 ? count * sizeof(T) : 16, c->stream);
  // the buffers are filled by copies outside the stream (set-up), so the allocation completes first
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return e;
  c->allocs.push_back(v);
  *p = static_cast<T*>(v);
  return cudaSuccess;
}

// Largest WENO face fraction of a direction at which its hybrid pass reads the WENO faces from
// the face buffer: measured on the 1024x256x192 boundary layer, the split form is ahead below a
// fraction of about 0.55 (FP64: 85.2 vs 87.0 ms per step at 0.51, 89.0 vs 87.3 at 0.61; 61.9 vs
// 78.1 at 0.06) and behind above it (99.8 vs 86.8 at 0.90).
constexpr double WENO_SPLIT_FRAC_DEFAULT = 0.55;
// Boxes below this many cells start with the split off (fraction 0: the hybrid passes alone, no
// list or face kernels launched and no buffers held).  A small box's step is launch-bound and the
// split adds about twenty launches per step, most of them leaving at once; measured on the
// served channel boxes of 0.13 - 1.2 M cells: 501 -> 436 Mcell-steps/s with the split on.
constexpr long long WENO_SPLIT_MIN_CELLS = 1LL << 21;

long long footprint(const streams_b200_params* p) {
  const long long sx = p->nx + 2LL * p->ng, sy = p->ny + 2LL * p->ng, sz = p->nz + 2LL * p->ng;
  const long long nvol = sx * sy * sz, nint = (long long)p->nx * p->ny * p->nz;
  const long long fb = p->precision == 1 ? 4 : 8;  // bytes of the flux-input fields
  long long b = 0;
  b += nvol * 5 * 8;   // w
  b += nvol * (p->precision == 1 ? 7 : 8) * fb;  // aux (+ the sound speed in the FP64 form)
  if (p->precision == 1) b += nvol * 3 * 8;  // FP64 velocities for the stage-3 sensor
  b += nint * fb;      // div3
  b += nint * 2 * 8;   // sensor, sensor_next
  b += nint * 10 * 8;  // two RK registers
  b += (long long)p->nx * p->nz * 3 * 8;
  // WENO faces apart (boxes that start with the split on): the largest direction's face buffer
  // (40 B per face), the three lists and the ghosted sensor flags (1 B per point)
  const long long nfx = (p->nx + 1LL) * p->ny * p->nz, nfy = (long long)p->nx * (p->ny + 1LL) * p->nz,
                  nfz = (long long)p->nx * p->ny * (p->nz + 1LL);
  if (nint >= WENO_SPLIT_MIN_CELLS) b += 40 * std::max(nfx, std::max(nfy, nfz)) + 4 * (nfx + nfy + nfz) + 32 + nvol;
  b += ((nint + 255) / 256) * 9 * 8 + ((p->nx + 31) / 32) * ((p->nz + 7) / 8) * (long long)p->ny * 5 * 8;
  return b + 4096;
}

std::string validate(const streams_b200_params* p) {
  if (p->nx < 1 || p->ny < 1 || p->nz < 1) return "grid sizes must be positive";
  // the x pass's launch grid carries ny / 4 rows in its y and nz planes in its z dimension
  if (p->ny > 4 * 65535 || p->nz > 65535) return "ny must be at most 262140 and nz at most 65535";
  if (p->ep_order < 2 || p->ep_order > 8 || p->ep_order % 2) return "ep_order must be 2, 4, 6 or 8";
  const int lmax = p->ep_order / 2;
  if (p->weno_scheme < 1 || p->weno_scheme > 4) return "weno_scheme must be 1..4";
  if (!stage_supported(lmax, p->weno_scheme))
    return "unsupported (ep_order, weno_scheme) pair for the device path";
  if (p->ng < lmax || p->ng < p->weno_scheme || p->ng < 2) return "ng too small for the stencils";
  if (p->nx < p->ng || p->ny < p->ng || p->nz < p->ng) return "every block dimension must be >= ng";
  if (p->weno_version != 0 && p->weno_version != 1) return "weno_version must be 0 or 1";
  if (p->weno_version == 1 && p->weno_scheme != 3) return "weno_version 1 requires weno_scheme 3";
  if (p->flux_splitting != 0 && p->flux_splitting != 1) return "flux_splitting must be 0 or 1";
  if (p->flux_splitting == 1 && !(p->ep_order == 6 && p->weno_scheme == 3))
    return "flux_splitting = 1 (Rusanov) is implemented for ep_order 6 with weno_scheme 3";
  if (p->conservative_viscous != 0 && p->conservative_viscous != 1) return "conservative_viscous must be 0 or 1";
  if (p->calorically_perfect != 0 && p->calorically_perfect != 1) return "calorically_perfect must be 0 or 1";
  if (p->calorically_perfect == 0) {
    if (p->indx_cp_l > 0 || p->indx_cp_r < 0 || p->indx_cp_r - p->indx_cp_l + 2 > STREAMS_B200_MAX_CP)
      return "cp polynomial: indx_cp_l <= 0 <= indx_cp_r with at most STREAMS_B200_MAX_CP coefficients";
    if (p->precision != 0) return "the thermally perfect gas (calorically_perfect = 0) is an FP64 (precision 0) path";
    if (!(p->ep_order == 6 && p->weno_scheme == 3))
      return "the thermally perfect gas is implemented for ep_order 6 with weno_scheme 3";
  }
  if (p->nrk != 3) return "only the Wray RK3 scheme (nrk = 3) is implemented";
  if (p->precision != 0 && p->precision != 1) return "precision must be 0 (FP64) or 1 (mixed)";
  if (p->visc_model < 0 || p->visc_model > 2) return "visc_model must be 0, 1 or 2";
  for (int d = 0; d < 3; ++d) {
    const int a = p->bctags[2 * d], b = p->bctags[2 * d + 1];
    if ((a == 0) != (b == 0)) return "a periodic direction needs tag 0 on both faces";
  }
  for (int l = 0; l < 6; ++l) {
    const int t = p->bctags[l];
    if (t != 0 && t != 2 && t != 6 && t != 10 && !(t == 7 && l == 3))
      return "boundary tags: periodic (0), extrapolation (2), isothermal wall (6), shock at ymax (7) and "
             "recycling inflow (10)";
    if (t == 6 && l != 2 && l != 3) return "isothermal walls (6) are implemented on the y faces";
    if (t == 6 && !p->is_y_staggered && l != 2) return "a node-based wall (6, not staggered) is implemented at ymin";
    if (t == 10 && l != 0) return "recycling inflow (10) is implemented at xmin";
    const int nr = p->bctags_nr[l];
    if (nr != 0 && nr != 1 && nr != 2 && nr != 3 && nr != 6) return "non-reflecting types: 0, 1, 2, 3, 6";
    if (nr != 0 && l >= 4) return "non-reflecting treatment is implemented on the x and y faces";
    if (nr != 0 && t == 0) return "a periodic face cannot be non-reflecting";
  }
  if (p->bctags[0] == 10 && (p->recyc != 1 || p->i_recyc < p->ng || p->i_recyc > p->nx || p->jbl_inflow < 1 ||
                             p->jbl_inflow > p->ny || p->bctags[4] != 0))
    return "recycling inflow needs recyc = 1, ng <= i_recyc <= nx, 1 <= jbl_inflow <= ny and periodic z";
  if (p->channel_case && !(p->volchan > 0)) return "channel forcing needs volchan > 0";
  if (p->channel_case && p->theta_wall >= -1.0)
    for (int l = 0; l < 6; ++l) {
      // the force_var energy shift is applied to the interior lazily, before the next aux pass;
      // ghosts stored by update_ghost would miss it
      const int t = p->bctags[l];
      if (t == 2 || t == 7 || t == 10 || (t == 6 && !p->is_y_staggered))
        return "bulk-temperature forcing (theta_wall >= -1) needs periodic faces and staggered walls";
    }
  return "";
}


void set_weno_split(Geom& g, double frac) {
  const double nf[3] = {(g.nx + 1.0) * g.ny * g.nz, g.nx * (g.ny + 1.0) * g.nz, g.nx * (double)g.ny * (g.nz + 1.0)};
  // the sample: planes 0, WSAMPLE, 2 WSAMPLE, ... of z (x and y faces) or of the z faces
  const double ns[3] = {(g.nx + 1.0) * g.ny * ((g.nz + WSAMPLE - 1) / WSAMPLE),
                        g.nx * (g.ny + 1.0) * ((g.nz + WSAMPLE - 1) / WSAMPLE),
                        g.nx * (double)g.ny * ((g.nz + WSAMPLE) / WSAMPLE)};
  g.weno_split_frac = frac;
  g.wsplit_on = frac > 0.0 ? 1 : 0;
  for (int d = 0; d < 3; ++d) {
    g.wthr[d] = (unsigned)std::min(std::floor(frac * nf[d]), 4294967294.0);
    g.wthr_s[d] = (unsigned)std::min(std::floor(frac * ns[d]), 4294967294.0);
  }
}

void fill_geom(streams_b200_ctx* c) {
  const streams_b200_params& p = c->p;
  Geom& g = c->g;
  g.nx = p.nx; g.ny = p.ny; g.nz = p.nz; g.ng = p.ng;
  g.sx = p.nx + 2 * p.ng; g.sy = p.ny + 2 * p.ng; g.sz = p.nz + 2 * p.ng;
  g.nvol = (long long)g.sx * g.sy * g.sz;
  g.nint = (long long)p.nx * p.ny * p.nz;
  for (int d = 0; d < 3; ++d) g.periodic[d] = (p.bctags[2 * d] == 0 && p.bctags[2 * d + 1] == 0);
  g.wall_ymin = p.bctags[2] == 6 && p.is_y_staggered;
  g.wall_ymax = p.bctags[3] == 6 && p.is_y_staggered;
  for (int l = 0; l < 6; ++l) {
    g.bctag[l] = p.bctags[l];
    g.nr[l] = p.bctags_nr[l];
  }
  for (int m = 0; m < 5; ++m) g.winf[m] = p.winf[m];
  g.p0 = p.p0;
  g.recyc = p.bctags[0] == 10;
  g.i_recyc = p.i_recyc;
  g.jbl_inflow = p.jbl_inflow;
  g.betarecyc = p.betarecyc;
  g.rand_scale = p.rng_seed == 0 ? 0.0 : 1.0;
  g.xshock_imp = p.xshock_imp; g.shock_angle = p.shock_angle; g.tanhfacs = p.tanhfacs;
  for (int m = 0; m < 5; ++m) g.winf_past_shock[m] = p.winf_past_shock[m];
  for (int l = 0; l < 6; ++l) g.fzf[l] = p.force_zero_flux[l];
  g.eul_imin = p.eul_imin; g.eul_imax = p.eul_imax; g.eul_jmin = p.eul_jmin;
  g.eul_jmax = p.eul_jmax; g.eul_kmin = p.eul_kmin; g.eul_kmax = p.eul_kmax;
  g.lmax_base = p.ep_order / 2;
  g.nkeep = p.nkeep;
  g.weno_scheme = p.weno_scheme;
  g.weno_version = p.weno_version;
  g.sensor_threshold = p.sensor_threshold;
  g.visc_model = p.visc_model;
  g.mu0 = p.mu0; g.t0 = p.t0; g.rgas0 = p.rgas0; g.rho0 = p.rho0; g.u0 = p.u0; g.l0 = p.l0;
  g.sutherland_s = p.sutherland_s; g.t_ref_dim = p.t_ref_dim; g.vtexp = p.powerlaw_vtexp; g.prandtl = p.prandtl;
  g.cp0 = p.cp0; g.cv0 = p.cv0; g.cp_last = p.cp_last; g.cv_last = p.cv_last;
  g.gamloc = p.cp0 / (p.cp0 - p.rgas0);
  g.gm1 = g.gamloc - 1.0;
  g.rgm1 = 1.0 / g.gm1;
  {
    // the same products and quotients the reference forms in wenorec_1d (u0_2, rho0_2u0_2, ...)
    const double u0_2 = p.u0 * p.u0, r2u2 = p.rho0 * p.rho0 * u0_2, r2u4 = r2u2 * u0_2;
    g.wbs_a = 1.0 / r2u2;
    g.wbs_b = 1.0 / r2u4;
    g.wbs_c = g.wbs_b / u0_2;
  }
  g.calorically_perfect = p.calorically_perfect;
  g.cp_l = p.indx_cp_l;
  g.cp_r = p.indx_cp_r;
  g.t_wall = p.t_wall;
  g.channel_case = p.channel_case;
  g.force_var = p.channel_case && p.theta_wall >= -1.0;
  g.volchan = p.volchan;
  g.t_bulk_target = p.t_bulk_target;
  g.precision = p.precision;
  g.conservative_viscous = p.conservative_viscous;
  g.flux_splitting = p.flux_splitting;
  g.march_threads = 148LL * 1024;
  g.march_minseg = 16;
  set_weno_split(g, g.nint >= WENO_SPLIT_MIN_CELLS ? WENO_SPLIT_FRAC_DEFAULT : 0.0);
}

// WENO faces apart: the face buffer (planes of the largest direction's face count), the lists
// with their counters and the ghosted sensor flags, allocated when the split is first turned on.
cudaError_t ensure_weno_buffers(streams_b200_ctx* c) {
  Geom& g = c->g;
  if (g.wface) return cudaSuccess;
  const long long nfx = (g.nx + 1LL) * g.ny * g.nz, nfy = (long long)g.nx * (g.ny + 1LL) * g.nz,
                  nfz = (long long)g.nx * g.ny * (g.nz + 1LL);
  const long long nfmax = std::max(nfx, std::max(nfy, nfz));
  double* wf;
  unsigned* wl;
  unsigned char* wb;
  cudaError_t e;
  if ((e = dev_alloc(c, &wf, 5 * nfmax)) || (e = dev_alloc(c, &wl, nfx + nfy + nfz + 8)) ||
      (e = dev_alloc(c, &wb, g.nvol)))
    return e;
  g.wbits = wb;
  g.wface = wf;
  g.nwface = nfmax;  // plane stride: 5 planes of doubles, or 10 planes of floats in the same bytes
  g.wlist[0] = wl;
  g.wlist[1] = wl + nfx;
  g.wlist[2] = wl + nfx + nfy;
  g.wcount = wl + nfx + nfy + nfz;  // [0..2] list lengths, [4..6] sample counts
  return cudaSuccess;
}

}  // namespace

namespace sb200 {
void set_global_error(const std::string& msg) { g_global_err = msg; }
}  // namespace sb200

extern "C" {

int streams_b200_abi_version(void) { return STREAMS_B200_ABI_VERSION; }
const char* streams_b200_global_error(void) { return g_global_err.c_str(); }
const char* streams_b200_last_error(const streams_b200_ctx* ctx) { return ctx ? ctx->err.c_str() : g_global_err.c_str(); }
long long streams_b200_footprint_bytes(const streams_b200_params* p) { return p ? footprint(p) : -1; }
long long streams_b200_launch_count(const streams_b200_ctx* ctx) { return ctx ? ctx->launches : -1; }

int streams_b200_destroy(streams_b200_ctx* ctx) {
  if (!ctx) return STREAMS_B200_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->prof.resolve();
  for (void* a : ctx->allocs) cudaFreeAsync(a, ctx->stream);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
  return STREAMS_B200_OK;
}

int streams_b200_create(const streams_b200_params* p, const streams_b200_grid* gr, streams_b200_ctx** out) {
  if (!p || !gr || !out) return set_err(nullptr, STREAMS_B200_EINVAL, "null argument");
  *out = nullptr;
  std::string why = validate(p);
  if (!why.empty()) return set_err(nullptr, STREAMS_B200_EINVAL, why);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return set_err(nullptr, STREAMS_B200_ENODEV, "no CUDA device available");
  }
  auto* c = new streams_b200_ctx();
  c->p = *p;
  cudaGetDevice(&c->device);
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, c->device);
  if (prop.major < 10) {
    delete c;
    return set_err(nullptr, STREAMS_B200_ENODEV, "the backend is built for sm_100a (B200); device is sm_" +
                                                     std::to_string(prop.major) + std::to_string(prop.minor));
  }
  fill_geom(c);
  Geom& g = c->g;
  auto fail = [&](cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    streams_b200_destroy(c);
    return set_err(nullptr, e == cudaErrorMemoryAllocation ? STREAMS_B200_ENOMEM : STREAMS_B200_ECUDA, m);
  };
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(e, "cudaStreamCreate");
  keep_pool_memory(c->device);
  // 1-D grid data
  const int ng = p->ng;
  double *dx, *dy, *dz, *dyn, *m1, *m2, *m3, *m4, *m5, *m6;
  int *ex, *ey, *ez;
  if ((e = dev_alloc(c, &dx, p->nx + 2 * ng)) || (e = dev_alloc(c, &dy, p->ny + 2 * ng)) ||
      (e = dev_alloc(c, &dz, p->nz + 2 * ng)) || (e = dev_alloc(c, &dyn, p->ny + 1)) ||
      (e = dev_alloc(c, &m1, p->nx)) || (e = dev_alloc(c, &m2, p->ny)) || (e = dev_alloc(c, &m3, p->nz)) ||
      (e = dev_alloc(c, &m4, p->nx)) || (e = dev_alloc(c, &m5, p->ny)) || (e = dev_alloc(c, &m6, p->nz)) ||
      (e = dev_alloc(c, &ex, p->nx + 1)) || (e = dev_alloc(c, &ey, p->ny + 1)) || (e = dev_alloc(c, &ez, p->nz + 1)))
    return fail(e, "cudaMalloc(grid)");
  const size_t nx = (size_t)p->nx, ny = (size_t)p->ny, nz = (size_t)p->nz, g2 = 2 * (size_t)ng;
  struct Cp { void* d; const void* h; size_t b; } cps[] = {
      {dx, gr->x, (nx + g2) * 8},      {dy, gr->y, (ny + g2) * 8},       {dz, gr->z, (nz + g2) * 8},
      {dyn, gr->yn, (ny + 1) * 8},     {m1, gr->dcsidx, nx * 8},         {m2, gr->detady, ny * 8},
      {m3, gr->dzitdz, nz * 8},        {m4, gr->dcsidxs, nx * 8},        {m5, gr->detadys, ny * 8},
      {m6, gr->dzitdzs, nz * 8},       {ex, gr->ep_ord_x, (nx + 1) * 4}, {ey, gr->ep_ord_y, (ny + 1) * 4},
      {ez, gr->ep_ord_z, (nz + 1) * 4}};
  for (auto& cp : cps) {
    if (!cp.h) {
      streams_b200_destroy(c);
      return set_err(nullptr, STREAMS_B200_EINVAL, "null grid array");
    }
    if ((e = cudaMemcpy(cp.d, cp.h, cp.b, cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e, "cudaMemcpy(grid)");
  }
  g.x = dx + (ng - 1); g.y = dy + (ng - 1); g.z = dz + (ng - 1);
  {
    // the viscous pass's grid divisions, one per line instead of one per cell (host IEEE
    // division: the quotients the device would form)
    const double* crd[3] = {gr->x, gr->y, gr->z};
    const int nn[3] = {p->nx, p->ny, p->nz};
    for (int d = 0; d < 3; ++d) {
      std::vector<double> r(nn[d]), h(nn[d]);
      std::vector<float> rf(nn[d]);
      for (int i = 1; i <= nn[d]; ++i) {
        const double dd = crd[d][i + ng] - crd[d][i + ng - 2];  // x(i+1) - x(i-1)
        r[i - 1] = 1.0 / dd;
        h[i - 1] = 2.0 / dd;
        rf[i - 1] = 1.0f / static_cast<float>(dd);
      }
      double *dr, *dh;
      float* drf;
      if ((e = dev_alloc(c, &dr, nn[d])) || (e = dev_alloc(c, &dh, nn[d])) || (e = dev_alloc(c, &drf, nn[d])))
        return fail(e, "cudaMalloc(grid)");
      if ((e = cudaMemcpy(dr, r.data(), nn[d] * 8, cudaMemcpyHostToDevice)) ||
          (e = cudaMemcpy(dh, h.data(), nn[d] * 8, cudaMemcpyHostToDevice)) ||
          (e = cudaMemcpy(drf, rf.data(), nn[d] * 4, cudaMemcpyHostToDevice)))
        return fail(e, "cudaMemcpy(grid)");
      g.vrl[d] = dr - 1;
      g.vhl[d] = dh - 1;
      g.vrlf[d] = drf - 1;
    }
  }
  g.yn = dyn - 1;
  g.dcsidx = m1 - 1; g.detady = m2 - 1; g.dzitdz = m3 - 1;
  g.dcsidxs = m4 - 1; g.detadys = m5 - 1; g.dzitdzs = m6 - 1;
  g.epx = ex; g.epy = ey; g.epz = ez;
  for (int lm = 0; lm < 4; ++lm)
    for (int l = 0; l < 4; ++l) g.coeff[lm][l] = gr->coeff_deriv1 ? gr->coeff_deriv1[lm * 4 + l] : 0.0;
  {
    // cp(T) / cv(T) polynomial coefficients of the gas (used by the thermally perfect gas)
    double* poly;
    if ((e = dev_alloc(c, &poly, 2 * MAX_CP))) return fail(e, "cudaMalloc(gas)");
    double h[2 * MAX_CP];
    for (int q = 0; q < MAX_CP; ++q) {
      h[q] = p->cp_coeff[q];
      h[MAX_CP + q] = p->cv_coeff[q];
    }
    if ((e = cudaMemcpy(poly, h, sizeof(h), cudaMemcpyHostToDevice))) return fail(e, "cudaMemcpy(gas)");
    g.cpc = poly;
    g.cvc = poly + MAX_CP;
  }
  if (p->conservative_viscous == 0) {
    if (!gr->dcsidx2 || !gr->detady2 || !gr->dzitdz2 || !gr->coeff_deriv2) {
      streams_b200_destroy(c);
      return set_err(nullptr, STREAMS_B200_EINVAL,
                     "conservative_viscous = 0 needs dcsidx2, detady2, dzitdz2 and coeff_deriv2 in the grid");
    }
    double *s1, *s2, *s3;
    if ((e = dev_alloc(c, &s1, p->nx)) || (e = dev_alloc(c, &s2, p->ny)) || (e = dev_alloc(c, &s3, p->nz)))
      return fail(e, "cudaMalloc(grid)");
    if ((e = cudaMemcpy(s1, gr->dcsidx2, nx * 8, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(s2, gr->detady2, ny * 8, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(s3, gr->dzitdz2, nz * 8, cudaMemcpyHostToDevice)))
      return fail(e, "cudaMemcpy(grid)");
    g.dcsidx2 = s1 - 1; g.detady2 = s2 - 1; g.dzitdz2 = s3 - 1;
    for (int lm = 0; lm < 4; ++lm)
      for (int l = 0; l < 5; ++l) g.coeff2[lm][l] = gr->coeff_deriv2[lm * 5 + l];
  }
  if (p->bctags[0] == 10) {
    if (!gr->wmean_inflow || !gr->yplus_inflow || !gr->eta_inflow || !gr->yplus_recyc || !gr->eta_recyc ||
        !gr->weta_inflow || !gr->map_j_inn || !gr->map_j_out) {
      streams_b200_destroy(c);
      return set_err(nullptr, STREAMS_B200_EINVAL, "recycling inflow needs the recyc_prepare arrays in the grid");
    }
    const size_t nyg = ny + g2;
    double *wm, *yi, *ei, *yr, *er, *we;
    int *mi, *mo;
    if ((e = dev_alloc(c, &wm, (size_t)p->ng * ny * 4)) || (e = dev_alloc(c, &yi, nyg)) ||
        (e = dev_alloc(c, &ei, nyg)) || (e = dev_alloc(c, &yr, nyg)) || (e = dev_alloc(c, &er, nyg)) ||
        (e = dev_alloc(c, &we, ny)) || (e = dev_alloc(c, &mi, ny)) || (e = dev_alloc(c, &mo, ny)))
      return fail(e, "cudaMalloc(inflow)");
    struct Cp2 { void* d; const void* h; size_t b; } ins[] = {
        {wm, gr->wmean_inflow, (size_t)p->ng * ny * 4 * 8}, {yi, gr->yplus_inflow, nyg * 8},
        {ei, gr->eta_inflow, nyg * 8}, {yr, gr->yplus_recyc, nyg * 8}, {er, gr->eta_recyc, nyg * 8},
        {we, gr->weta_inflow, ny * 8}, {mi, gr->map_j_inn, ny * 4}, {mo, gr->map_j_out, ny * 4}};
    for (auto& cp : ins)
      if ((e = cudaMemcpy(cp.d, cp.h, cp.b, cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e, "cudaMemcpy(inflow)");
    g.wmean_inflow = wm;
    g.yplus_inflow = yi + (ng - 1); g.eta_inflow = ei + (ng - 1);
    g.yplus_recyc = yr + (ng - 1); g.eta_recyc = er + (ng - 1);
    g.weta_inflow = we - 1; g.map_j_inn = mi - 1; g.map_j_out = mo - 1;
  }
  // WENO faces apart: at most 2^32 faces in a direction (32-bit list entries); buffers when on
  {
    const long long nfmax = std::max((p->nx + 1LL) * p->ny * p->nz,
                                     std::max((long long)p->nx * (p->ny + 1LL) * p->nz,
                                              (long long)p->nx * p->ny * (p->nz + 1LL)));
    if (nfmax >= (1LL << 32)) {
      streams_b200_destroy(c);
      return set_err(nullptr, STREAMS_B200_EINVAL, "more than 2^32 faces in one direction");
    }
    if (g.wsplit_on && (e = ensure_weno_buffers(c))) return fail(e, "cudaMalloc(weno faces)");
  }
  // state
  DevState& d = c->d;
  const bool mixed = p->precision == 1;
  if (mixed) {
    if ((e = dev_alloc(c, &d.auxf, g.nvol * 7)) || (e = dev_alloc(c, &d.div3f, g.nint)) ||
        (e = dev_alloc(c, &d.vel64, g.nvol * 3)))
      return fail(e, "cudaMalloc(state)");
  } else {
    if ((e = dev_alloc(c, &d.aux, g.nvol * 8)) || (e = dev_alloc(c, &d.div3, g.nint)))
      return fail(e, "cudaMalloc(state)");
  }
  if ((e = dev_alloc(c, &d.sensor, g.nint)) || (e = dev_alloc(c, &d.sensor_next, g.nint)))
    return fail(e, "cudaMalloc(state)");
  if ((e = dev_alloc(c, &d.w, g.nvol * 5)) || (e = dev_alloc(c, &c->fl_a, g.nint * 5)) ||
      (e = dev_alloc(c, &c->fl_b, g.nint * 5)) || (e = dev_alloc(c, &d.wallprop, (size_t)p->nx * p->nz * 3)) ||
      (e = dev_alloc(c, &d.sc, 1)))
    return fail(e, "cudaMalloc(state)");
  if (g.recyc) {
    const size_t npl = (size_t)p->ny * p->nz * 3;
    if ((e = dev_alloc(c, &d.rplane, npl)) || (e = dev_alloc(c, &d.recyc_av, (size_t)p->ng * p->ny * 5)) ||
        (e = dev_alloc(c, &d.rng, 1)) || (e = dev_alloc(c, &d.rwords, npl)))
      return fail(e, "cudaMalloc(inflow state)");
    std::vector<double> half(npl, 0.5);  // recyc_prepare's neutral plane
    streams_b200::GlibcRand r(p->rng_seed);
    r.discard(p->rng_draws);
    RngState hs;
    for (int q = 0; q < 34; ++q) hs.ring[q] = r.ring()[q];
    hs.pos = r.position();
    std::vector<unsigned int> jump;
    rand_jump_table((long long)(p->jbl_inflow - 1) * p->nz * 3, jump);
    if ((e = dev_alloc(c, &d.rcoef, jump.size() + 1))) return fail(e, "cudaMalloc(inflow state)");
    if ((e = cudaMemcpy(d.rplane, half.data(), npl * 8, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(d.rng, &hs, sizeof(RngState), cudaMemcpyHostToDevice)) ||
        (!jump.empty() && (e = cudaMemcpy(d.rcoef, jump.data(), jump.size() * 4, cudaMemcpyHostToDevice))))
      return fail(e, "cudaMemcpy(inflow state)");
  }
  d.red_capacity = reduction_slots(g);
  if ((e = dev_alloc(c, &d.red, d.red_capacity))) return fail(e, "cudaMalloc(reductions)");
  d.fl_a = c->fl_a;
  d.fl_b = c->fl_b;
  d.prof = &c->prof;
  const size_t fb = mixed ? 4 : 8;
  void* auxp = mixed ? (void*)d.auxf : (void*)d.aux;
  void* dv = mixed ? (void*)d.div3f : (void*)d.div3;
  if ((e = cudaMemsetAsync(d.w, 0, g.nvol * 5 * 8, c->stream)) || (e = cudaMemsetAsync(auxp, 0, g.nvol * (mixed ? 7 : 8) * fb, c->stream)) ||
      (e = cudaMemsetAsync(d.sensor, 0, g.nint * 8, c->stream)) ||
      (e = cudaMemsetAsync(d.sensor_next, 0, g.nint * 8, c->stream)) ||
      (e = cudaMemsetAsync(dv, 0, g.nint * fb, c->stream)) || (e = cudaMemsetAsync(c->fl_a, 0, g.nint * 40, c->stream)) ||
      (e = cudaMemsetAsync(c->fl_b, 0, g.nint * 40, c->stream)) || (e = cudaMemsetAsync(d.sc, 0, sizeof(Scalars), c->stream)) ||
      (e = cudaStreamSynchronize(c->stream)))
    return fail(e, "initialise state");
  *out = c;
  return STREAMS_B200_OK;
}

int streams_b200_copy_from_field(streams_b200_ctx* c, const double* w) {
  if (!c || !w) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  cudaSetDevice(c->device);
  SB_CHECK(c, cudaMemcpyAsync(c->d.w, w, c->g.nvol * 5 * 8, cudaMemcpyHostToDevice, c->stream));
  c->shift_pending = false;
  c->aux_current = false;
  c->stats_ready = false;
  return STREAMS_B200_OK;
}

int streams_b200_copy_from_device(streams_b200_ctx* c, const double* w) {
  if (!c || !w) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  cudaSetDevice(c->device);
  SB_CHECK(c, cudaMemcpyAsync(c->d.w, w, c->g.nvol * 5 * 8, cudaMemcpyDeviceToDevice, c->stream));
  c->shift_pending = false;
  c->aux_current = false;
  c->stats_ready = false;
  return STREAMS_B200_OK;
}

static int finalize_w(streams_b200_ctx* c) {
  // apply a pending force_var shift and rebuild the ghost layers of w (update_ghost + bcswap);
  // aux is left alone, so that the statistics of the step can still be sampled after a download
  if (c->shift_pending) {
    SB_CHECK(c, launch_apply_shift(c->g, c->d, c->stream, &c->launches));
    c->shift_pending = false;
  }
  SB_CHECK(c, launch_fill_ghosts(c->g, c->d, c->stream, &c->launches));
  return STREAMS_B200_OK;
}

int streams_b200_copy_to_field(streams_b200_ctx* c, double* w) {
  if (!c || !w) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  cudaSetDevice(c->device);
  int rc = finalize_w(c);
  if (rc) return rc;
  SB_CHECK(c, cudaMemcpyAsync(w, c->d.w, c->g.nvol * 5 * 8, cudaMemcpyDeviceToHost, c->stream));
  SB_CHECK(c, cudaStreamSynchronize(c->stream));
  return STREAMS_B200_OK;
}

int streams_b200_copy_to_device(streams_b200_ctx* c, double* w) {
  if (!c || !w) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  cudaSetDevice(c->device);
  int rc = finalize_w(c);
  if (rc) return rc;
  SB_CHECK(c, cudaMemcpyAsync(w, c->d.w, c->g.nvol * 5 * 8, cudaMemcpyDeviceToDevice, c->stream));
  return STREAMS_B200_OK;
}

int streams_b200_init_run(streams_b200_ctx* c) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  cudaSetDevice(c->device);
  // run() starts with update_ghost (singleideal_cpu.F90:1546)
  if (has_stored_ghosts(c->g)) SB_CHECK(c, launch_bc_fill(c->g, c->d, c->stream, &c->launches));
  SB_CHECK(c, launch_aux(c->g, c->d, c->shift_pending ? 1 : 0, c->stream, &c->launches));
  c->shift_pending = false;
  c->aux_current = true;
  c->stats_ready = false;
  SB_CHECK(c, launch_init_sensor(c->g, c->d, c->stream, &c->launches));
  SB_CHECK(c, cudaMemsetAsync(c->fl_a, 0, c->g.nint * 40, c->stream));
  SB_CHECK(c, cudaMemsetAsync(c->fl_b, 0, c->g.nint * 40, c->stream));
  return STREAMS_B200_OK;
}

static int do_compute_dt(streams_b200_ctx* c) {
  if (c->p.cfl < 0) {
    double dt = -c->p.cfl;
    SB_CHECK(c, cudaMemcpyAsync(&c->d.sc->dt, &dt, 8, cudaMemcpyHostToDevice, c->stream));
    SB_CHECK(c, cudaStreamSynchronize(c->stream));
    return STREAMS_B200_OK;
  }
  if (!c->aux_current || c->shift_pending) {
    SB_CHECK(c, launch_aux(c->g, c->d, c->shift_pending ? 1 : 0, c->stream, &c->launches));
    c->shift_pending = false;
    c->aux_current = true;
    c->stats_ready = false;
  }
  SB_CHECK(c, launch_dt(c->g, c->d, c->p.cfl, c->stream, &c->launches));
  return STREAMS_B200_OK;
}

int streams_b200_compute_dt(streams_b200_ctx* c, double* dt) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  cudaSetDevice(c->device);
  int rc = do_compute_dt(c);
  if (rc) return rc;
  if (dt) {
    SB_CHECK(c, cudaMemcpyAsync(dt, &c->d.sc->dt, 8, cudaMemcpyDeviceToHost, c->stream));
    SB_CHECK(c, cudaStreamSynchronize(c->stream));
  }
  return STREAMS_B200_OK;
}

int streams_b200_set_dt(streams_b200_ctx* c, double dt) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  cudaSetDevice(c->device);
  SB_CHECK(c, cudaMemcpyAsync(&c->d.sc->dt, &dt, 8, cudaMemcpyHostToDevice, c->stream));
  SB_CHECK(c, cudaStreamSynchronize(c->stream));
  return STREAMS_B200_OK;
}

int streams_b200_set_time(streams_b200_ctx* c, double t) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  cudaSetDevice(c->device);
  SB_CHECK(c, cudaMemcpyAsync(&c->d.sc->time, &t, 8, cudaMemcpyHostToDevice, c->stream));
  SB_CHECK(c, cudaStreamSynchronize(c->stream));
  return STREAMS_B200_OK;
}

static int do_rk_sync(streams_b200_ctx* c, bool add_time) {
  const bool fv = c->g.force_var != 0;
  for (int istep = 1; istep <= 3; ++istep) {
    StageArgs a{};
    a.istep = istep;
    a.rhork = c->p.rhork[istep - 1];
    a.gamrk = c->p.gamrk[istep - 1];
    a.apply_shift = c->shift_pending ? 1 : 0;
    a.run_aux = (c->aux_current && !c->shift_pending) ? 0 : 1;
    a.want_stats = istep == 3;
    a.add_time = add_time && istep == 3;
    // fixed register roles: stage 1 writes A, stage 2 reads A writes B, stage 3 reads B writes A
    double* prev = istep == 2 ? c->fl_a : c->fl_b;
    double* next = istep == 2 ? c->fl_b : c->fl_a;
    SB_CHECK(c, launch_stage(c->g, c->d, a, prev, next, c->stream, &c->launches));
    c->last_fl = next;
    c->shift_pending = fv;
    c->aux_current = false;
  }
  c->have_stats = true;
  c->stats_ready = true;
  return STREAMS_B200_OK;
}

int streams_b200_rk_sync(streams_b200_ctx* c) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  cudaSetDevice(c->device);
  return do_rk_sync(c, false);
}

int streams_b200_advance(streams_b200_ctx* c, int nsteps, int iter_dt_recompute, int icyc_start, int icyc0) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  if (nsteps < 0 || iter_dt_recompute < 1) return set_err(c, STREAMS_B200_EINVAL, "bad step counts");
  cudaSetDevice(c->device);
  int icyc = icyc_start;
  for (int n = 0; n < nsteps; ++n) {
    icyc = icyc + 1;
    if (c->p.cfl > 0 && (icyc - icyc0) % iter_dt_recompute == 0) {
      int rc = do_compute_dt(c);
      if (rc) return rc;
    }
    int rc = do_rk_sync(c, true);
    if (rc) return rc;
  }
  return STREAMS_B200_OK;
}

int streams_b200_get_scalars(streams_b200_ctx* c, double out[7]) {
  if (!c || !out) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  cudaSetDevice(c->device);
  Scalars s{};
  SB_CHECK(c, cudaMemcpyAsync(&s, c->d.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, c->stream));
  SB_CHECK(c, cudaStreamSynchronize(c->stream));
  out[0] = s.dt; out[1] = s.time; out[2] = s.dpdx; out[3] = s.rhobulk; out[4] = s.ubulk; out[5] = s.tbulk;
  out[6] = s.tbdiff;
  return STREAMS_B200_OK;
}

int streams_b200_compute_residual(streams_b200_ctx* c, double out[7]) {
  if (!c || !out) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  if (!c->have_stats) return set_err(c, STREAMS_B200_EINVAL, "compute_residual needs a completed rk_sync");
  cudaSetDevice(c->device);
  Scalars s{};
  SB_CHECK(c, cudaMemcpyAsync(&s, c->d.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, c->stream));
  SB_CHECK(c, cudaStreamSynchronize(c->stream));
  const double restemp = (double)c->p.nx * (double)c->p.ny * (double)c->p.nz;
  out[0] = std::sqrt(s.residual_sum / restemp);
  out[1] = s.rhomin; out[2] = s.rhomax; out[3] = s.tmin; out[4] = s.tmax; out[5] = s.pmin; out[6] = s.pmax;
  if (std::isnan(out[0])) return set_err(c, STREAMS_B200_ENAN, "NaN residual");
  return STREAMS_B200_OK;
}

int streams_b200_count_weno(streams_b200_ctx* c, double out[3]) {
  if (!c || !out) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  cudaSetDevice(c->device);
  SB_CHECK(c, launch_count_weno(c->g, c->d, c->stream, &c->launches));
  const long long nb = (c->g.nint + 255) / 256;
  std::vector<double> h((size_t)nb * 3);
  SB_CHECK(c, cudaMemcpyAsync(h.data(), c->d.red, h.size() * 8, cudaMemcpyDeviceToHost, c->stream));
  SB_CHECK(c, cudaStreamSynchronize(c->stream));
  double s[3] = {0, 0, 0};
  for (long long b = 0; b < nb; ++b)
    for (int r = 0; r < 3; ++r) s[r] += h[b * 3 + r];
  const streams_b200_params& p = c->p;
  out[0] = s[0] / ((double)(p.eul_imax - p.eul_imin + 1) * p.ny * p.nz);
  out[1] = s[1] / ((double)p.nx * (p.eul_jmax - p.eul_jmin + 1) * p.nz);
  out[2] = s[2] / ((double)p.nx * p.ny * (p.eul_kmax - p.eul_kmin + 1));
  return STREAMS_B200_OK;
}

int streams_b200_get_wallprop(streams_b200_ctx* c, double* out) {
  if (!c || !out) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  cudaSetDevice(c->device);
  SB_CHECK(c, cudaMemcpyAsync(out, c->d.wallprop, (size_t)c->p.nx * c->p.nz * 3 * 8, cudaMemcpyDeviceToHost, c->stream));
  SB_CHECK(c, cudaStreamSynchronize(c->stream));
  return STREAMS_B200_OK;
}

int streams_b200_get_stream(streams_b200_ctx* c, void** stream) {
  if (!c || !stream) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  *stream = (void*)c->stream;
  return STREAMS_B200_OK;
}

int streams_b200_profile_enable(streams_b200_ctx* c, int on) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  cudaSetDevice(c->device);
  if (on < 0) {
    c->prof.reset();
    c->prof.on = false;
  } else {
    c->prof.on = on != 0;
  }
  return STREAMS_B200_OK;
}

int streams_b200_profile_read(streams_b200_ctx* c, int kid, double* total_ms, long long* count) {
  if (!c || kid < 0 || kid >= K_NUM) return set_err(c, STREAMS_B200_EINVAL, "bad kernel id");
  cudaSetDevice(c->device);
  SB_CHECK(c, c->prof.resolve());
  if (total_ms) *total_ms = c->prof.total_ms[kid];
  if (count) *count = c->prof.count[kid];
  return STREAMS_B200_OK;
}

int streams_b200_kernel_count(void) { return K_NUM; }
const char* streams_b200_kernel_name(int kid) { return kernel_name(kid); }

int streams_b200_kernel_binary_versions(int* out, int max) {
  if (!out || max < 0) return STREAMS_B200_EINVAL;
  const int v[3] = {binary_version_stage(), binary_version_bc(), binary_version_stats()};
  for (int q = 0; q < 3 && q < max; ++q) out[q] = v[q];
  return 3;
}

int streams_b200_debug_fetch(streams_b200_ctx* c, int which, double* out, long long n) {
  if (!c || !out) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  cudaSetDevice(c->device);
  const bool mixed = c->p.precision == 1;
  const void* src = nullptr;
  long long cnt = 0;
  bool is_float = false;
  switch (which) {
    case 0: src = mixed ? (const void*)c->d.auxf : (const void*)c->d.aux; cnt = 7 * c->g.nvol; is_float = mixed; break;
    case 1: src = c->last_fl ? c->last_fl : c->fl_a; cnt = 5 * c->g.nint; break;
    case 2: src = c->d.sensor; cnt = c->g.nint; break;
    case 3: src = mixed ? (const void*)c->d.div3f : (const void*)c->d.div3; cnt = c->g.nint; is_float = mixed; break;
    default: return set_err(c, STREAMS_B200_EINVAL, "unknown diagnostic array");
  }
  if (n < cnt) return set_err(c, STREAMS_B200_EINVAL, "output buffer too small");
  if (is_float) {
    std::vector<float> tmp((size_t)cnt);
    SB_CHECK(c, cudaMemcpyAsync(tmp.data(), src, cnt * 4, cudaMemcpyDeviceToHost, c->stream));
    SB_CHECK(c, cudaStreamSynchronize(c->stream));
    for (long long q = 0; q < cnt; ++q) out[q] = tmp[(size_t)q];
  } else {
    SB_CHECK(c, cudaMemcpyAsync(out, src, cnt * 8, cudaMemcpyDeviceToHost, c->stream));
    SB_CHECK(c, cudaStreamSynchronize(c->stream));
  }
  return STREAMS_B200_OK;
}

int streams_b200_synchronize(streams_b200_ctx* c) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  cudaSetDevice(c->device);
  SB_CHECK(c, cudaStreamSynchronize(c->stream));
  SB_CHECK(c, cudaGetLastError());
  return STREAMS_B200_OK;
}

int streams_b200_query(streams_b200_ctx* c) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  cudaSetDevice(c->device);
  const cudaError_t e = cudaStreamQuery(c->stream);
  if (e == cudaErrorNotReady) return 1;
  SB_CHECK(c, e);
  return 0;
}

int streams_b200_batch_class(streams_b200_ctx* c, long long* cls) {
  if (!c || !cls) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  const long long k = batch_key(c->g);
  *cls = k < 0 ? -1 : 2 * k + (c->p.cfl > 0 ? 1 : 0);
  return STREAMS_B200_OK;
}

static int ensure_stats(streams_b200_ctx* c, bool three_d) {
  const size_t n2 = (size_t)NV_STAT * c->p.nx * c->p.ny;
  if (!c->d.wstat) {
    SB_CHECK(c, dev_alloc(c, &c->d.wstat, n2));
    SB_CHECK(c, dev_alloc(c, &c->d.wstat_z, n2));
    SB_CHECK(c, dev_alloc(c, &c->d.wstat_vel, (size_t)c->g.nvol * 3));
    SB_CHECK(c, cudaMemsetAsync(c->d.wstat, 0, n2 * 8, c->stream));
    SB_CHECK(c, cudaMemsetAsync(c->d.wstat_z, 0, n2 * 8, c->stream));
  }
  if (three_d && !c->d.wstat3d) {
    const size_t n3 = (size_t)NV_STAT_3D * c->g.nint;
    SB_CHECK(c, dev_alloc(c, &c->d.wstat3d, n3));
    SB_CHECK(c, cudaMemsetAsync(c->d.wstat3d, 0, n3 * 8, c->stream));
  }
  return STREAMS_B200_OK;
}

static int stats_sample_check(streams_b200_ctx* c, int itav) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  if (itav < 0) return set_err(c, STREAMS_B200_EINVAL, "itav must be >= 0");
  if (!c->stats_ready)
    return set_err(c, STREAMS_B200_EINVAL,
                   "statistics are sampled right after a completed rk_sync, before the next step's compute_dt "
                   "and with no upload in between");
  return STREAMS_B200_OK;
}

int streams_b200_compute_stats(streams_b200_ctx* c, int itav) {
  int rc = stats_sample_check(c, itav);
  if (rc) return rc;
  cudaSetDevice(c->device);
  if ((rc = ensure_stats(c, false))) return rc;
  SB_CHECK(c, launch_stats(c->g, c->d, c->fl_b, c->fl_a, c->p.rhork[2], c->p.gamrk[2], c->shift_pending ? 1 : 0,
                           itav, c->stream, &c->launches));
  return STREAMS_B200_OK;
}

int streams_b200_compute_stats_3d(streams_b200_ctx* c, int itav) {
  int rc = stats_sample_check(c, itav);
  if (rc) return rc;
  cudaSetDevice(c->device);
  if ((rc = ensure_stats(c, true))) return rc;
  SB_CHECK(c, launch_stats3d(c->g, c->d, itav, c->stream, &c->launches));
  return STREAMS_B200_OK;
}

static int stats_buffer(streams_b200_ctx* c, int which, double** buf, long long* cnt) {
  const long long n2 = (long long)NV_STAT * c->p.nx * c->p.ny;
  int rc = ensure_stats(c, which == 2);
  if (rc) return rc;
  switch (which) {
    case 0: *buf = c->d.wstat; *cnt = n2; break;
    case 1: *buf = c->d.wstat_z; *cnt = n2; break;
    case 2: *buf = c->d.wstat3d; *cnt = (long long)NV_STAT_3D * c->g.nint; break;
    default: return set_err(c, STREAMS_B200_EINVAL, "statistics array: 0 w_stat, 1 w_stat_z, 2 w_stat_3d");
  }
  return STREAMS_B200_OK;
}

int streams_b200_get_stats(streams_b200_ctx* c, int which, double* out, long long n) {
  if (!c || !out) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  cudaSetDevice(c->device);
  double* buf = nullptr;
  long long cnt = 0;
  int rc = stats_buffer(c, which, &buf, &cnt);
  if (rc) return rc;
  if (n < cnt) return set_err(c, STREAMS_B200_EINVAL, "output buffer too small");
  SB_CHECK(c, cudaMemcpyAsync(out, buf, cnt * 8, cudaMemcpyDeviceToHost, c->stream));
  SB_CHECK(c, cudaStreamSynchronize(c->stream));
  return STREAMS_B200_OK;
}

int streams_b200_set_stats(streams_b200_ctx* c, int which, const double* in, long long n) {
  if (!c || !in) return set_err(c, STREAMS_B200_EINVAL, "null argument");
  if (which == 1) return set_err(c, STREAMS_B200_EINVAL, "w_stat_z is recomputed by every sample");
  cudaSetDevice(c->device);
  double* buf = nullptr;
  long long cnt = 0;
  int rc = stats_buffer(c, which, &buf, &cnt);
  if (rc) return rc;
  if (n != cnt) return set_err(c, STREAMS_B200_EINVAL, "statistics array size mismatch");
  SB_CHECK(c, cudaMemcpyAsync(buf, in, cnt * 8, cudaMemcpyHostToDevice, c->stream));
  SB_CHECK(c, cudaStreamSynchronize(c->stream));
  return STREAMS_B200_OK;
}

int streams_b200_set_tuning(streams_b200_ctx* c, long long march_threads, int march_minseg) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  if (march_minseg < MARCH_MINSEG_MIN || march_minseg > (1 << 20))
    return set_err(c, STREAMS_B200_EINVAL, "march_minseg must be in [4, 2^20]");
  if (march_threads < 1024 || march_threads > (1LL << 26))
    return set_err(c, STREAMS_B200_EINVAL, "march_threads must be in [1024, 2^26]");
  c->g.march_threads = march_threads;
  c->g.march_minseg = march_minseg;
  return STREAMS_B200_OK;
}

int streams_b200_get_tuning(streams_b200_ctx* c, long long* march_threads, int* march_minseg) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  if (march_threads) *march_threads = c->g.march_threads;
  if (march_minseg) *march_minseg = c->g.march_minseg;
  return STREAMS_B200_OK;
}

int streams_b200_set_weno_split(streams_b200_ctx* c, double max_fraction) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  if (!(max_fraction >= 0.0 && max_fraction <= 1.0))
    return set_err(c, STREAMS_B200_EINVAL, "max_fraction must be in [0, 1]");
  if (max_fraction > 0.0) {
    cudaSetDevice(c->device);
    const cudaError_t e = ensure_weno_buffers(c);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_err(c, STREAMS_B200_ENOMEM, std::string("WENO face buffers: ") + cudaGetErrorString(e));
    }
  }
  set_weno_split(c->g, max_fraction);
  return STREAMS_B200_OK;
}

int streams_b200_get_weno_split(streams_b200_ctx* c, double* max_fraction) {
  if (!c) return set_err(c, STREAMS_B200_EINVAL, "null context");
  if (max_fraction) *max_fraction = c->g.weno_split_frac;
  return STREAMS_B200_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Batched form: one CUDA graph per replay of steps_per_graph steps of every box.  Boxes whose
// stages take the same kernels form a group that advances by launches over a box table
// (batch_kernels.cu): one launch per kernel kind and stage for the whole group.  A box that
// belongs to no group (a configuration the table form does not cover, or the only box of its
// kind) keeps its own step sequence as a parallel branch of the graph.

// A branch of the batch: one box alone, or a group of boxes sharing launches (table != -1)
struct BatchBranch {
  std::vector<int> boxes;
  int table = -1;
};

struct streams_b200_batch {
  std::vector<streams_b200_ctx*> ctxs;
  std::vector<long long> launches_per_replay;  // per box (a group's launches count on its first box)
  std::vector<long long> tuned_threads;        // per box tuning the graph was captured with
  std::vector<int> tuned_minseg;
  std::vector<double> tuned_wsplit;
  int groups_per_class = 1;                    // 0: no shared launches; n: a class's boxes in n groups
  std::vector<BatchBranch> branches;
  std::vector<BoxTable> tables;
  bool grouped = false;                        // branches and tables match the boxes' tuning
  int steps_per_graph = 1, dt_every = 1;
  long long step = 0;  // batch steps taken (drives the dt recompute pattern)
  long long replays = 0;
  int device = 0;
  cudaStream_t master = nullptr;
  cudaEvent_t ev_master = nullptr;
  std::vector<cudaEvent_t> ev_box;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::string err;
};

namespace {

int batch_err(streams_b200_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg; else g_global_err = msg;
  return code;
}

#define SB_BCHECK(b, call)                                                                                   \
  do {                                                                                                       \
    cudaError_t e_ = (call);                                                                                 \
    if (e_ != cudaSuccess) return batch_err((b), STREAMS_B200_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// A context is in the steady state when its host flags are those that every completed step
// leaves behind; the captured step sequence is valid from (and returns to) that state.
bool steady(const streams_b200_ctx* c) {
  return c->have_stats && !c->aux_current && c->shift_pending == (c->g.force_var != 0);
}

// One step of one box, as streams_b200_advance issues it, with the batch's dt pattern.
int box_step(streams_b200_ctx* c, long long step, int dt_every) {
  if (c->p.cfl > 0 && step % dt_every == 0) {
    int rc = do_compute_dt(c);
    if (rc) return rc;
  }
  return do_rk_sync(c, true);
}

void drop_graph(streams_b200_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

void drop_groups(streams_b200_batch* b) {
  // eager group steps run on the boxes' streams: the tables may be freed once those are done
  if (!b->tables.empty())
    for (auto* c : b->ctxs) cudaStreamSynchronize(c->stream);
  for (auto& t : b->tables) box_table_free(t, b->master);
  b->tables.clear();
  b->branches.clear();
  b->grouped = false;
}

// Group key of a box: the stage kernels it takes (batch_key) and the host-side step sequence
// (time step computed or fixed, RK coefficients); -1 when it advances alone.
std::string group_key(const streams_b200_ctx* c) {
  const long long k = batch_key(c->g);
  if (k < 0) return std::string();
  std::string out = std::to_string(k) + (c->p.cfl > 0 ? "+" : "-");
  out.append(reinterpret_cast<const char*>(c->p.rhork), sizeof(c->p.rhork));
  out.append(reinterpret_cast<const char*>(c->p.gamrk), sizeof(c->p.gamrk));
  return out;
}

// Branches of the batch and the box tables of its groups, from the boxes' current tuning.
int make_groups(streams_b200_batch* b) {
  drop_groups(b);
  const int n = (int)b->ctxs.size();
  std::vector<std::string> keys(n);
  for (int i = 0; i < n; ++i) keys[i] = b->groups_per_class > 0 ? group_key(b->ctxs[i]) : std::string();
  std::vector<bool> done(n, false);
  std::vector<BatchBranch> cand;
  for (int i = 0; i < n; ++i) {
    if (done[i]) continue;
    std::vector<int> cls{i};
    done[i] = true;
    if (!keys[i].empty())
      for (int k = i + 1; k < n; ++k)
        if (!done[k] && keys[k] == keys[i]) {
          cls.push_back(k);
          done[k] = true;
        }
    // a class's boxes in groups_per_class groups of about equal cell counts (largest box first
    // into the lightest group), so that the groups' launches, on their own graph branches,
    // overlap one another's memory-bound and arithmetic-bound passes
    const int ng = std::max(1, std::min<int>(b->groups_per_class, (int)cls.size() / 2));
    std::vector<BatchBranch> parts(ng);
    std::vector<long long> load(ng, 0);
    std::vector<int> order = cls;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int c) { return b->ctxs[a]->g.nint > b->ctxs[c]->g.nint; });
    for (int q : order) {
      const int t = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      parts[t].boxes.push_back(q);
      load[t] += b->ctxs[q]->g.nint;
    }
    for (auto& pt : parts) {
      std::sort(pt.boxes.begin(), pt.boxes.end());
      cand.push_back(pt);
    }
  }
  for (BatchBranch& br : cand) {
    if (br.boxes.size() > 1) {
      std::vector<BoxRec> recs;
      for (int q : br.boxes) {
        streams_b200_ctx* c = b->ctxs[q];
        recs.push_back(box_rec(c->g, c->d, c->fl_a, c->fl_b, c->p.cfl));
      }
      BoxTable t;
      cudaError_t e = box_table_build(t, recs, b->master);
      if (e != cudaSuccess) {
        drop_groups(b);
        return batch_err(b, STREAMS_B200_ECUDA, std::string("box table: ") + cudaGetErrorString(e));
      }
      br.table = (int)b->tables.size();
      b->tables.push_back(t);
    }
    b->branches.push_back(br);
  }
  for (int i = 0; i < n; ++i) {
    b->tuned_threads[i] = b->ctxs[i]->g.march_threads;
    b->tuned_minseg[i] = b->ctxs[i]->g.march_minseg;
    b->tuned_wsplit[i] = b->ctxs[i]->g.weno_split_frac;
  }
  b->grouped = true;
  return STREAMS_B200_OK;
}

// a box was re-tuned since the groups were formed (or the graph captured)
bool tuning_changed(const streams_b200_batch* b) {
  for (size_t i = 0; i < b->ctxs.size(); ++i)
    if (b->ctxs[i]->g.march_threads != b->tuned_threads[i] || b->ctxs[i]->g.march_minseg != b->tuned_minseg[i] ||
        b->ctxs[i]->g.weno_split_frac != b->tuned_wsplit[i])
      return true;
  return false;
}

// The host flags of a group's boxes agree (they do from the first completed step on).
bool flags_agree(const streams_b200_batch* b, const BatchBranch& br) {
  const streams_b200_ctx* c0 = b->ctxs[br.boxes[0]];
  for (int q : br.boxes) {
    const streams_b200_ctx* c = b->ctxs[q];
    if (c->aux_current != c0->aux_current || c->shift_pending != c0->shift_pending) return false;
  }
  return true;
}

// One step of a group on the stream s, as box_step issues it for each box (do_compute_dt and
// do_rk_sync, with the same host flags), by launches over the group's box table.
int group_step(streams_b200_batch* b, const BatchBranch& br, long long step, cudaStream_t s) {
  const BoxTable& t = b->tables[br.table];
  streams_b200_ctx* c0 = b->ctxs[br.boxes[0]];
  long long nl = 0;
  cudaError_t e = cudaSuccess;
  if (c0->p.cfl > 0 && step % b->dt_every == 0) {
    if (!c0->aux_current || c0->shift_pending) {
      e = batch_launch_aux(t, c0->shift_pending ? 1 : 0, s, &nl);
      for (int q : br.boxes) {
        streams_b200_ctx* c = b->ctxs[q];
        c->shift_pending = false;
        c->aux_current = true;
        c->stats_ready = false;
      }
    }
    if (e == cudaSuccess) e = batch_launch_dt(t, s, &nl);
  }
  const bool fv = c0->g.force_var != 0;
  for (int istep = 1; istep <= 3 && e == cudaSuccess; ++istep) {
    StageArgs a{};
    a.istep = istep;
    a.rhork = c0->p.rhork[istep - 1];
    a.gamrk = c0->p.gamrk[istep - 1];
    a.apply_shift = c0->shift_pending ? 1 : 0;
    a.run_aux = (c0->aux_current && !c0->shift_pending) ? 0 : 1;
    a.want_stats = istep == 3;
    a.add_time = istep == 3;
    e = batch_launch_stage(t, a, s, &nl);
    for (int q : br.boxes) {
      streams_b200_ctx* c = b->ctxs[q];
      c->last_fl = istep == 2 ? c->fl_b : c->fl_a;
      c->shift_pending = fv;
      c->aux_current = false;
    }
  }
  if (e != cudaSuccess)
    return batch_err(b, STREAMS_B200_ECUDA, std::string("group step: ") + cudaGetErrorString(e));
  for (int q : br.boxes) {
    streams_b200_ctx* c = b->ctxs[q];
    c->have_stats = true;
    c->stats_ready = true;
  }
  c0->launches += nl;
  return STREAMS_B200_OK;
}

int capture(streams_b200_batch* b) {
  drop_graph(b);
  if (!b->grouped) {
    int rc = make_groups(b);
    if (rc) return rc;
  }
  SB_BCHECK(b, cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
  int rc = STREAMS_B200_OK;
  std::string why;
  cudaError_t e = cudaEventRecord(b->ev_master, b->master);
  for (size_t r = 0; r < b->branches.size() && e == cudaSuccess && rc == STREAMS_B200_OK; ++r) {
    const BatchBranch& br = b->branches[r];
    const int i = br.boxes[0];
    streams_b200_ctx* c = b->ctxs[i];
    const long long l0 = c->launches;
    e = cudaStreamWaitEvent(c->stream, b->ev_master, 0);
    for (int s = 0; s < b->steps_per_graph && e == cudaSuccess && rc == STREAMS_B200_OK; ++s) {
      if (br.table >= 0) {
        rc = group_step(b, br, s, c->stream);
        if (rc) why = "group of box " + std::to_string(i) + ": " + b->err;
      } else {
        rc = box_step(c, s, b->dt_every);
        if (rc) why = "box " + std::to_string(i) + ": " + c->err;
      }
    }
    if (e == cudaSuccess && rc == STREAMS_B200_OK) e = cudaEventRecord(b->ev_box[i], c->stream);
    if (e == cudaSuccess && rc == STREAMS_B200_OK) e = cudaStreamWaitEvent(b->master, b->ev_box[i], 0);
    for (int q : br.boxes) b->launches_per_replay[q] = 0;
    b->launches_per_replay[i] = c->launches - l0;
    c->launches = l0;
  }
  for (size_t i = 0; i < b->ctxs.size(); ++i) {
    b->tuned_threads[i] = b->ctxs[i]->g.march_threads;
    b->tuned_minseg[i] = b->ctxs[i]->g.march_minseg;
    b->tuned_wsplit[i] = b->ctxs[i]->g.weno_split_frac;
  }
  cudaGraph_t gr = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(b->master, &gr);
  if (e != cudaSuccess || rc != STREAMS_B200_OK || e2 != cudaSuccess) {
    if (gr) cudaGraphDestroy(gr);
    cudaGetLastError();
    if (rc) return batch_err(b, rc, "capture: " + why);
    return batch_err(b, STREAMS_B200_ECUDA,
                     std::string("capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  b->graph = gr;
  SB_BCHECK(b, cudaGraphInstantiate(&b->exec, b->graph, 0));
  return STREAMS_B200_OK;
}

// eager steps: every lone box on its own stream, every group on its first box's stream (the
// other boxes' streams joined before and after)
int eager_steps(streams_b200_batch* b, int n) {
  if (n > 0 && !b->grouped) {
    int rc = make_groups(b);
    if (rc) return rc;
  }
  for (int s = 0; s < n; ++s) {
    for (const BatchBranch& br : b->branches) {
      if (br.table >= 0 && flags_agree(b, br)) {
        streams_b200_ctx* c0 = b->ctxs[br.boxes[0]];
        for (size_t q = 1; q < br.boxes.size(); ++q) {
          streams_b200_ctx* c = b->ctxs[br.boxes[q]];
          SB_BCHECK(b, cudaEventRecord(b->ev_box[br.boxes[q]], c->stream));
          SB_BCHECK(b, cudaStreamWaitEvent(c0->stream, b->ev_box[br.boxes[q]], 0));
        }
        int rc = group_step(b, br, b->step, c0->stream);
        if (rc) return rc;
        SB_BCHECK(b, cudaEventRecord(b->ev_box[br.boxes[0]], c0->stream));
        for (size_t q = 1; q < br.boxes.size(); ++q)
          SB_BCHECK(b, cudaStreamWaitEvent(b->ctxs[br.boxes[q]]->stream, b->ev_box[br.boxes[0]], 0));
        continue;
      }
      for (int i : br.boxes) {
        int rc = box_step(b->ctxs[i], b->step, b->dt_every);
        if (rc) return batch_err(b, rc, "box " + std::to_string(i) + ": " + b->ctxs[i]->err);
      }
    }
    ++b->step;
  }
  return STREAMS_B200_OK;
}

}  // namespace

extern "C" {

int streams_b200_batch_create(streams_b200_ctx** ctxs, int n, int steps_per_graph, int dt_every,
                              streams_b200_batch** out) {
  if (!ctxs || !out || n < 1) return batch_err(nullptr, STREAMS_B200_EINVAL, "batch needs at least one context");
  *out = nullptr;
  if (steps_per_graph < 1 || dt_every < 1 || steps_per_graph % dt_every != 0)
    return batch_err(nullptr, STREAMS_B200_EINVAL, "steps_per_graph must be a positive multiple of dt_every");
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i]) return batch_err(nullptr, STREAMS_B200_EINVAL, "null context in batch");
    if (ctxs[i]->device != ctxs[0]->device)
      return batch_err(nullptr, STREAMS_B200_EINVAL, "all contexts of a batch must be on one device");
    for (int k = 0; k < i; ++k)
      if (ctxs[k] == ctxs[i]) return batch_err(nullptr, STREAMS_B200_EINVAL, "context listed twice in batch");
  }
  auto* b = new streams_b200_batch();
  b->ctxs.assign(ctxs, ctxs + n);
  b->launches_per_replay.assign(n, 0);
  b->tuned_threads.assign(n, 0);
  b->tuned_minseg.assign(n, 0);
  b->tuned_wsplit.assign(n, -1.0);
  b->ev_box.assign(n, nullptr);
  b->steps_per_graph = steps_per_graph;
  b->dt_every = dt_every;
  b->device = ctxs[0]->device;
  cudaSetDevice(b->device);
  cudaError_t e = cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_master, cudaEventDisableTiming);
  for (int i = 0; i < n && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&b->ev_box[i], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    std::string m = std::string("batch set-up: ") + cudaGetErrorString(e);
    streams_b200_batch_destroy(b);
    return batch_err(nullptr, STREAMS_B200_ECUDA, m);
  }
  *out = b;
  return STREAMS_B200_OK;
}

int streams_b200_batch_advance(streams_b200_batch* b, int nsteps) {
  if (!b) return batch_err(b, STREAMS_B200_EINVAL, "null batch");
  if (nsteps < 0) return batch_err(b, STREAMS_B200_EINVAL, "negative step count");
  cudaSetDevice(b->device);
  for (auto* c : b->ctxs)
    if (c->prof.on) return batch_err(b, STREAMS_B200_EINVAL, "a profiled context cannot run in a batch");
  if ((b->exec || b->grouped) && tuning_changed(b)) {
    drop_graph(b);  // a box was re-tuned since the capture
    drop_groups(b);
  }
  bool all_steady = true;
  for (auto* c : b->ctxs) all_steady = all_steady && steady(c);
  if (!all_steady && nsteps > 0) {
    drop_graph(b);
    int rc = eager_steps(b, 1);
    if (rc) return rc;
    --nsteps;
  }
  // graph replays start on a step of the dt pattern's period (steps_per_graph is a multiple)
  int lead = 0;
  if (b->step % b->dt_every != 0) lead = (int)(b->dt_every - b->step % b->dt_every);
  if (lead > nsteps) lead = nsteps;
  int rc = eager_steps(b, lead);
  if (rc) return rc;
  nsteps -= lead;
  const int nrep = nsteps / b->steps_per_graph;
  if (nrep > 0) {
    if (!b->exec) {
      rc = capture(b);
      if (rc) return rc;
    }
    for (size_t i = 0; i < b->ctxs.size(); ++i) {
      SB_BCHECK(b, cudaEventRecord(b->ev_box[i], b->ctxs[i]->stream));
      SB_BCHECK(b, cudaStreamWaitEvent(b->master, b->ev_box[i], 0));
    }
    for (int r = 0; r < nrep; ++r) SB_BCHECK(b, cudaGraphLaunch(b->exec, b->master));
    SB_BCHECK(b, cudaEventRecord(b->ev_master, b->master));
    for (size_t i = 0; i < b->ctxs.size(); ++i) {
      SB_BCHECK(b, cudaStreamWaitEvent(b->ctxs[i]->stream, b->ev_master, 0));
      b->ctxs[i]->launches += b->launches_per_replay[i] * nrep;
    }
    b->replays += nrep;
    b->step += (long long)nrep * b->steps_per_graph;
  }
  return eager_steps(b, nsteps - nrep * b->steps_per_graph);
}

int streams_b200_batch_synchronize(streams_b200_batch* b) {
  if (!b) return batch_err(b, STREAMS_B200_EINVAL, "null batch");
  cudaSetDevice(b->device);
  SB_BCHECK(b, cudaStreamSynchronize(b->master));
  for (auto* c : b->ctxs) SB_BCHECK(b, cudaStreamSynchronize(c->stream));
  return STREAMS_B200_OK;
}

int streams_b200_batch_invalidate(streams_b200_batch* b) {
  if (!b) return batch_err(b, STREAMS_B200_EINVAL, "null batch");
  cudaSetDevice(b->device);
  drop_graph(b);
  drop_groups(b);
  return STREAMS_B200_OK;
}

int streams_b200_batch_set_shared_launches(streams_b200_batch* b, int groups_per_class) {
  if (!b) return batch_err(b, STREAMS_B200_EINVAL, "null batch");
  if (groups_per_class < 0) return batch_err(b, STREAMS_B200_EINVAL, "negative groups_per_class");
  cudaSetDevice(b->device);
  if (b->groups_per_class != groups_per_class) {
    drop_graph(b);
    drop_groups(b);
    b->groups_per_class = groups_per_class;
  }
  return STREAMS_B200_OK;
}

int streams_b200_batch_groups(streams_b200_batch* b, int* ngroups, int* nshared) {
  if (!b) return batch_err(b, STREAMS_B200_EINVAL, "null batch");
  cudaSetDevice(b->device);
  if (!b->grouped) {
    int rc = make_groups(b);
    if (rc) return rc;
  }
  int g = 0, n = 0;
  for (const BatchBranch& br : b->branches)
    if (br.table >= 0) {
      ++g;
      n += (int)br.boxes.size();
    }
  if (ngroups) *ngroups = g;
  if (nshared) *nshared = n;
  return STREAMS_B200_OK;
}

int streams_b200_batch_stats(streams_b200_batch* b, long long* replays, long long* launches_per_replay) {
  if (!b) return batch_err(b, STREAMS_B200_EINVAL, "null batch");
  long long t = 0;
  for (long long v : b->launches_per_replay) t += v;
  if (replays) *replays = b->replays;
  if (launches_per_replay) *launches_per_replay = t;
  return STREAMS_B200_OK;
}

const char* streams_b200_batch_last_error(streams_b200_batch* b) { return b ? b->err.c_str() : ""; }

int streams_b200_batch_destroy(streams_b200_batch* b) {
  if (!b) return STREAMS_B200_OK;
  cudaSetDevice(b->device);
  if (b->master) cudaStreamSynchronize(b->master);
  drop_graph(b);
  for (auto* c : b->ctxs) cudaStreamSynchronize(c->stream);
  drop_groups(b);
  for (auto ev : b->ev_box)
    if (ev) cudaEventDestroy(ev);
  if (b->ev_master) cudaEventDestroy(b->ev_master);
  if (b->master) cudaStreamDestroy(b->master);
  delete b;
  return STREAMS_B200_OK;
}

}  // extern "C"
