// Time-step reduction over caller-owned device arrays that allocates no memory.
//
// Some callers cannot let a library call cudaMalloc: a host code that owns every byte of device
// memory through its own pool (a Fortran solver object that maps its arrays with OpenACC or CUDA
// Fortran and forbids foreign allocations), or one that runs under a fixed memory budget where
// an allocation inside the time loop may fail or fragment the pool.  For them this file offers
// the CFL time-step reduction of compute_dt without a context: the caller passes its own device
// arrays and receives dt in a device word it owns.  The only scratch is the file-scope static
// array below; it is part of the library image, so every GPU that loads the library holds it
// until the process exits, and no call allocates or frees anything.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "common.cuh"
#include "streams_b200.h"

namespace {

constexpr int DTN_NT = 256;               // threads per block: one block per 256 interior cells
constexpr int DTN_MAX_BLOCKS = 16384;     // => at most 4,194,304 interior cells per call
constexpr int DTN_SLOTS = 9;              // inverse time scales reduced per block
constexpr int DTN_MAX_DEVICES = 64;

// Block partial maxima of the last call (16384 x 9 doubles = 1.125 MiB).  Every block writes
// its nine slots before the finishing kernel reads them, so nothing has to start at zero; the
// array keeps the contents of the last call, and calls that overlap on the GPU race on it.
__device__ __align__(256) double g_dt_partials[DTN_MAX_BLOCKS * DTN_SLOTS];

std::mutex g_mutex;
double* g_partials_ptr[DTN_MAX_DEVICES] = {};  // device address of g_dt_partials, per device

struct DtArgs {
  int nx, ny, nz, ng, sx, sy;
  long long nvol;
  const double *w, *aux, *dcsidx, *detady, *dzitdz, *dcsidxs, *detadys, *dzitdzs;
  double rgas0, prandtl, gamloc;
};

// Same arithmetic as compute_dt_subroutine (kernels_cpu.F90:6814-6880); metric arrays are
// indexed from 0 (dcsidx[i-1] is dcsidx(i)).
__global__ void __launch_bounds__(DTN_NT) k_dt_noalloc(DtArgs a, double* __restrict__ part) {
  __shared__ double sm[DTN_SLOTS * (DTN_NT / 32)];
  const long long n = (long long)a.nx * a.ny * a.nz;
  const long long q = (long long)blockIdx.x * DTN_NT + threadIdx.x;
  double v[DTN_SLOTS] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (q < n) {
    const int i = (int)(q % a.nx) + 1, j = (int)((q / a.nx) % a.ny) + 1, k = (int)(q / ((long long)a.nx * a.ny)) + 1;
    const long long c = ((long long)(k + a.ng - 1) * a.sy + (j + a.ng - 1)) * a.sx + (i + a.ng - 1);
    double rho = a.w[c];
    double ri = 1.0 / rho;
    double uu = a.aux[a.nvol + c], vv = a.aux[2 * a.nvol + c], ww = a.aux[3 * a.nvol + c];
    double tt = a.aux[5 * a.nvol + c], mu = a.aux[6 * a.nvol + c];
    double nu = ri * mu;
    double kr = nu / a.prandtl;
    double cs = sqrt(a.gamloc * a.rgas0 * tt);
    v[0] = (fabs(uu) + cs) * a.dcsidx[i - 1];
    v[1] = (fabs(vv) + cs) * a.detady[j - 1];
    v[2] = (fabs(ww) + cs) * a.dzitdz[k - 1];
    v[3] = nu * a.dcsidxs[i - 1];
    v[4] = nu * a.detadys[j - 1];
    v[5] = nu * a.dzitdzs[k - 1];
    v[6] = kr * a.dcsidxs[i - 1];
    v[7] = kr * a.detadys[j - 1];
    v[8] = kr * a.dzitdzs[k - 1];
  }
#pragma unroll
  for (int r = 0; r < DTN_SLOTS; ++r)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[r] = fmax(v[r], __shfl_down_sync(0xffffffffu, v[r], o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int r = 0; r < DTN_SLOTS; ++r) sm[r * (DTN_NT / 32) + warp] = v[r];
  __syncthreads();
  if (threadIdx.x < DTN_SLOTS) {
    double m = 0.0;
    for (int wq = 0; wq < DTN_NT / 32; ++wq) m = fmax(m, sm[threadIdx.x * (DTN_NT / 32) + wq]);
    part[(long long)blockIdx.x * DTN_SLOTS + threadIdx.x] = m;
  }
}

__global__ void __launch_bounds__(1024) k_dt_noalloc_finish(const double* __restrict__ part, int nblk, double cfl,
                                                            double* __restrict__ dt) {
  __shared__ double sm[32];
  double m = 0.0;
  for (int b = threadIdx.x; b < nblk * DTN_SLOTS; b += 1024) m = fmax(m, part[b]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int wq = 0; wq < 32; ++wq) a = fmax(a, sm[wq]);
    double dt_min = 1.0 / a;
    *dt = cfl * dt_min;
  }
}

static_assert((long long)DTN_MAX_BLOCKS * DTN_NT == STREAMS_B200_DT_NOALLOC_MAX_CELLS,
              "the header's cell limit must match the static scratch");

}  // namespace

namespace sb200 {
void set_global_error(const std::string& msg);  // backend.cu: text of streams_b200_global_error()
}

namespace {
int fail(int code, const std::string& msg) {
  sb200::set_global_error(msg);
  return code;
}
}  // namespace

extern "C" {

int streams_b200_compute_dt_noalloc(int nx, int ny, int nz, int ng, const double* w, const double* aux,
                                    const double* dcsidx, const double* detady, const double* dzitdz,
                                    const double* dcsidxs, const double* detadys, const double* dzitdzs,
                                    double rgas0, double prandtl, double gamma, double cfl, double* dt,
                                    void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || ng < 1)
    return fail(STREAMS_B200_EINVAL, "compute_dt_noalloc: sizes must be positive");
  const long long ncell = (long long)nx * ny * nz;
  if (ncell > (long long)DTN_MAX_BLOCKS * DTN_NT)
    return fail(STREAMS_B200_EINVAL, "compute_dt_noalloc: " + std::to_string(ncell) +
                                         " interior cells exceed the static scratch limit of " +
                                         std::to_string((long long)DTN_MAX_BLOCKS * DTN_NT) +
                                         " cells; use streams_b200_compute_dt on a context instead");
  if (!w || !aux || !dcsidx || !detady || !dzitdz || !dcsidxs || !detadys || !dzitdzs || !dt)
    return fail(STREAMS_B200_EINVAL, "compute_dt_noalloc: null array pointer");
  if (!(cfl > 0)) return fail(STREAMS_B200_EINVAL, "compute_dt_noalloc: cfl must be positive");
  // one constant gamma: a thermally perfect gas (gamma(T) per cell) must use the context's
  // streams_b200_compute_dt; nonsense constants are refused rather than giving a wrong dt
  if (!(gamma > 1)) return fail(STREAMS_B200_EINVAL, "compute_dt_noalloc: gamma must exceed 1 (calorically perfect gas)");
  if (!(rgas0 > 0)) return fail(STREAMS_B200_EINVAL, "compute_dt_noalloc: rgas0 must be positive");
  if (!(prandtl > 0)) return fail(STREAMS_B200_EINVAL, "compute_dt_noalloc: prandtl must be positive");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(STREAMS_B200_ENODEV, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= DTN_MAX_DEVICES) return fail(STREAMS_B200_ENODEV, "compute_dt_noalloc: device index too large");
  double* part = nullptr;
  {
    // one-time set-up per device, with that device current: the host-side name of the array is
    // only a stand-in, the kernel needs the array's device address
    std::lock_guard<std::mutex> lk(g_mutex);
    if (!g_partials_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_dt_partials);
      if (e != cudaSuccess)
        return fail(STREAMS_B200_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_partials_ptr[dev] = static_cast<double*>(p);
    }
    part = g_partials_ptr[dev];
  }
  DtArgs a;
  a.nx = nx; a.ny = ny; a.nz = nz; a.ng = ng;
  a.sx = nx + 2 * ng; a.sy = ny + 2 * ng;
  a.nvol = (long long)a.sx * a.sy * (nz + 2 * ng);
  a.w = w; a.aux = aux;
  a.dcsidx = dcsidx; a.detady = detady; a.dzitdz = dzitdz;
  a.dcsidxs = dcsidxs; a.detadys = detadys; a.dzitdzs = dzitdzs;
  a.rgas0 = rgas0; a.prandtl = prandtl; a.gamloc = gamma;
  const int nblk = (int)((ncell + DTN_NT - 1) / DTN_NT);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_dt_noalloc<<<nblk, DTN_NT, 0, s>>>(a, part);
  k_dt_noalloc_finish<<<1, 1024, 0, s>>>(part, nblk, cfl, dt);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(STREAMS_B200_ECUDA, std::string("compute_dt_noalloc launch: ") + cudaGetErrorString(e));
  return STREAMS_B200_OK;
}

}  // extern "C"
