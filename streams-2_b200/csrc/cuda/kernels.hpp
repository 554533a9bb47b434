// Host-side launchers of the stage kernels (implemented in stage_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace sb200 {

// Kernel identifiers of the optional per-kernel event profiler.
enum KernelId {
  K_AUX = 0, K_EULER_X, K_VISC, K_EULER_Y, K_EULER_Z, K_FINISH_RHS, K_UPDATE, K_FINISH_UPD, K_DT, K_DT_FINISH,
  K_INIT_SENSOR, K_APPLY_SHIFT, K_FILL_GHOSTS, K_COUNT_WENO, K_ADD_TIME, K_BC_FILL, K_BC_NR, K_RAND_PLANE,
  K_STATS, K_STATS3D, K_WENO_LIST, K_WENO_FACES, K_NUM
};
const char* kernel_name(int kid);
// binaryVersion (10 * major + minor) of one kernel of each CUDA source, as loaded by the driver
int binary_version_stage();
int binary_version_bc();
int binary_version_stats();

// Per-kernel CUDA-event timing (off unless enabled on the context).
struct Prof {
  bool on = false;
  struct Rec { int kid; cudaEvent_t a, b; };
  std::vector<Rec> pending;
  double total_ms[K_NUM] = {};
  long long count[K_NUM] = {};
  void begin(int kid, cudaStream_t s);
  void end(cudaStream_t s);
  cudaError_t resolve();  // synchronises on the recorded events and accumulates
  void reset();
};

// Device buffers of one context (single block).
struct DevState {
  double* w = nullptr;        // ghosted, 5 variables
  // FP64 form
  double* aux = nullptr;      // ghosted, 8 variables: rho, u, v, w, H, T, mu, sound speed
  double* sensor = nullptr;   // interior: Ducros theta used by the fluxes (both forms)
  double* sensor_next = nullptr;
  double* div3 = nullptr;     // interior: div/3
  // mixed form: primitive fields and div/3 in FP32 (the sensor stays FP64 in both forms)
  float* auxf = nullptr;
  float* div3f = nullptr;
  double* vel64 = nullptr;    // FP64 velocities of the stage-3 aux pass (3 x nvol): the stage-3 sensor
  double* fl_a = nullptr;     // interior, 5 variables (two RK registers, ping-pong)
  double* fl_b = nullptr;
  double* wallprop = nullptr; // nx*nz*3
  double* red = nullptr;      // block partials of the reductions
  Scalars* sc = nullptr;      // device scalars
  long long red_capacity = 0; // doubles in red
  // recycling inflow: the random plane inflow_random_plane(j,k,c) at [(c*nz + k-1)*ny + j-1],
  // the spanwise means of the recycling plane [(m*ny + j-1)*ng + i-1], the generator state
  double* rplane = nullptr;
  unsigned int* rwords = nullptr;  // raw draws of one stage (the full 32-bit words)
  // jump-ahead table of the parallel generator: for chunk c of RAND_CHUNK draws, the 31
  // coefficients of t^(31 + c RAND_CHUNK) mod (t^31 - t^28 - 1) over the integers mod 2^32
  unsigned int* rcoef = nullptr;
  double* recyc_av = nullptr;
  RngState* rng = nullptr;
  // running statistics (allocated on first use), statistic index fastest:
  // w_stat(70, nx, ny), w_stat_z(70, nx, ny), w_stat_3d(14, nx, ny, nz)
  double* wstat = nullptr;
  double* wstat_z = nullptr;
  double* wstat3d = nullptr;
  double* wstat_vel = nullptr;  // scratch of a sample: velocities at interior and ghost points (3 x nvol)
  Prof* prof = nullptr;       // optional per-kernel timing
};

// Launch with optional per-kernel event timing on the launching stream
#define SB_LAUNCH(dst, kid, s, ...)                                  \
  do {                                                               \
    if ((dst).prof && (dst).prof->on) (dst).prof->begin((kid), (s)); \
    __VA_ARGS__;                                                     \
    if ((dst).prof && (dst).prof->on) (dst).prof->end((s));          \
  } while (0)

struct StageArgs {
  int istep;           // 1..nrk
  double rhork, gamrk; // RK coefficients of the stage
  int apply_shift;     // apply the pending force_var energy shift before the aux pass
  int want_stats;      // update pass accumulates residual and min/max (stage 3)
  int run_aux;         // recompute aux (skipped when it is already current)
  int add_time;        // accumulate time += dt on the device after the stage
};

// Launch-count instrumentation is kept by the caller.
cudaError_t launch_aux(const Geom& g, DevState& d, int apply_shift, cudaStream_t s, long long* nl);
cudaError_t launch_init_sensor(const Geom& g, DevState& d, cudaStream_t s, long long* nl);
cudaError_t launch_dt(const Geom& g, DevState& d, double cfl, cudaStream_t s, long long* nl);
// One RK stage.  fl_prev holds the previous stage's right-hand side (unused at stage 1),
// fl_new receives this stage's.  At stage 3 the next Ducros sensor becomes current.
cudaError_t launch_stage(const Geom& g, DevState& d, const StageArgs& a, double* fl_prev, double* fl_new,
                         cudaStream_t s, long long* nl);
bool stage_supported(int lmax_base, int weno_scheme);
cudaError_t launch_apply_shift(const Geom& g, DevState& d, cudaStream_t s, long long* nl);
cudaError_t launch_fill_ghosts(const Geom& g, DevState& d, cudaStream_t s, long long* nl);
cudaError_t launch_count_weno(const Geom& g, DevState& d, cudaStream_t s, long long* nl);
cudaError_t launch_add_time(DevState& d, cudaStream_t s, long long* nl);

// partial-sum slots needed for a geometry
// open boundaries (bc_kernels.cu)
cudaError_t launch_bc_fill(const Geom& g, DevState& d, cudaStream_t s, long long* nl);
// draws per chunk of the parallel inflow-plane generator
constexpr int RAND_CHUNK = 64;
// The jump-ahead table (nchunk x 31 words) of a stage's draws, built on the host at create.
void rand_jump_table(long long total, std::vector<unsigned int>& table);
cudaError_t launch_rand_plane(const Geom& g, DevState& d, cudaStream_t s, long long* nl);
cudaError_t launch_bc_nr(const Geom& g, DevState& d, double* fl, cudaStream_t s, long long* nl);
bool has_stored_ghosts(const Geom& g);
// running statistics (stats_kernels.cu), sampled after a completed step: fl2 / fl3 are the RK
// registers written by stages 2 and 3, pending says whether the force_var shift is still pending
cudaError_t launch_stats(const Geom& g, DevState& d, const double* fl2, const double* fl3, double rhork3,
                         double gamrk3, int pending, int itav, cudaStream_t s, long long* nl);
cudaError_t launch_stats3d(const Geom& g, DevState& d, int itav, cudaStream_t s, long long* nl);
long long reduction_slots(const Geom& g);

// Launches over a box table (batch_kernels.cu): the stages of a group of boxes, one launch per
// kernel kind for all of them.  Per box: its geometry, device buffers and launch shapes.
struct BoxRec {
  Geom g;
  double* w;
  void* aux;   // double (FP64 form) or float (mixed form)
  void* div3;
  double* sensor;
  double* sensor_next;
  double* vel64;
  double* fl_a;  // RK registers: stage 2 writes fl_b, stages 1 and 3 write fl_a
  double* fl_b;
  double* wallprop;
  double* red;
  Scalars* sc;
  double cfl;
  int sly, nsy, slz, nsz;  // march segments (length, count) of the y and z passes
  unsigned xg[3];          // grid of the x pass (one-dimensional)
  unsigned nb_vol, nb_pt, nb_y, nb_z;  // blocks of the aux pass, pointwise passes, y and z passes
  unsigned nb_vs;                      // blocks of the staged viscous pass
  unsigned nb_up;                      // blocks of the update and time-step passes
};
// block of a launch over a box table: the box and the block's index in the box's own grid
struct BlockRef {
  unsigned box, local;
};
enum BatchKind { BK_VOL = 0, BK_PT, BK_X, BK_Y, BK_Z, BK_VS, BK_UP, BK_NUM };
struct BoxTable {
  int nbox = 0;
  BoxRec* rec = nullptr;       // device
  BlockRef* blocks = nullptr;  // device: the blocks of each kind, box after box
  long long off[BK_NUM] = {};
  unsigned cnt[BK_NUM] = {};
  Geom g0{};  // host copy of the first box's geometry: the group's common configuration
};
// Group key of a geometry (boxes with equal keys share launches), -1 for a box whose stage
// needs launches that the table form does not have (stored ghosts, recycling inflow,
// non-reflecting faces, WENO faces computed apart).
long long batch_key(const Geom& g);
BoxRec box_rec(const Geom& g, const DevState& d, double* fl_a, double* fl_b, double cfl);
cudaError_t box_table_build(BoxTable& t, const std::vector<BoxRec>& recs, cudaStream_t s);
void box_table_free(BoxTable& t, cudaStream_t s);
cudaError_t batch_launch_aux(const BoxTable& t, int apply_shift, cudaStream_t s, long long* nl);
cudaError_t batch_launch_dt(const BoxTable& t, cudaStream_t s, long long* nl);
cudaError_t batch_launch_stage(const BoxTable& t, const StageArgs& a, cudaStream_t s, long long* nl);

}  // namespace sb200
