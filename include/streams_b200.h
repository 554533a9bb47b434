/*
 * streams_b200.h -- C ABI of the B200 (sm_100a) backend for the per-Runge-Kutta-stage
 * right-hand side and update of the STREAmS-2 Cartesian compressible Navier-Stokes solver.
 *
 * Everything here is plain C: opaque handles, POD structs, host or device pointers and
 * sizes.  A Fortran solver object binds it with ISO_C_BINDING exactly as the HIP backend
 * binds its C++ wrappers (code/src/singleideal/kernels_amd.F90:1658-1677, passing
 * `type(c_ptr), value` arrays and `value` scalars).
 *
 * Conventions
 *   - Every entry point returns 0 on success and a negative STREAMS_B200_E* code on error.
 *     Nothing calls exit(); the message of the last failure on a context is returned by
 *     streams_b200_last_error(ctx) (streams_b200_global_error() when no context exists).
 *   - The conserved field w is the reference's field%w array: w(1-ng:nx+ng, 1-ng:ny+ng,
 *     1-ng:nz+ng, 1:5), Fortran order (i fastest, variable slowest), REAL64
 *     (code/src/field.F90:404-454).
 *   - A context owns all of its device memory and one CUDA stream.  Calls on one context
 *     are not reentrant; distinct contexts may be driven from distinct host threads.
 *   - The device path computes in FP64 (precision = 0) or in the mixed form (precision = 1:
 *     FP32 flux and viscous arithmetic with compensated flux-difference sums; FP64 state,
 *     RK register, temperature recovery and reductions).
 */
#ifndef STREAMS_B200_H
#define STREAMS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define STREAMS_B200_ABI_VERSION 3
/* largest number of cp(T) polynomial coefficients (indx_cp_r - indx_cp_l + 2) */
#define STREAMS_B200_MAX_CP 12

/* error codes */
#define STREAMS_B200_OK 0
#define STREAMS_B200_EINVAL -1      /* invalid argument or unsupported option */
#define STREAMS_B200_ECUDA -2       /* a CUDA runtime call failed */
#define STREAMS_B200_ENOMEM -3      /* device allocation failed or over budget */
#define STREAMS_B200_ENAN -4        /* NaN detected in a reduction (the reference's "boom") */
#define STREAMS_B200_ETIMEOUT -5    /* a bounded device wait gave up */
#define STREAMS_B200_ENODEV -6      /* no usable sm_100 device */

/*
 * Solver parameters.  Field names follow equation_singleideal_object
 * (code/src/singleideal/singleideal.F90:36-280) after initialize() has run, so the
 * Fortran side fills this struct from equation_base%... one to one.
 */
typedef struct streams_b200_params {
  /* sizes: interior cells of the (single) block and ghost layers (field%nx, ny, nz, grid%ng) */
  int nx, ny, nz, ng;
  /* numerics (singleideal.F90:489-545) */
  int ep_order;             /* central order; lmax = ep_order/2 (2, 4, 6, 8) */
  int nkeep;                /* KEEP(n) variant: 0 internal-energy split, <0 enthalpy split, >0 KEEP(n) */
  int weno_scheme;          /* WENO order = 2*weno_scheme-1 (1..4) */
  int weno_version;         /* 0 Jiang-Shu, 1 WENO-Z (weno_scheme 3 only) */
  int flux_splitting;       /* 0 Roe characteristic splitting, 1 component-wise Rusanov splitting
                               (sixth-order central / WENO5; tests/test_gpu_parity.py rusanov cases) */
  int conservative_viscous; /* 1 conservative 2nd-order viscous form, 0 non-conservative form at
                               visc_order (tests/test_gpu_parity.py nonconservative cases) */
  double sensor_threshold;  /* Ducros threshold; <0 full WENO, >1 full central */
  /* boundary conditions (bctags after the periodic normalisation, singleideal.F90:379-403) */
  int bctags[6];            /* xmin xmax ymin ymax zmin zmax: 0 periodic, 6 viscous wall */
  int force_zero_flux[6];   /* bc_preproc (singleideal.F90:4703-4750) */
  int eul_imin, eul_imax, eul_jmin, eul_jmax, eul_kmin, eul_kmax;
  int is_y_staggered;       /* staggered y walls (channel) */
  /* fluid (set_fluid_prop, singleideal.F90:2685-2774) */
  int visc_model;           /* 0 inviscid, 1 power law, 2 Sutherland */
  int calorically_perfect;  /* 1 constant cp, 0 cp(T) polynomial (thermally perfect, FP64 form) */
  double mu0, t0, rgas0, rho0, u0, l0;
  double sutherland_s, t_ref_dim, powerlaw_vtexp, prandtl;
  double cp0, cv0;          /* cp_coeff(0), cv_coeff(0) */
  double cp_last, cv_last;  /* cp_coeff(indx_cp_r+1), cv_coeff(indx_cp_r+1) */
  /* channel forcing (force_rhs / force_var, singleideal_cpu.F90:845-933) */
  int channel_case;
  double theta_wall, t_wall, t_bulk_target, volchan;
  /* time integration (runge_kutta_initialize, singleideal.F90:4773-4795) */
  int nrk;
  double rhork[4], gamrk[4];
  double cfl;               /* >0 CFL number, <0 fixed time step -cfl */
  /* arithmetic of the device path: 0 = FP64, 1 = mixed (FP32 fluxes, FP64 state) */
  int precision;
  /* open boundaries (boundary layer): characteristic non-reflecting type per face (bctags_nr of
   * equation_base; 0 none, 1, 2, 3, 6 as bc_nr_lat_x/y_kernel), free-stream state winf, p0 */
  int bctags_nr[6];
  double winf[5];
  double p0;
  /* recycling-rescaling inflow (bctags[0] = 10, recyc_prepare): station i_recyc, last node
   * below l0 jbl_inflow, betarecyc, and the crandom sequence the inflow plane is drawn from
   * (seed and the number of draws the set-up took) */
  int recyc, i_recyc, jbl_inflow;
  double betarecyc;
  unsigned int rng_seed;
  long long rng_draws;
  /* impinging oblique shock at the top (bctags[3] = 7, set_oblique_shock): impingement point,
   * shock angle [rad], tanh smoothing length, post-shock conserved state */
  double xshock_imp, shock_angle, tanhfacs;
  double winf_past_shock[5];
  /* thermally perfect gas (calorically_perfect = 0): cp(T)/rgas0 = sum of cp_coeff(l) (T/t0)^l,
   * l = indx_cp_l..indx_cp_r, and the energy datum at l = indx_cp_r+1, as set_fluid_prop leaves
   * cp_coeff and cv_coeff (times rgas0); stored at [l - indx_cp_l].  For calorically_perfect = 1
   * indx_cp_l = indx_cp_r = 0 and the two entries equal cp0, cp_last (cv0, cv_last). */
  int indx_cp_l, indx_cp_r;
  double cp_coeff[STREAMS_B200_MAX_CP];
  double cv_coeff[STREAMS_B200_MAX_CP];
} streams_b200_params;

/*
 * One-dimensional grid data of the block (field%x, y, z, yn and the metrics of
 * set_local_grid, code/src/field.F90:456-516).  Host pointers; copied at create time.
 */
typedef struct streams_b200_grid {
  const double* x;          /* x(1-ng:nx+ng)   nx+2*ng values */
  const double* y;          /* y(1-ng:ny+ng)   ny+2*ng values */
  const double* z;          /* z(1-ng:nz+ng)   nz+2*ng values */
  const double* yn;         /* yn(1:ny+1)      cell faces in y */
  const double* dcsidx;     /* dcsidx(1:nx) */
  const double* detady;     /* detady(1:ny) */
  const double* dzitdz;     /* dzitdz(1:nz) */
  const double* dcsidxs;    /* dcsidxs(1:nx) */
  const double* detadys;    /* detadys(1:ny) */
  const double* dzitdzs;    /* dzitdzs(1:nz) */
  const double* coeff_deriv1; /* coeff_deriv1(1:4,1:4), Fortran order (l fastest) */
  const int* ep_ord_x;      /* ep_ord_change(i,*,*,1), i = 0..nx */
  const int* ep_ord_y;      /* ep_ord_change(*,j,*,2), j = 0..ny */
  const int* ep_ord_z;      /* ep_ord_change(*,*,k,3), k = 0..nz */
  /* second-derivative data of the non-conservative viscous form (conservative_viscous = 0;
   * may be NULL otherwise): compute_metrics (code/src/grid.F90:71-141) and get_deriv_coeffs */
  const double* dcsidx2;    /* dcsidx2(1:nx) */
  const double* detady2;    /* detady2(1:ny) */
  const double* dzitdz2;    /* dzitdz2(1:nz) */
  const double* coeff_deriv2; /* coeff_deriv2(0:4,1:4), Fortran order (l fastest) */
  /* recycling inflow data of recyc_prepare (recyc = 1 only; may be NULL otherwise) */
  const double* wmean_inflow; /* wmean(1-i, j, m), i = 1..ng, j = 1..ny, m = 1..4: i fastest */
  const double* yplus_inflow; /* yplus_inflow(1-ng:ny+ng) */
  const double* eta_inflow;   /* eta_inflow(1-ng:ny+ng) */
  const double* yplus_recyc;  /* yplus_recyc(1-ng:ny+ng) */
  const double* eta_recyc;    /* eta_recyc(1-ng:ny+ng) */
  const double* weta_inflow;  /* weta_inflow(1:ny) */
  const int* map_j_inn;       /* map_j_inn(1:ny) */
  const int* map_j_out;       /* map_j_out(1:ny) */
} streams_b200_grid;

typedef struct streams_b200_ctx streams_b200_ctx;

/* Library identification. */
int streams_b200_abi_version(void);
const char* streams_b200_global_error(void);

/*
 * Create a context: validates the parameters, allocates the device state and uploads the grid.
 * Replaces equation_singleideal_gpu_object%initialize / base_gpu%initialize
 * (code/src/singleideal/singleideal_gpu.F90 initialize; code/src/base_gpu.F90:2033-2064).
 */
int streams_b200_create(const streams_b200_params* p, const streams_b200_grid* g, streams_b200_ctx** out);
int streams_b200_destroy(streams_b200_ctx* ctx);
const char* streams_b200_last_error(const streams_b200_ctx* ctx);

/* Bytes of device memory a context with these parameters allocates (admission control). */
long long streams_b200_footprint_bytes(const streams_b200_params* p);

/*
 * Field transfer.  Replace base_gpu%copy_from_field / copy_to_field
 * (code/src/base_gpu.F90).  The host array is w(1-ng:nx+ng,1-ng:ny+ng,1-ng:nz+ng,5).
 * The _device variants take a device pointer with the same layout.
 */
int streams_b200_copy_from_field(streams_b200_ctx* ctx, const double* w_host);
int streams_b200_copy_to_field(streams_b200_ctx* ctx, double* w_host);
int streams_b200_copy_from_device(streams_b200_ctx* ctx, const double* w_dev);
int streams_b200_copy_to_device(streams_b200_ctx* ctx, double* w_dev);

/*
 * Preamble of run() (code/src/singleideal/singleideal_cpu.F90:1542-1557): update_ghost,
 * compute_aux, visflx(mode=2) for the initial Ducros sensor, bcswap_var of the sensor,
 * zero_flux.  Call once after the initial field is uploaded.
 */
int streams_b200_init_run(streams_b200_ctx* ctx);

/*
 * compute_aux(central=1, ghost=0) + compute_dt (singleideal_cpu.F90:1476-1517);
 * the new time step is kept on the device and also returned in *dt (may be NULL).
 */
int streams_b200_compute_dt(streams_b200_ctx* ctx, double* dt);

/* Set the device time step explicitly (cfl < 0 runs, or a host-imposed dt). */
int streams_b200_set_dt(streams_b200_ctx* ctx, double dt);

/*
 * One Runge-Kutta step = nrk stages of the RHS and update, with the channel bulk
 * forcing, ghost fills and the stage-3 sensor update.  Replaces rk_sync
 * (code/src/singleideal/singleideal_cpu.F90:332-409).  Uses the device time step.
 */
int streams_b200_rk_sync(streams_b200_ctx* ctx);

/*
 * Advance nsteps time steps without host synchronisation: each step recomputes dt when
 * (icyc - icyc0) % iter_dt_recompute == 0 (the run() loop, singleideal_cpu.F90:1576-1590),
 * then runs rk_sync and accumulates the time on the device.  Not captured if nsteps == 0.
 */
int streams_b200_advance(streams_b200_ctx* ctx, int nsteps, int iter_dt_recompute, int icyc_start, int icyc0);

/* Read device scalars: out[0..6] = dt, time, dpdx, rhobulk, ubulk, tbulk, tbdiff. */
int streams_b200_get_scalars(streams_b200_ctx* ctx, double out[7]);
int streams_b200_set_time(streams_b200_ctx* ctx, double time);

/*
 * compute_residual (singleideal_cpu.F90:1339-1364): out[0..6] = residual_rhou (sqrt of the
 * mean of (fln_2/dt)^2), rhomin, rhomax, tmin, tmax, pmin, pmax.  Returns STREAMS_B200_ENAN
 * (after filling out) when the residual is NaN.
 */
int streams_b200_compute_residual(streams_b200_ctx* ctx, double out[7]);

/* Fraction of WENO faces per direction (count_weno, singleideal_cpu.F90:1389-1429). */
int streams_b200_count_weno(streams_b200_ctx* ctx, double out[3]);

/* Wall shear / heat flux at j=1 (wallprop(1:nx,1:nz,2:4) of visflx_reduced_ord2). */
int streams_b200_get_wallprop(streams_b200_ctx* ctx, double* out /* nx*nz*3 */);

/*
 * Running statistics.  Replace equation_singleideal_object%compute_stats
 * (code/src/singleideal/singleideal.F90:2003-2179) and compute_stats_3d (:2513-2543) as
 * manage_output calls them (singleideal_gpu.F90:2012-2034): right after a completed rk_sync,
 * before the next step's compute_dt, with no upload in between (a download is allowed);
 * otherwise STREAMS_B200_EINVAL.  itav is the number of samples already averaged (the caller
 * increments it after the call, as manage_output does).  compute_stats adds the z-average of 70
 * point quantities (velocity derivatives of order visc_order, T and mu of the stage-3 aux pass,
 * Reynolds stresses, vorticity, viscous stresses, ...) to w_stat(70, nx, ny):
 *   w_stat = (w_stat*itav + w_stat_z)/(itav + 1);
 * compute_stats_3d does the same per cell for the 14 quantities of w_stat_3d(14, nx, ny, nz).
 * The arrays live on the device (allocated on first use, zero-initialised: 2*70*nx*ny and
 * 14*nx*ny*nz doubles, plus a scratch of 3 doubles per ghosted point for the velocities of a
 * sample) in the reference's layout, statistic index fastest.  get_stats /
 * set_stats copy which = 0 (w_stat), 1 (w_stat_z of the last sample, read only) or
 * 2 (w_stat_3d); n is the buffer size in doubles (set_stats: exactly the array size), e.g. to
 * restore w_stat from stat.bin on a restart with restart_type = 2 (read_stats, :1646-1700).
 */
#define STREAMS_B200_NV_STAT 70
#define STREAMS_B200_NV_STAT_3D 14
int streams_b200_compute_stats(streams_b200_ctx* ctx, int itav);
int streams_b200_compute_stats_3d(streams_b200_ctx* ctx, int itav);
int streams_b200_get_stats(streams_b200_ctx* ctx, int which, double* out, long long n);
int streams_b200_set_stats(streams_b200_ctx* ctx, int which, const double* in, long long n);

/* Synchronise the context's stream and report any asynchronous error. */
int streams_b200_synchronize(streams_b200_ctx* ctx);
/* Non-blocking completion check (no counterpart in the reference): 1 while work issued on the
 * context's stream is pending, 0 once it has completed, a negative status on a device error.
 * The serving loop polls it instead of waiting on every resident solve. */
int streams_b200_query(streams_b200_ctx* ctx);

/* Number of kernel launches issued by this context since creation (instrumentation). */
long long streams_b200_launch_count(const streams_b200_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that order their own work after it. */
int streams_b200_get_stream(streams_b200_ctx* ctx, void** stream);

/*
 * Per-kernel CUDA-event timing.  profile_enable(ctx, 1) records an event pair around every
 * launch of the context from then on (0 stops and keeps the totals; -1 clears them);
 * profile_read resolves the recorded events and returns the accumulated device time and launch
 * count of kernel kid (0 <= kid < streams_b200_kernel_count()).
 */
int streams_b200_profile_enable(streams_b200_ctx* ctx, int on);
int streams_b200_profile_read(streams_b200_ctx* ctx, int kid, double* total_ms, long long* count);
int streams_b200_kernel_count(void);
const char* streams_b200_kernel_name(int kid);
/*
 * Architecture of the loaded device code: cudaFuncGetAttributes(...).binaryVersion of one kernel
 * of each CUDA source of the library (100 for sm_100a) into out[0 .. min(max, n) - 1]; returns
 * n, the number of sources (3), or STREAMS_B200_EINVAL.  A value of -1 means the driver could not
 * load that source's kernels on the current device.  No counterpart in the reference.
 */
int streams_b200_kernel_binary_versions(int* out, int max);

/*
 * Diagnostics: copy an internal device array to the host (synchronous).  which =
 *   0  aux fields rho, u, v, w, H, T, mu (7 ghosted arrays, w_aux(:,:,:,1:7))   7*nvol doubles
 *   1  right-hand side fl of the last completed stage (5 interior arrays)        5*nint doubles
 *   2  Ducros sensor used by the next stage's fluxes (w_aux(1:nx,1:ny,1:nz,8))    nint doubles
 *   3  div/3 of the last stage (w_aux(1:nx,1:ny,1:nz,10))                        nint doubles
 * n is the capacity of out in doubles.
 */
int streams_b200_debug_fetch(streams_b200_ctx* ctx, int which, double* out, long long n);

/*
 * Launch shape of the y and z flux passes (no counterpart in the reference, whose GPU kernels
 * use fixed thread blocks).  Each (x, y-or-z) line is cut into segments of at least
 * march_minseg cells so that about march_threads threads run.  Defaults: 151552 (148 SMs x
 * 1024) and 16.  Limits: march_minseg >= 4, 1024 <= march_threads <= 2^26.  A tuning changes
 * only the thread partition; results are bit-identical for equal tunings and otherwise differ
 * in the summation order of the force_rhs block partials.  get_tuning reads the current values.
 */
int streams_b200_set_tuning(streams_b200_ctx* ctx, long long march_threads, int march_minseg);
int streams_b200_get_tuning(streams_b200_ctx* ctx, long long* march_threads, int* march_minseg);

/*
 * Where the WENO faces of the hybrid scheme are computed (no counterpart in the reference, whose
 * euler kernels evaluate the WENO branch in place).  At the first stage of each step the faces
 * of each direction whose stencil sees the Ducros sensor are listed on the device; when a
 * direction's list holds at most max_fraction of its faces, their fluxes are computed apart by
 * a kernel of their own and the direction's hybrid pass reads them from a face buffer, otherwise
 * the hybrid pass computes them itself.  The choice is made on the device per direction and
 * step (no host synchronisation); the lists are built only when a sample of every 16th plane is
 * within the fraction.  1 always computes the WENO faces apart; 0 turns the split off (the hybrid
 * passes alone, no list or face kernel launched).  Default: 0.55 for boxes of at least 2^21
 * cells, 0 for smaller ones (launch-bound, where the split's extra launches cost more than it
 * saves).  The face buffers (about 53 bytes per cell) are allocated when the split is first on;
 * STREAMS_B200_ENOMEM if that fails.  Both forms evaluate the same arithmetic: FP64 results are
 * identical up to the compiler's contraction of the WENO arithmetic in the two kernels
 * (observed: bit-identical, or differences of a few ulp).
 */
int streams_b200_set_weno_split(streams_b200_ctx* ctx, double max_fraction);
int streams_b200_get_weno_split(streams_b200_ctx* ctx, double* max_fraction);

/*
 * Batched form: many independent contexts (boxes of any size and flow parameters, one device,
 * one precision each) advanced together.  The step sequences (compute_dt + rk_sync) of
 * steps_per_graph steps are captured once into one CUDA graph; each streams_b200_batch_advance
 * replays it.  Boxes whose stages take the same kernels (precision, scheme orders and form,
 * channel forcing, viscous form; periodic or staggered-wall faces only, WENO faces computed
 * inside the hybrid passes) form a group that advances by shared launches: one launch per
 * kernel kind and stage covers every box of the group, each block working on one box in the
 * block partition the box uses alone.  Other boxes keep their own step sequence as a parallel
 * branch of the graph.  No counterpart in the reference (one box per MPI rank there).
 *
 *   steps_per_graph  time steps per graph replay (>= 1)
 *   dt_every         dt is recomputed at batch steps s with s % dt_every == 0 (contexts with
 *                    cfl < 0 keep their fixed dt); must divide steps_per_graph
 *
 * batch_advance(b, nsteps) advances every box by exactly nsteps steps: a box that has not
 * completed a step since its last upload/init_run first takes one ordinary step (the graph
 * holds the steady step sequence), then whole graph replays, then the remainder as ordinary
 * steps.  It is asynchronous; streams_b200_batch_synchronize waits for all boxes.  Results
 * are bit-identical to advancing each context alone with streams_b200_advance(ctx, n, dt_every,
 * s0, 0) under the same tuning.  Contexts must outlive the batch and must not be profiled
 * (profile_enable) while in a batch.  Work issued on a box's own stream between batch calls
 * (uploads, direct advance, downloads) is ordered with the replays; a re-tuned box makes the
 * next advance capture the graph again, and streams_b200_batch_invalidate forces that.
 */
typedef struct streams_b200_batch streams_b200_batch;
int streams_b200_batch_create(streams_b200_ctx** ctxs, int n, int steps_per_graph, int dt_every,
                              streams_b200_batch** out);
int streams_b200_batch_advance(streams_b200_batch* b, int nsteps);
int streams_b200_batch_synchronize(streams_b200_batch* b);
int streams_b200_batch_invalidate(streams_b200_batch* b);
/* Class of a context for shared launches: contexts of one batch with equal non-negative
 * classes (and equal RK coefficients) form a group; -1 for a context that always advances on
 * its own branch. */
int streams_b200_batch_class(streams_b200_ctx* ctx, long long* cls);
/* Graph replays issued and kernel launches they contain (instrumentation). */
int streams_b200_batch_stats(streams_b200_batch* b, long long* replays, long long* launches_per_replay);
/* Shared launches: the boxes of a class in groups_per_class groups (1, the default: one group per
 * class; the groups' launch chains are parallel branches of the graph), or 0: every box its own
 * branch. */
int streams_b200_batch_set_shared_launches(streams_b200_batch* b, int groups_per_class);
/* Groups that share launches and the boxes they hold. */
int streams_b200_batch_groups(streams_b200_batch* b, int* ngroups, int* nshared);
const char* streams_b200_batch_last_error(streams_b200_batch* b);
int streams_b200_batch_destroy(streams_b200_batch* b);

/*
 * CFL time step over caller-owned device arrays, allocating nothing.
 *
 * No counterpart in the reference: STREAmS-2's compute_dt always runs on the solver's own
 * arrays.  This entry point is for callers that cannot let a library call cudaMalloc, such as
 * a host code that owns every byte of device memory through its own pool or mapping (a Fortran
 * solver that keeps its arrays under OpenACC or CUDA Fortran), or one that runs under a fixed
 * memory budget in which an allocation inside the time loop may fail or fragment the pool.
 * It needs no context: the caller passes its own device arrays and a device word for dt.
 *
 *   w        device w(1-ng:nx+ng,1-ng:ny+ng,1-ng:nz+ng,5)   (only the density is read)
 *   aux      device aux fields rho,u,v,w,H,T,mu, 7 arrays of the same ghosted shape
 *            (the layout of streams_b200_debug_fetch(ctx, 0, ...)), current for w
 *   dcsidx.. device metric arrays of nx, ny, nz entries (set_local_grid, field.F90:456-516)
 *   gamma    cp/(cp - rgas0) of the calorically perfect gas, > 1.  The time step of a thermally
 *            perfect gas (calorically_perfect = 0) takes gamma(T) per cell: such cases must use
 *            the context's streams_b200_compute_dt.  gamma <= 1, rgas0 <= 0 or prandtl <= 0
 *            return STREAMS_B200_EINVAL.
 *   dt       device address that receives cfl / max(inverse time scales)
 *   stream   cudaStream_t on which both kernels run (asynchronous; NULL = default stream)
 *
 * The block partial maxima live in a static device array compiled into the library, so every
 * GPU that loads the library holds 1.125 MiB for it until the process exits.  At most
 * STREAMS_B200_DT_NOALLOC_MAX_CELLS interior cells per call; larger sizes return
 * STREAMS_B200_EINVAL with the reason in streams_b200_global_error().  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  All calls share the array: calls whose kernels overlap on the
 * GPU (other streams, other host threads) race on it and must be serialised by the caller.
 */
#define STREAMS_B200_DT_NOALLOC_MAX_CELLS 4194304LL
int streams_b200_compute_dt_noalloc(int nx, int ny, int nz, int ng, const double* w, const double* aux,
                                    const double* dcsidx, const double* detady, const double* dzitdz,
                                    const double* dcsidxs, const double* detadys, const double* dzitdzs,
                                    double rgas0, double prandtl, double gamma, double cfl, double* dt,
                                    void* stream);

#ifdef __cplusplus
}
#endif

#endif /* STREAMS_B200_H */
