// Host launchers of the stage kernels (stage_device.cuh): one Runge-Kutta stage, the time
// step, the aux and sensor passes, and the per-kernel profiler.
#include <algorithm>

#include "stage_device.cuh"

namespace sb200 {


const char* kernel_name(int kid) {
  static const char* names[K_NUM] = {"k_aux", "k_euler_x", "k_visc", "k_euler_y", "k_euler_z", "k_finish_rhs",
                                     "k_update", "k_finish_upd", "k_dt", "k_dt_finish", "k_init_sensor",
                                     "k_apply_shift", "k_fill_ghosts", "k_count_weno", "k_add_time",
                                     "k_bc_fill", "k_bc_nr", "k_rand_plane", "k_stats", "k_stats3d",
                                     "k_weno_list", "k_weno_faces"};
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

long long reduction_slots(const Geom& g) {
  long long a = (long long)nblocks(g.nint, 256) * (NRED_UPD > 9 ? NRED_UPD : 9);
  int sl, ns;
  long long nt;
  // the largest segment count any tuning can reach: segments of MARCH_MINSEG_MIN cells
  march_split_with(g, 2, 1LL << 40, MARCH_MINSEG_MIN, &sl, &ns, &nt);
  long long b = (long long)nblocks(nt, MT_NT) * 5;
  return a > b ? a : b;
}


// A pending energy shift is applied to the interior in its own pass first: the aux pass reads
// interior points as the sources of ghost states, so it must not rewrite them itself.
template <class R, bool TP>
static void aux_launch_tp(const Geom& g, DevState& d, int apply_shift, int write_ghost, int kid, cudaStream_t s,
                          long long* nl, double* vel) {
  if (apply_shift) {
    SB_LAUNCH(d, K_APPLY_SHIFT, s,
              k_apply_shift<R, TP><<<nblocks(g.nint, AUX_NT), AUX_NT, 0, s>>>(g, d.w, aux_of<R>(d), d.sc));
    ++*nl;
  }
  SB_LAUNCH(d, kid, s,
            k_aux<R, TP><<<nblocks(g.nvol, AUX_NT), AUX_NT, 0, s>>>(g, d.w, aux_of<R>(d), write_ghost, vel));
  ++*nl;
}
// the thermally perfect instantiations exist for the FP64 form only
template <class R>
static void aux_launch(const Geom& g, DevState& d, int apply_shift, int write_ghost, int kid, cudaStream_t s,
                       long long* nl, double* vel = nullptr) {
  if constexpr (sizeof(R) == sizeof(double)) {
    if (!g.calorically_perfect) {
      aux_launch_tp<R, true>(g, d, apply_shift, write_ghost, kid, s, nl, vel);
      return;
    }
  }
  aux_launch_tp<R, false>(g, d, apply_shift, write_ghost, kid, s, nl, vel);
}

cudaError_t launch_aux(const Geom& g, DevState& d, int apply_shift, cudaStream_t s, long long* nl) {
  if (g.precision == 1) aux_launch<float>(g, d, apply_shift, 0, K_AUX, s, nl);
  else aux_launch<double>(g, d, apply_shift, 0, K_AUX, s, nl);
  return cudaGetLastError();
}

cudaError_t launch_fill_ghosts(const Geom& g, DevState& d, cudaStream_t s, long long* nl) {
  if (g.precision == 1) aux_launch<float>(g, d, 0, 2, K_FILL_GHOSTS, s, nl);
  else aux_launch<double>(g, d, 0, 2, K_FILL_GHOSTS, s, nl);
  return cudaGetLastError();
}

cudaError_t launch_apply_shift(const Geom& g, DevState& d, cudaStream_t s, long long* nl) {
  if (g.precision == 1)
    SB_LAUNCH(d, K_APPLY_SHIFT, s, k_apply_shift<float><<<nblocks(g.nint, AUX_NT), AUX_NT, 0, s>>>(g, d.w, d.auxf, d.sc));
  else if (!g.calorically_perfect)
    SB_LAUNCH(d, K_APPLY_SHIFT, s,
              k_apply_shift<double, true><<<nblocks(g.nint, AUX_NT), AUX_NT, 0, s>>>(g, d.w, d.aux, d.sc));
  else
    SB_LAUNCH(d, K_APPLY_SHIFT, s, k_apply_shift<double><<<nblocks(g.nint, AUX_NT), AUX_NT, 0, s>>>(g, d.w, d.aux, d.sc));
  ++*nl;
  return cudaGetLastError();
}

cudaError_t launch_init_sensor(const Geom& g, DevState& d, cudaStream_t s, long long* nl) {
  if (!g.conservative_viscous)
    SB_LAUNCH(d, K_INIT_SENSOR, s, k_sensor64<<<nblocks(g.nint, 256), 256, 0, s>>>(g, d.w, d.sensor, 3));
  else if (g.precision == 1)
    SB_LAUNCH(d, K_INIT_SENSOR, s, k_sensor64<<<nblocks(g.nint, 256), 256, 0, s>>>(g, d.w, d.sensor, 0));
  else
    SB_LAUNCH(d, K_INIT_SENSOR, s, k_init_sensor<double><<<nblocks(g.nint, 256), 256, 0, s>>>(g, d.aux, d.sensor));
  ++*nl;
  return cudaGetLastError();
}

cudaError_t launch_dt(const Geom& g, DevState& d, double cfl, cudaStream_t s, long long* nl) {
  const unsigned nb = pt_blocks(g.nint);
  if (g.precision == 1)
    SB_LAUNCH(d, K_DT, s, k_dt<float><<<nb, 256, 0, s>>>(g, d.w, d.auxf, d.red));
  else
    SB_LAUNCH(d, K_DT, s, k_dt<double><<<nb, 256, 0, s>>>(g, d.w, d.aux, d.red));
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

template <class R, int LB, int WS, int FS = 0>
static cudaError_t stage_impl(const Geom& g, DevState& d, const StageArgs& a, double* fl_prev, double* fl_new,
                              cudaStream_t s, long long* nl) {
  const dim3 xb(XF_TX, XF_TY);
  const unsigned xg = x_blocks(g);
  int sly, nsy, slz, nsz;
  long long nty, ntz;
  march_split(g, 1, &sly, &nsy, &nty);
  march_split(g, 2, &slz, &nsz, &ntz);
  const unsigned gyb = nblocks(nty, MT_NT), gzb = nblocks(ntz, MT_NT);
  R* aux = aux_of<R>(d);
  double* sensor = d.sensor;
  double* sensor_next = d.sensor_next;
  R* div3 = div3_of<R>(d);
  const bool fp64 = sizeof(R) == sizeof(double);
  // the mixed form's stage-3 sensor is taken in FP64 from velocities that this aux pass stores
  double* vel = (!fp64 && a.istep == 3) ? d.vel64 : nullptr;
  if (a.run_aux) aux_launch<R>(g, d, a.apply_shift, 0, K_AUX, s, nl, vel);
  // the hybrid passes hold the WENO scratch for the steps at which they compute WENO faces
  const size_t xsm = weno_scratch_bytes<R, WS>(XF_NT);
  const size_t msm = weno_scratch_bytes<R, WS>(MT_NT);
  const size_t wsm = weno_scratch_bytes<R, WS>(WF_NT);
  // per instantiation and device: allow more than 48 KB of dynamic shared memory
  static unsigned long long smem_set = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(smem_set & (1ULL << dev))) {
    cudaFuncSetAttribute(k_xflux<R, LB, WS, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xsm);
    cudaFuncSetAttribute(k_march<R, 1, LB, WS, false, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msm);
    cudaFuncSetAttribute(k_march<R, 2, LB, WS, false, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msm);
    cudaFuncSetAttribute(k_march<R, 2, LB, WS, true, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msm);
    if (SB_WENO_SPLIT) {
      cudaFuncSetAttribute(k_weno_faces<R, 0, LB, WS, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm);
      cudaFuncSetAttribute(k_weno_faces<R, 1, LB, WS, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm);
      cudaFuncSetAttribute(k_weno_faces<R, 2, LB, WS, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm);
      // a larger L1 rather than a fourth block (SB_WF_CARVEOUT)
      for (auto fn : {(const void*)k_weno_faces<R, 0, LB, WS, FS>, (const void*)k_weno_faces<R, 1, LB, WS, FS>,
                      (const void*)k_weno_faces<R, 2, LB, WS, FS>})
        cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, SB_WF_CARVEOUT);
    }
    smem_set |= 1ULL << dev;
  }
  // WENO faces apart: the lists at the first stage of a step (the sensor is fixed for the step),
  // the face fluxes before each hybrid pass
  const long long wnf = std::max(wface_count<0>(g), std::max(wface_count<1>(g), wface_count<2>(g)));
  const unsigned wgrid = (unsigned)std::min<long long>((long long)nblocks(wnf, WF_NT), 148LL * 16);
  const bool split_on = SB_WENO_SPLIT && g.wsplit_on;
  if (split_on && a.istep == 1) {
    SB_LAUNCH(d, K_WENO_LIST, s, cudaMemsetAsync(g.wcount, 0, 8 * sizeof(unsigned), s));
    // the sample counts, then the flags and the lists of the directions whose sample is within
    // the threshold (the others leave at once)
    const unsigned ns2 = (unsigned)(g.nz + WSAMPLE - 1) / WSAMPLE, ns2z = (unsigned)(g.nz + WSAMPLE) / WSAMPLE;
    SB_LAUNCH(d, K_WENO_LIST, s,
              k_weno_sample<0, WS><<<dim3(nblocks(g.nx + 1, 32), nblocks(g.ny, 8), ns2), WL_NT, 0, s>>>(g, sensor));
    SB_LAUNCH(d, K_WENO_LIST, s,
              k_weno_sample<1, WS><<<dim3(nblocks(g.nx, 32), nblocks(g.ny + 1, 8), ns2), WL_NT, 0, s>>>(g, sensor));
    SB_LAUNCH(d, K_WENO_LIST, s,
              k_weno_sample<2, WS><<<dim3(nblocks(g.nx, 32), nblocks(g.ny, 8), ns2z), WL_NT, 0, s>>>(g, sensor));
    // grid-stride over one resident wave (148 SMs x 8 blocks): a grid of one block per tile,
    // whose blocks leave at once when no list is built, measured 2.5 ms per step of empty
    // blocks on the 1024x256x192 boundary layer
    const unsigned gb = 148 * 8;
    SB_LAUNCH(d, K_WENO_LIST, s, k_weno_bits<<<gb, 256, 0, s>>>(g, sensor));
    SB_LAUNCH(d, K_WENO_LIST, s, k_weno_list<0, WS><<<gb, WL_NT, 0, s>>>(g));
    SB_LAUNCH(d, K_WENO_LIST, s, k_weno_list<1, WS><<<gb, WL_NT, 0, s>>>(g));
    SB_LAUNCH(d, K_WENO_LIST, s, k_weno_list<2, WS><<<gb, WL_NT, 0, s>>>(g));
    *nl += 7;
  }
  if (split_on) {
    SB_LAUNCH(d, K_WENO_FACES, s, k_weno_faces<R, 0, LB, WS, FS><<<wgrid, WF_NT, wsm, s>>>(g, aux));
    ++*nl;
  }
  SB_LAUNCH(d, K_EULER_X, s, k_xflux<R, LB, WS, FS><<<xg, xb, xsm, s>>>(g, aux, sensor, fl_new));
  if (g.conservative_viscous && SB_VISC_TILED)
    SB_LAUNCH(d, K_VISC, s,
              k_visc_tiled<R, (FS & 2) != 0><<<visc_tiled_blocks(g), VT_NT, 0, s>>>(
                  g, aux, fl_new, div3, sensor_next, d.wallprop, fp64 && a.istep == 3));
  else if (g.conservative_viscous)
    SB_LAUNCH(d, K_VISC, s,
              k_visc<R, (FS & 2) != 0><<<nblocks(g.nint, 256), 256, 0, s>>>(g, aux, fl_new, div3, sensor_next, d.wallprop,
                                                             fp64 && a.istep == 3));
  else
    SB_LAUNCH(d, K_VISC, s,
              k_visc_ns<R, (FS & 2) != 0><<<nblocks(g.nint, 256), 256, 0, s>>>(g, aux, fl_new, div3, sensor_next, d.wallprop,
                                                                fp64 && a.istep == 3));
  if (!fp64 && a.istep == 3) {
    // the mixed form takes the stage-3 sensor in FP64 from the stage's starting state
    if (a.run_aux)
      SB_LAUNCH(d, K_INIT_SENSOR, s,
                k_sensor_vel<<<nblocks(g.nint, 256), 256, 0, s>>>(g, d.vel64, sensor_next,
                                                                  g.conservative_viscous ? 1 : 2));
    else
      SB_LAUNCH(d, K_INIT_SENSOR, s,
                k_sensor64<<<nblocks(g.nint, 256), 256, 0, s>>>(g, d.w, sensor_next, g.conservative_viscous ? 1 : 2));
    ++*nl;
  }
  if (split_on) {
    SB_LAUNCH(d, K_WENO_FACES, s, k_weno_faces<R, 1, LB, WS, FS><<<wgrid, WF_NT, wsm, s>>>(g, aux));
    ++*nl;
  }
  if (gyb > 0) {
    SB_LAUNCH(d, K_EULER_Y, s,
              k_march<R, 1, LB, WS, false, FS><<<gyb, MT_NT, msm, s>>>(g, aux, sensor, fl_new, div3, d.w, fl_prev, d.sc,
                                                          a.rhork, a.gamrk, a.istep, sly, nsy, d.red));
    if (split_on) {
      SB_LAUNCH(d, K_EULER_Y, s,
                k_march<R, 1, LB, WS, false, FS, true><<<gyb, MT_NT, 0, s>>>(g, aux, sensor, fl_new, div3, d.w, fl_prev,
                                                                   d.sc, a.rhork, a.gamrk, a.istep, sly, nsy, d.red));
      ++*nl;
    }
  }
  if (split_on) {
    SB_LAUNCH(d, K_WENO_FACES, s, k_weno_faces<R, 2, LB, WS, FS><<<wgrid, WF_NT, wsm, s>>>(g, aux));
    ++*nl;
  }
  // the channel's force_rhs partials are a separate instantiation (fewer registers without them)
  if (g.channel_case) {
    SB_LAUNCH(d, K_EULER_Z, s,
              k_march<R, 2, LB, WS, true, FS><<<gzb, MT_NT, msm, s>>>(g, aux, sensor, fl_new, div3, d.w, fl_prev, d.sc,
                                                                  a.rhork, a.gamrk, a.istep, slz, nsz, d.red));
    if (split_on)
      SB_LAUNCH(d, K_EULER_Z, s,
                k_march<R, 2, LB, WS, true, FS, true><<<gzb, MT_NT, 0, s>>>(g, aux, sensor, fl_new, div3, d.w, fl_prev,
                                                                  d.sc, a.rhork, a.gamrk, a.istep, slz, nsz, d.red));
  } else {
    SB_LAUNCH(d, K_EULER_Z, s,
              k_march<R, 2, LB, WS, false, FS><<<gzb, MT_NT, msm, s>>>(g, aux, sensor, fl_new, div3, d.w, fl_prev, d.sc,
                                                                   a.rhork, a.gamrk, a.istep, slz, nsz, d.red));
    if (split_on)
      SB_LAUNCH(d, K_EULER_Z, s,
                k_march<R, 2, LB, WS, false, FS, true><<<gzb, MT_NT, 0, s>>>(g, aux, sensor, fl_new, div3, d.w, fl_prev,
                                                                   d.sc, a.rhork, a.gamrk, a.istep, slz, nsz, d.red));
  }
  if (split_on) ++*nl;
  *nl += 4;
  if (g.recyc) launch_rand_plane(g, d, s, nl);  // euler_z draws the inflow plane of the stage
  launch_bc_nr(g, d, fl_new, s, nl);
  if (g.channel_case) {
    SB_LAUNCH(d, K_FINISH_RHS, s, k_finish_rhs<<<1, FIN_NT, 0, s>>>(g, d.red, (long long)gzb, a.istep == 1, d.sc));
    ++*nl;
  }
  const unsigned nbu = pt_blocks(g.nint);
  SB_LAUNCH(d, K_UPDATE, s,
            k_update<R, (FS & 2) != 0><<<nbu, UPD_NT, 0, s>>>(g, d.w, fl_prev, fl_new, d.sc, a.rhork, a.gamrk, a.istep,
                                            a.want_stats, d.red, sensor_next, sensor, aux));
  SB_LAUNCH(d, K_FINISH_UPD, s, k_finish_upd<<<1, FIN_NT, 0, s>>>(g, d.red, nbu, a.want_stats, a.add_time, d.sc));
  *nl += 2;
  if (has_stored_ghosts(g)) launch_bc_fill(g, d, s, nl);  // update_ghost
  return cudaGetLastError();
}

// nkeep = 0 (the default) with the central flux specialised at compile time, else the general
// form; WENO-JS or, for the WENO5 scheme, WENO-Z
template <class R, int LB, int WS, int FS>
static cudaError_t stage_kg(const Geom& g, DevState& d, const StageArgs& a, double* fl_prev, double* fl_new,
                            cudaStream_t s, long long* nl) {
  if constexpr (WS == 3) {
    if (g.weno_version == 1) {
      if (g.nkeep != 0) return stage_impl<R, LB, WS, FS | 4 | 8>(g, d, a, fl_prev, fl_new, s, nl);
      return stage_impl<R, LB, WS, FS | 8>(g, d, a, fl_prev, fl_new, s, nl);
    }
  }
  if (g.nkeep != 0) return stage_impl<R, LB, WS, FS | 4>(g, d, a, fl_prev, fl_new, s, nl);
  return stage_impl<R, LB, WS, FS>(g, d, a, fl_prev, fl_new, s, nl);
}

template <class R>
static cudaError_t stage_dispatch(const Geom& g, DevState& d, const StageArgs& a, double* fl_prev, double* fl_new,
                                  cudaStream_t s, long long* nl) {
  if (!g.calorically_perfect) {
    // the thermally perfect gas is instantiated for the FP64 sixth-order central / WENO5 scheme
    if constexpr (sizeof(R) == sizeof(double)) {
      if (g.lmax_base == 3 && g.weno_scheme == 3)
        return g.flux_splitting == 1 ? stage_kg<R, 3, 3, 3>(g, d, a, fl_prev, fl_new, s, nl)
                                     : stage_kg<R, 3, 3, 2>(g, d, a, fl_prev, fl_new, s, nl);
    }
    return cudaErrorInvalidValue;
  }
  if (g.flux_splitting == 1) {
    // the Rusanov splitting is instantiated for the sixth-order central / WENO5 scheme
    if (g.lmax_base == 3 && g.weno_scheme == 3) return stage_kg<R, 3, 3, 1>(g, d, a, fl_prev, fl_new, s, nl);
    return cudaErrorInvalidValue;
  }
  if (g.lmax_base == 3 && g.weno_scheme == 3) return stage_kg<R, 3, 3, 0>(g, d, a, fl_prev, fl_new, s, nl);
  if (g.lmax_base == 2 && g.weno_scheme == 2) return stage_kg<R, 2, 2, 0>(g, d, a, fl_prev, fl_new, s, nl);
  if (g.lmax_base == 4 && g.weno_scheme == 4) return stage_kg<R, 4, 4, 0>(g, d, a, fl_prev, fl_new, s, nl);
  if (g.lmax_base == 3 && g.weno_scheme == 2) return stage_kg<R, 3, 2, 0>(g, d, a, fl_prev, fl_new, s, nl);
  return cudaErrorInvalidValue;
}

cudaError_t launch_stage(const Geom& g, DevState& d, const StageArgs& a, double* fl_prev, double* fl_new,
                         cudaStream_t s, long long* nl) {
  if (g.precision == 1) return stage_dispatch<float>(g, d, a, fl_prev, fl_new, s, nl);
  return stage_dispatch<double>(g, d, a, fl_prev, fl_new, s, nl);
}

bool stage_supported(int lmax_base, int weno_scheme) {
  return (lmax_base == 3 && weno_scheme == 3) || (lmax_base == 2 && weno_scheme == 2) ||
         (lmax_base == 4 && weno_scheme == 4) || (lmax_base == 3 && weno_scheme == 2);
}

// binaryVersion of this file's kernels as the driver loaded them (architecture check)
int binary_version_stage() {
  cudaFuncAttributes a;
  return cudaFuncGetAttributes(&a, k_add_time) == cudaSuccess ? a.binaryVersion : -1;
}

}  // namespace sb200
