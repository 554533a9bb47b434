// Launches over a box table: the stage kernels of many boxes of uneven sizes and flow
// parameters, one launch per kernel kind for all boxes of a group.
//
// A group is a set of boxes whose stages take the same kernels (the same instantiation of the
// stage templates: precision, central and WENO orders, flux form, channel forcing, viscous form;
// no stored ghosts, recycling inflow, non-reflecting faces or WENO faces computed apart).  The
// table holds per box its geometry, its device buffers and the launch shapes that the box would
// use alone (x-pass grid, march segments).  A launch of kind K has one block per block of every
// box's own grid for K, listed box after box in the block table as (box, block of the box's
// grid); each block copies its box's geometry into shared memory and runs the kernel body
// (stage_device.cuh) on it with that block index.  A box therefore computes exactly what it
// computes alone, in the same block partition, and its reductions sum the same block partials
// in the same order: the results are bit-identical to the box advanced alone.  The per-box
// reductions (force_rhs, force_var, residual, time step) keep one block per box.
#include <cstring>

#include "stage_device.cuh"

namespace sb200 {

namespace {

static_assert(sizeof(Geom) % 8 == 0, "Geom is copied to shared memory in 8-byte words");

// Where a CTA reads its box's record: 2 copies the whole record (geometry and buffer pointers)
// into shared memory, 1 the geometry only, 0 reads both from the table in global memory (48-box
// channel mix, FP64 / mixed Mcell-steps/s: 608.0 / 762.3, 600.6 / 756.0, 588.6 / 754.6).
#ifndef SB_BOX_SMEM
#define SB_BOX_SMEM 2
#endif

__device__ __forceinline__ void copy_words(const void* src_p, void* dst_p, int nwords) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y, nt = blockDim.x * blockDim.y;
  const unsigned long long* src = static_cast<const unsigned long long*>(src_p);
  unsigned long long* dst = static_cast<unsigned long long*>(dst_p);
  for (int q = tid; q < nwords; q += nt) dst[q] = src[q];
}
static_assert(sizeof(BoxRec) % 8 == 0, "BoxRec is copied in 8-byte words");

// Tiles of one launch: CTA c works through the tiles [c SPAN, (c + 1) SPAN) of the block table
// (consecutive tiles, mostly of one box, so that a CTA enters a box once for SPAN tiles); each
// tile runs body(record, geometry, block index in the box's grid).
template <unsigned SPAN, class F>
__device__ __forceinline__ void for_tiles(const BoxRec* __restrict__ rec, const BlockRef* __restrict__ blocks,
                                          unsigned ntile, F&& body) {
#if SB_BOX_SMEM == 2
  __shared__ BoxRec rs;
  auto enter = [&](unsigned box) { copy_words(rec + box, &rs, (int)(sizeof(BoxRec) / 8)); };
  auto run = [&](unsigned, unsigned l) { body(static_cast<const BoxRec*>(&rs), static_cast<const Geom&>(rs.g), l); };
#elif SB_BOX_SMEM == 1
  __shared__ Geom gs;
  auto enter = [&](unsigned box) { copy_words(&rec[box].g, &gs, (int)(sizeof(Geom) / 8)); };
  auto run = [&](unsigned box, unsigned l) { body(rec + box, static_cast<const Geom&>(gs), l); };
#else
  auto enter = [&](unsigned) {};
  auto run = [&](unsigned box, unsigned l) { body(rec + box, rec[box].g, l); };
#endif
  if constexpr (SPAN == 1) {
    const BlockRef b = blocks[blockIdx.x];
    enter(b.box);
    if (SB_BOX_SMEM) __syncthreads();
    run(b.box, b.local);
  } else {
    const unsigned t0 = blockIdx.x * SPAN, t1 = min(ntile, t0 + SPAN);
    unsigned cur = 0xffffffffu;
    for (unsigned t = t0; t < t1; ++t) {
      const BlockRef b = blocks[t];
      if (SB_BOX_SMEM && b.box != cur) {  // uniform over the CTA
        __syncthreads();                   // the previous box's tiles are done with the copy
        enter(b.box);
        __syncthreads();
        cur = b.box;
      }
      run(b.box, b.local);
      // the bodies end with block reductions through shared memory: the next tile may not write
      // those buffers before every thread has read this tile's result
      if (t + 1 < t1) __syncthreads();
    }
  }
}
// one block per box (the per-box reductions)
__device__ __forceinline__ const BoxRec* enter_box_direct(const BoxRec* __restrict__ rec, Geom& gs) {
  const BoxRec* r = rec + blockIdx.x;
  copy_words(&r->g, &gs, (int)(sizeof(Geom) / 8));
  __syncthreads();
  return r;
}
// RK register written by stage istep and the one it reads (do_rk_sync's fixed roles)
__device__ __forceinline__ double* fl_new_of(const BoxRec* r, int istep) { return istep == 2 ? r->fl_b : r->fl_a; }
__device__ __forceinline__ double* fl_prev_of(const BoxRec* r, int istep) { return istep == 2 ? r->fl_a : r->fl_b; }

template <unsigned SPAN, class A, bool TP>
__global__ void __launch_bounds__(AUX_NT) kb_apply_shift(const BoxRec* __restrict__ rec,
    const BlockRef* __restrict__ blocks, unsigned ntile) {
  for_tiles<SPAN>(rec, blocks, ntile, [&](const BoxRec* r, const Geom& g, unsigned l) {
    d_apply_shift<A, TP>(g, r->w, static_cast<const A*>(r->aux), r->sc, Blk{l, 0, 0});
  });
}

template <unsigned SPAN, class A, bool TP>
__global__ void __launch_bounds__(AUX_NT, AUX_MINB) kb_aux(const BoxRec* __restrict__ rec,
    const BlockRef* __restrict__ blocks, unsigned ntile, int want_vel) {
  for_tiles<SPAN>(rec, blocks, ntile, [&](const BoxRec* r, const Geom& g, unsigned l) {
    d_aux<A, TP>(g, r->w, static_cast<A*>(r->aux), 0, want_vel ? r->vel64 : nullptr, Blk{l, 0, 0});
  });
}

template <unsigned SPAN, class R, int LB, int WS, int FS>
__global__ void __launch_bounds__(XF_NT, sizeof(R) == 8 ? XF_MINB_D : XF_MINB_F)
    kb_xflux(const BoxRec* __restrict__ rec, const BlockRef* __restrict__ blocks, unsigned ntile, int istep) {
  for_tiles<SPAN>(rec, blocks, ntile, [&](const BoxRec* r, const Geom& g, unsigned l) {
    d_xflux<R, LB, WS, FS>(g, static_cast<const R*>(r->aux), r->sensor, fl_new_of(r, istep), Blk{l, 0, 0});
  });
}

template <unsigned SPAN, class R, bool TP>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? VISC_MINB : VISC_MINB_F)
    kb_visc(const BoxRec* __restrict__ rec, const BlockRef* __restrict__ blocks, unsigned ntile,
    int istep, int do_sensor) {
  for_tiles<SPAN>(rec, blocks, ntile, [&](const BoxRec* r, const Geom& g, unsigned l) {
    d_visc<R, TP>(g, static_cast<const R*>(r->aux), fl_new_of(r, istep), static_cast<R*>(r->div3), r->sensor_next,
                  r->wallprop, do_sensor, Blk{l, 0, 0});
  });
}

template <unsigned SPAN, class R, bool TP>
__global__ void __launch_bounds__(VT_NT, sizeof(R) == 8 ? VISC_MINB : VISC_MINB_F)
    kb_visc_tiled(const BoxRec* __restrict__ rec, const BlockRef* __restrict__ blocks, unsigned ntile,
    int istep, int do_sensor) {
  for_tiles<SPAN>(rec, blocks, ntile, [&](const BoxRec* r, const Geom& g, unsigned l) {
    d_visc_tiled<R, TP>(g, static_cast<const R*>(r->aux), fl_new_of(r, istep), static_cast<R*>(r->div3),
                        r->sensor_next, r->wallprop, do_sensor, Blk{l, 0, 0});
  });
}

template <unsigned SPAN, class R, bool TP>
__global__ void __launch_bounds__(256) kb_visc_ns(const BoxRec* __restrict__ rec,
    const BlockRef* __restrict__ blocks, unsigned ntile, int istep, int do_sensor) {
  for_tiles<SPAN>(rec, blocks, ntile, [&](const BoxRec* r, const Geom& g, unsigned l) {
    d_visc_ns<R, TP>(g, static_cast<const R*>(r->aux), fl_new_of(r, istep), static_cast<R*>(r->div3), r->sensor_next,
                     r->wallprop, do_sensor, Blk{l, 0, 0});
  });
}

// the mixed form's stage-3 sensor in FP64: from the aux pass's velocities or from w
template <unsigned SPAN>
__global__ void __launch_bounds__(256) kb_sensor(const BoxRec* __restrict__ rec,
    const BlockRef* __restrict__ blocks, unsigned ntile, int from_vel) {
  for_tiles<SPAN>(rec, blocks, ntile, [&](const BoxRec* r, const Geom& g, unsigned l) {
    const int mode = g.conservative_viscous ? 1 : 2;
    if (from_vel)
      d_sensor_vel(g, r->vel64, r->sensor_next, mode, Blk{l, 0, 0});
    else
      d_sensor64(g, r->w, r->sensor_next, mode, Blk{l, 0, 0});
  });
}

template <unsigned SPAN, class R, int DIR, int LB, int WS, bool CH, int FS>
__global__ void __launch_bounds__(MT_NT, sizeof(R) == 8 ? MT_MINB_D : (CH ? MT_MINB_F_CH : MT_MINB_F))
    kb_march(const BoxRec* __restrict__ rec, const BlockRef* __restrict__ blocks, unsigned ntile, double rhork, double gamrk, int istep) {
  for_tiles<SPAN>(rec, blocks, ntile, [&](const BoxRec* r, const Geom& g, unsigned l) {
    const int seglen = DIR == 1 ? r->sly : r->slz, nseg = DIR == 1 ? r->nsy : r->nsz;
    d_march<R, DIR, LB, WS, CH, FS, false>(g, static_cast<const R*>(r->aux), r->sensor, fl_new_of(r, istep),
                                           static_cast<const R*>(r->div3), r->w, fl_prev_of(r, istep), r->sc, rhork,
                                           gamrk, istep, seglen, nseg, r->red, Blk{l, 0, 0});
  });
}

__global__ void __launch_bounds__(FIN_NT) kb_finish_rhs(const BoxRec* __restrict__ rec, int first_stage) {
  __shared__ Geom gs;
  const BoxRec* r = enter_box_direct(rec, gs);
  d_finish_rhs(gs, r->red, r->nb_z, first_stage, r->sc, Blk{0, 0, 0});
}

template <unsigned SPAN, class R, bool TP>
__global__ void __launch_bounds__(UPD_NT, UPD_MINB) kb_update(const BoxRec* __restrict__ rec,
    const BlockRef* __restrict__ blocks, unsigned ntile, double rhork, double gamrk, int istep,
    int stats) {
  for_tiles<SPAN>(rec, blocks, ntile, [&](const BoxRec* r, const Geom& g, unsigned l) {
    d_update<R, TP>(g, r->w, fl_prev_of(r, istep), fl_new_of(r, istep), r->sc, rhork, gamrk, istep, stats, r->red,
                    r->sensor_next, r->sensor, static_cast<R*>(r->aux), Blk{l, 0, 0});
  });
}

__global__ void __launch_bounds__(FIN_NT) kb_finish_upd(const BoxRec* __restrict__ rec, int stats, int add_time) {
  __shared__ Geom gs;
  const BoxRec* r = enter_box_direct(rec, gs);
  d_finish_upd(gs, r->red, r->nb_up, stats, add_time, r->sc, Blk{0, 0, 0});
}

template <unsigned SPAN, class R>
__global__ void __launch_bounds__(256, DT_MINB) kb_dt(const BoxRec* __restrict__ rec,
    const BlockRef* __restrict__ blocks, unsigned ntile) {
  for_tiles<SPAN>(rec, blocks, ntile, [&](const BoxRec* r, const Geom& g, unsigned l) {
    d_dt<R>(g, r->w, static_cast<const R*>(r->aux), r->red, Blk{l, 0, 0});
  });
}

__global__ void __launch_bounds__(FIN_NT) kb_dt_finish(const BoxRec* __restrict__ rec) {
  const BoxRec* r = rec + blockIdx.x;
  d_dt_finish(r->red, r->nb_up, r->cfl, r->sc, Blk{0, 0, 0});
}

// Tiles per CTA: the short tiles of the aux, shift and sensor passes are taken four at a time so
// that a CTA enters a box (table entry, record copy) once for several; the update and time-step
// passes (1024 cells a tile), the viscous and the flux passes take one.
constexpr unsigned SPAN_PT = 4;
struct Launch {
  unsigned ntile;
  const BlockRef* blocks;
  unsigned grid(unsigned span) const { return (ntile + span - 1) / span; }
};
inline Launch launch_of(const BoxTable& t, int kind) { return Launch{t.cnt[kind], t.blocks + t.off[kind]}; }

template <class R, bool TP>
void batch_aux_tp(const BoxTable& t, int apply_shift, int want_vel, cudaStream_t s, long long* nl) {
  if (apply_shift) {
    const Launch L = launch_of(t, BK_PT);
    kb_apply_shift<SPAN_PT, R, TP><<<L.grid(SPAN_PT), AUX_NT, 0, s>>>(t.rec, L.blocks, L.ntile);
    ++*nl;
  }
  const Launch L = launch_of(t, BK_VOL);
  kb_aux<SPAN_PT, R, TP><<<L.grid(SPAN_PT), AUX_NT, 0, s>>>(t.rec, L.blocks, L.ntile, want_vel);
  ++*nl;
}

template <class R>
void batch_aux(const BoxTable& t, int apply_shift, int want_vel, cudaStream_t s, long long* nl) {
  if constexpr (sizeof(R) == sizeof(double)) {
    if (!t.g0.calorically_perfect) {
      batch_aux_tp<R, true>(t, apply_shift, want_vel, s, nl);
      return;
    }
  }
  batch_aux_tp<R, false>(t, apply_shift, want_vel, s, nl);
}

template <class R, int LB, int WS, int FS>
cudaError_t batch_stage_impl(const BoxTable& t, const StageArgs& a, cudaStream_t s, long long* nl) {
  const Geom& g = t.g0;
  constexpr bool fp64 = sizeof(R) == sizeof(double);
  constexpr bool TP = (FS & 2) != 0;
  const int nbox = t.nbox;
  if (a.run_aux) batch_aux<R>(t, a.apply_shift, !fp64 && a.istep == 3, s, nl);
  const size_t xsm = weno_scratch_bytes<R, WS>(XF_NT);
  const size_t msm = weno_scratch_bytes<R, WS>(MT_NT);
  static unsigned long long smem_set = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(smem_set & (1ULL << dev))) {
    cudaFuncSetAttribute(kb_xflux<1, R, LB, WS, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xsm);
    cudaFuncSetAttribute(kb_march<1, R, 1, LB, WS, false, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msm);
    cudaFuncSetAttribute(kb_march<1, R, 2, LB, WS, false, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msm);
    cudaFuncSetAttribute(kb_march<1, R, 2, LB, WS, true, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msm);
    smem_set |= 1ULL << dev;
  }
  const Launch X = launch_of(t, BK_X), P = launch_of(t, BK_PT), Y = launch_of(t, BK_Y), Z = launch_of(t, BK_Z);
  kb_xflux<1, R, LB, WS, FS><<<X.grid(1), dim3(XF_TX, XF_TY), xsm, s>>>(t.rec, X.blocks, X.ntile, a.istep);
  const int do_sensor = fp64 && a.istep == 3;
  if (g.conservative_viscous && SB_VISC_TILED) {
    const Launch V = launch_of(t, BK_VS);
    kb_visc_tiled<1, R, TP><<<V.grid(1), VT_NT, 0, s>>>(t.rec, V.blocks, V.ntile, a.istep, do_sensor);
  } else if (g.conservative_viscous)
    kb_visc<1, R, TP><<<P.grid(1), 256, 0, s>>>(t.rec, P.blocks, P.ntile, a.istep, do_sensor);
  else
    kb_visc_ns<1, R, TP><<<P.grid(1), 256, 0, s>>>(t.rec, P.blocks, P.ntile, a.istep, do_sensor);
  *nl += 2;
  if (!fp64 && a.istep == 3) {
    kb_sensor<SPAN_PT><<<P.grid(SPAN_PT), 256, 0, s>>>(t.rec, P.blocks, P.ntile, a.run_aux);
    ++*nl;
  }
  if (Y.ntile > 0) {
    kb_march<1, R, 1, LB, WS, false, FS><<<Y.grid(1), MT_NT, msm, s>>>(t.rec, Y.blocks, Y.ntile, a.rhork, a.gamrk,
                                                                       a.istep);
    ++*nl;
  }
  if (g.channel_case) {
    kb_march<1, R, 2, LB, WS, true, FS><<<Z.grid(1), MT_NT, msm, s>>>(t.rec, Z.blocks, Z.ntile, a.rhork, a.gamrk,
                                                                      a.istep);
    kb_finish_rhs<<<nbox, FIN_NT, 0, s>>>(t.rec, a.istep == 1);
    *nl += 2;
  } else {
    kb_march<1, R, 2, LB, WS, false, FS><<<Z.grid(1), MT_NT, msm, s>>>(t.rec, Z.blocks, Z.ntile, a.rhork, a.gamrk,
                                                                       a.istep);
    ++*nl;
  }
  const Launch U = launch_of(t, BK_UP);
  kb_update<1, R, TP><<<U.grid(1), UPD_NT, 0, s>>>(t.rec, U.blocks, U.ntile, a.rhork, a.gamrk, a.istep,
                                                     a.want_stats);
  kb_finish_upd<<<nbox, FIN_NT, 0, s>>>(t.rec, a.want_stats, a.add_time);
  *nl += 2;
  return cudaGetLastError();
}

// the instantiations of stage_dispatch / stage_kg (stage_kernels.cu)
template <class R, int LB, int WS, int FS>
cudaError_t batch_stage_kg(const BoxTable& t, const StageArgs& a, cudaStream_t s, long long* nl) {
  const Geom& g = t.g0;
  if constexpr (WS == 3) {
    if (g.weno_version == 1) {
      if (g.nkeep != 0) return batch_stage_impl<R, LB, WS, FS | 4 | 8>(t, a, s, nl);
      return batch_stage_impl<R, LB, WS, FS | 8>(t, a, s, nl);
    }
  }
  if (g.nkeep != 0) return batch_stage_impl<R, LB, WS, FS | 4>(t, a, s, nl);
  return batch_stage_impl<R, LB, WS, FS>(t, a, s, nl);
}

template <class R>
cudaError_t batch_stage_dispatch(const BoxTable& t, const StageArgs& a, cudaStream_t s, long long* nl) {
  const Geom& g = t.g0;
  if (!g.calorically_perfect) {
    if constexpr (sizeof(R) == sizeof(double)) {
      if (g.lmax_base == 3 && g.weno_scheme == 3)
        return g.flux_splitting == 1 ? batch_stage_kg<R, 3, 3, 3>(t, a, s, nl) : batch_stage_kg<R, 3, 3, 2>(t, a, s, nl);
    }
    return cudaErrorInvalidValue;
  }
  if (g.flux_splitting == 1) {
    if (g.lmax_base == 3 && g.weno_scheme == 3) return batch_stage_kg<R, 3, 3, 1>(t, a, s, nl);
    return cudaErrorInvalidValue;
  }
  if (g.lmax_base == 3 && g.weno_scheme == 3) return batch_stage_kg<R, 3, 3, 0>(t, a, s, nl);
  if (g.lmax_base == 2 && g.weno_scheme == 2) return batch_stage_kg<R, 2, 2, 0>(t, a, s, nl);
  if (g.lmax_base == 4 && g.weno_scheme == 4) return batch_stage_kg<R, 4, 4, 0>(t, a, s, nl);
  if (g.lmax_base == 3 && g.weno_scheme == 2) return batch_stage_kg<R, 3, 2, 0>(t, a, s, nl);
  return cudaErrorInvalidValue;
}

}  // namespace

long long batch_key(const Geom& g) {
  if (has_stored_ghosts(g) || g.recyc || (SB_WENO_SPLIT && g.wsplit_on)) return -1;
  for (int l = 0; l < 6; ++l)
    if (g.nr[l] > 0) return -1;
  if (!stage_supported(g.lmax_base, g.weno_scheme)) return -1;
  long long k = 0;
  auto put = [&](long long v, int bits) { k = (k << bits) | (v & ((1LL << bits) - 1)); };
  put(g.precision, 2);
  put(g.lmax_base, 4);
  put(g.weno_scheme, 4);
  put(g.flux_splitting, 2);
  put(g.nkeep != 0, 1);
  put(g.weno_version, 2);
  put(g.calorically_perfect, 1);
  put(g.channel_case, 1);
  put(g.conservative_viscous, 1);
  put(g.force_var, 1);
  return k;
}

BoxRec box_rec(const Geom& g, const DevState& d, double* fl_a, double* fl_b, double cfl) {
  BoxRec r;
  std::memset(&r, 0, sizeof(r));
  r.g = g;
  r.w = d.w;
  r.aux = g.precision == 1 ? static_cast<void*>(d.auxf) : static_cast<void*>(d.aux);
  r.div3 = g.precision == 1 ? static_cast<void*>(d.div3f) : static_cast<void*>(d.div3);
  r.sensor = d.sensor;
  r.sensor_next = d.sensor_next;
  r.vel64 = d.vel64;
  r.fl_a = fl_a;
  r.fl_b = fl_b;
  r.wallprop = d.wallprop;
  r.red = d.red;
  r.sc = d.sc;
  r.cfl = cfl;
  long long nty, ntz;
  march_split(g, 1, &r.sly, &r.nsy, &nty);
  march_split(g, 2, &r.slz, &r.nsz, &ntz);
  r.xg[0] = x_blocks(g);
  r.xg[1] = 1;
  r.xg[2] = 1;
  r.nb_y = nblocks(nty, MT_NT);
  r.nb_z = nblocks(ntz, MT_NT);
  r.nb_pt = nblocks(g.nint, 256);
  r.nb_vol = nblocks(g.nvol, AUX_NT);
  r.nb_vs = visc_tiled_blocks(g);
  r.nb_up = pt_blocks(g.nint);
  return r;
}

// Tables live in the device's stream-ordered pool, freed once the stream's work is done.
void box_table_free(BoxTable& t, cudaStream_t s) {
  if (t.rec || t.blocks) cudaStreamSynchronize(s);
  if (t.rec) cudaFreeAsync(t.rec, s);
  if (t.blocks) cudaFreeAsync(t.blocks, s);
  t.rec = nullptr;
  t.blocks = nullptr;
  t.nbox = 0;
}

cudaError_t box_table_build(BoxTable& t, const std::vector<BoxRec>& recs, cudaStream_t s) {
  box_table_free(t, s);
  if (recs.empty()) return cudaErrorInvalidValue;
  std::vector<BlockRef> blocks;
  for (int k = 0; k < BK_NUM; ++k) {
    t.off[k] = (long long)blocks.size();
    for (size_t b = 0; b < recs.size(); ++b) {
      const BoxRec& r = recs[b];
      const unsigned long long n = k == BK_VOL ? r.nb_vol
                                   : k == BK_PT ? r.nb_pt
                                   : k == BK_X  ? (unsigned long long)r.xg[0] * r.xg[1] * r.xg[2]
                                   : k == BK_Y  ? r.nb_y
                                   : k == BK_Z  ? r.nb_z
                                   : k == BK_VS ? r.nb_vs
                                                : r.nb_up;
      for (unsigned long long q = 0; q < n; ++q) blocks.push_back(BlockRef{(unsigned)b, (unsigned)q});
    }
    const long long c = (long long)blocks.size() - t.off[k];
    if (c > 0x7fffffffLL) return cudaErrorInvalidValue;  // one launch's grid
    t.cnt[k] = (unsigned)c;
  }
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&t.rec), recs.size() * sizeof(BoxRec), s);
  if (e == cudaSuccess)
    e = cudaMallocAsync(reinterpret_cast<void**>(&t.blocks), std::max<size_t>(blocks.size(), 1) * sizeof(BlockRef), s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(t.rec, recs.data(), recs.size() * sizeof(BoxRec), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !blocks.empty())
    e = cudaMemcpyAsync(t.blocks, blocks.data(), blocks.size() * sizeof(BlockRef), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host vectors go out of scope
  if (e != cudaSuccess) {
    box_table_free(t, s);
    return e;
  }
  t.nbox = (int)recs.size();
  t.g0 = recs[0].g;
  return cudaSuccess;
}

cudaError_t batch_launch_aux(const BoxTable& t, int apply_shift, cudaStream_t s, long long* nl) {
  if (t.g0.precision == 1) batch_aux<float>(t, apply_shift, 0, s, nl);
  else batch_aux<double>(t, apply_shift, 0, s, nl);
  return cudaGetLastError();
}

cudaError_t batch_launch_dt(const BoxTable& t, cudaStream_t s, long long* nl) {
  const Launch U = launch_of(t, BK_UP);
  if (t.g0.precision == 1)
    kb_dt<1, float><<<U.grid(1), 256, 0, s>>>(t.rec, U.blocks, U.ntile);
  else
    kb_dt<1, double><<<U.grid(1), 256, 0, s>>>(t.rec, U.blocks, U.ntile);
  kb_dt_finish<<<t.nbox, FIN_NT, 0, s>>>(t.rec);
  *nl += 2;
  return cudaGetLastError();
}

cudaError_t batch_launch_stage(const BoxTable& t, const StageArgs& a, cudaStream_t s, long long* nl) {
  if (t.g0.precision == 1) return batch_stage_dispatch<float>(t, a, s, nl);
  return batch_stage_dispatch<double>(t, a, s, nl);
}

}  // namespace sb200
