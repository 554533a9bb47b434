// Device functions of the hybrid convective flux at one cell face: energy-preserving split-form
// central flux (KEEP variants) and characteristic WENO where the Ducros sensor fires.
// Restates euler_{x,y,z}_*hybrid_kernel, compute_roe_average, eigenvectors_{x,y,z} and
// wenorec_1d of code/src/singleideal/kernels_cpu.F90 (lines cited per function).
#pragma once

#include "common.cuh"

// keep the sound speed of every stencil point in the window (1) or recompute it in the WENO
// branch (0, default: fewer registers and spills in the march kernels, measured 2-7 % faster)
#ifndef SB_CACHE_C
#define SB_CACHE_C 0
#endif

// characteristic fields reconstructed per iteration of the WENO branch's field loop (1: one copy
// of wenorec, the loop rolled; the unrolled loop overflowed the instruction cache)
#ifndef SB_WENO_UNROLL
#define SB_WENO_UNROLL 1
#endif
#define SB_PRAGMA_(x) _Pragma(#x)
#define SB_UNROLL_(n) SB_PRAGMA_(unroll n)

// quotients and square roots of the mixed form's FP32 flux arithmetic: IEEE (0), the hardware
// approximations (1), or the hardware approximations refined by one Newton step (2)
#ifndef SB_FP32_FAST
#define SB_FP32_FAST 2
#endif

namespace sb200 {

// Quotient and square root (of a positive value) in the flux arithmetic: IEEE in FP64, where the
// reference's operations are kept; with SB_FP32_FAST the FP32 form takes the hardware reciprocal
// and reciprocal square root (at most 2 ulp: the mixed form's error is set by FP32 rounding).
// With SB_FP32_FAST = 2 the approximate reciprocal r of b is refined by one Newton-Raphson step
// (e = 1 - b r, r += r e) and the quotient q = a r corrected by its remainder (Markstein:
// q += r (a - b q)); the approximate reciprocal square root y of x gives s = x y, corrected by one
// Newton step for the square root (s += (x - s s) y / 2).  Without the refinement the errors of
// the raw approximations do not average out over many steps (the transverse momenta of a
// WENO-only channel drifted twice as far from the FP64 oracle in 100 steps).
template <class R>
__device__ __forceinline__ R fdiv(R a, R b) {
  if constexpr (sizeof(R) == sizeof(double) || !SB_FP32_FAST) {
    return a / b;
  } else if constexpr (SB_FP32_FAST == 1) {
    return __fdividef(a, b);
  } else {
    float r = __fdividef(1.0f, b);
    const float e = __fmaf_rn(-b, r, 1.0f);
    r = __fmaf_rn(r, e, r);
    const float q = a * r;
    return __fmaf_rn(r, __fmaf_rn(-b, q, a), q);
  }
}
template <class R>
__device__ __forceinline__ R fsqrt_pos(R x) {
  if constexpr (sizeof(R) == sizeof(double) || !SB_FP32_FAST) {
    return sqrt(x);
  } else if constexpr (SB_FP32_FAST == 1) {
    return x * rsqrtf(x);
  } else {
    const float y = rsqrtf(x);
    const float sx = x * y;
    return __fmaf_rn(__fmaf_rn(-sx, sx, x), 0.5f * y, sx);
  }
}

// Error-free transformations for the mixed form: the face fluxes are accumulated as float-float
// pairs (hi + lo) so that the flux differences of neighbouring faces can be formed in FP64
// without the cancellation of the FP32 rounding of their final sums.  Explicit rounding
// intrinsics keep the compiler from contracting them.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}
// acc (hi, lo) += a * b
__device__ __forceinline__ void acc_prod(float& hi, float& lo, float a, float b) {
  const float p = __fmul_rn(a, b);
  const float ep = __fmaf_rn(a, b, -p);
  float s, es;
  two_sum(hi, p, s, es);
  hi = s;
  lo = lo + (es + ep);
}
__device__ __forceinline__ void acc_prod(double& hi, double& lo, double a, double b) {
  hi = hi + a * b;
  (void)lo;
}
__device__ __forceinline__ void acc_add(float& hi, float& lo, float b) {
  float s, es;
  two_sum(hi, b, s, es);
  hi = s;
  lo = lo + es;
}
__device__ __forceinline__ void acc_add(double& hi, double& lo, double b) {
  hi = hi + b;
  (void)lo;
}

// 1/a and 1/b from one division in FP64, 1/(a b) times the other factor: the weight sums of
// the two sides of a WENO reconstruction are positive and stay far inside the FP64 exponent
// range (products of (eps + beta)^2 terms, eps = 1e-6, or WENO-Z ratios), so the product neither
// overflows nor underflows.  FP32 keeps two divisions (its range is too narrow for the product).
template <class R>
__device__ __forceinline__ void recip_pair(R a, R b, R& ra, R& rb) {
  if constexpr (sizeof(R) == sizeof(double)) {
    const R r = R(1) / (a * b);
    ra = b * r;
    rb = a * r;
  } else {
    ra = fdiv(R(1), a);
    rb = fdiv(R(1), b);
  }
}

// Stencil of a face: NP = 2*S points at offsets o = -(S-1) .. S from the face's lower point.
template <class R, int S>
struct Stencil {
  R rho[2 * S], u[2 * S], v[2 * S], w[2 * S], h[2 * S], t[2 * S];
#if SB_CACHE_C
  R c[2 * S];  // sound speed sqrt(gamma R T) of each point, computed once when the point is loaded
#endif
};

// wenorec_1d (kernels_cpu.F90:2526-2724) for one characteristic variable.  The nonlinear weights
// are normalised by one reciprocal of their sum (the reference divides each weight by the sum;
// the results differ in the last bit only).
// vp[l-1], vm[l-1] hold the reference's vp(m,l), vm(m,l), l = 1..2*WS; i = iweno = WS.
template <class R, int WS>
__device__ __forceinline__ R wenorec(const R (&vp)[2 * WS], const R (&vm)[2 * WS], int ord, int version,
                                     R betascale) {
  auto VP = [&](int l) -> R { return vp[l - 1]; };
  auto VM = [&](int l) -> R { return vm[l - 1]; };
  constexpr int i = WS;
  const R eps6 = R(0.000001);
  if (ord == 1) {
    return VP(i) + VM(i + 1);
  }
  if constexpr (WS >= 2) {
    if (ord == 2) {
      const R dwe0 = R(1.0) / R(3.0), dwe1 = R(2.0) / R(3.0);
      R a = VP(i) - VP(i - 1), b = VP(i + 1) - VP(i);
      R bp0 = betascale * (a * a), bp1 = betascale * (b * b);
      R c = VM(i + 2) - VM(i + 1), d = VM(i + 1) - VM(i);
      R bm0 = betascale * (c * c), bm1 = betascale * (d * d);
      R tp0 = eps6 + bp0, tp1 = eps6 + bp1, tm0 = eps6 + bm0, tm1 = eps6 + bm1;
      bp0 = dwe0 / (tp0 * tp0);
      bm0 = dwe0 / (tm0 * tm0);
      bp1 = dwe1 / (tp1 * tp1);
      bm1 = dwe1 / (tm1 * tm1);
      R rsp, rsm;
      recip_pair((R(0) + bp0) + bp1, (R(0) + bm0) + bm1, rsp, rsm);
      bp0 = bp0 * rsp; bp1 = bp1 * rsp; bm0 = bm0 * rsm; bm1 = bm1 * rsm;
      R vminus = bp0 * (-VP(i - 1) + R(3) * VP(i)) + bp1 * (VP(i) + VP(i + 1));
      R vplus = bm0 * (-VM(i + 2) + R(3) * VM(i + 1)) + bm1 * (VM(i) + VM(i + 1));
      return R(0.5) * (vminus + vplus);
    }
  }
  if constexpr (WS >= 3) {
    if (ord == 3) {
      const R dwe[3] = {R(1.0) / R(10.0), R(6.0) / R(10.0), R(3.0) / R(10.0)};
      const R d0 = R(13.0) / R(12.0), d1 = R(1.0) / R(4.0);
      const R c0 = R(1.0) / R(3.0), c1 = R(5.0) / R(6.0), c2 = R(-1.0) / R(6.0), c3 = R(-7.0) / R(6.0),
              c4 = R(11.0) / R(6.0);
      R bp[3], bm[3];
      {
        R a = VP(i) - R(2) * VP(i + 1) + VP(i + 2), b = R(3) * VP(i) - R(4) * VP(i + 1) + VP(i + 2);
        bp[2] = d0 * (a * a) + d1 * (b * b);
        a = VP(i - 1) - R(2) * VP(i) + VP(i + 1);
        b = VP(i - 1) - VP(i + 1);
        bp[1] = d0 * (a * a) + d1 * (b * b);
        a = VP(i) - R(2) * VP(i - 1) + VP(i - 2);
        b = R(3) * VP(i) - R(4) * VP(i - 1) + VP(i - 2);
        bp[0] = d0 * (a * a) + d1 * (b * b);
        a = VM(i + 1) - R(2) * VM(i) + VM(i - 1);
        b = R(3) * VM(i + 1) - R(4) * VM(i) + VM(i - 1);
        bm[2] = d0 * (a * a) + d1 * (b * b);
        a = VM(i + 2) - R(2) * VM(i + 1) + VM(i);
        b = VM(i + 2) - VM(i);
        bm[1] = d0 * (a * a) + d1 * (b * b);
        a = VM(i + 1) - R(2) * VM(i + 2) + VM(i + 3);
        b = R(3) * VM(i + 1) - R(4) * VM(i + 2) + VM(i + 3);
        bm[0] = d0 * (a * a) + d1 * (b * b);
      }
#pragma unroll
      for (int l = 2; l >= 0; --l) {
        bp[l] = betascale * bp[l];
        bm[l] = betascale * bm[l];
      }
      if (version == 0) {
        // omega_l = (d_l / t_l) / sum_k (d_k / t_k), t_l = (eps + beta_l)^2, formed with one
        // division per side: omega_l = d_l prod_{m != l} t_m / sum_k d_k prod_{m != k} t_m
        // (the same weights; the products stay far inside the exponent range for eps = 1e-6)
        R tp[3], tm[3];
#pragma unroll
        for (int l = 0; l < 3; ++l) {
          const R a = eps6 + bp[l], b = eps6 + bm[l];
          tp[l] = a * a;
          tm[l] = b * b;
        }
        const R np0 = dwe[0] * (tp[1] * tp[2]), np1 = dwe[1] * (tp[0] * tp[2]), np2 = dwe[2] * (tp[0] * tp[1]);
        const R nm0 = dwe[0] * (tm[1] * tm[2]), nm1 = dwe[1] * (tm[0] * tm[2]), nm2 = dwe[2] * (tm[0] * tm[1]);
        R rsp, rsm;
        recip_pair((np0 + np1) + np2, (nm0 + nm1) + nm2, rsp, rsm);
        bp[0] = np0 * rsp; bp[1] = np1 * rsp; bp[2] = np2 * rsp;
        bm[0] = nm0 * rsm; bm[1] = nm1 * rsm; bm[2] = nm2 * rsm;
      } else {
        // eps40 is a single-precision literal in the reference
        const R eps40 = R(static_cast<double>(1.e-35f));
        R tau5p = fabs(bp[0] - bp[2]) + eps40;
        R tau5m = fabs(bm[0] - bm[2]) + eps40;
#pragma unroll
        for (int l = 0; l < 3; ++l) {
          bp[l] = (bp[l] + eps40) / (bp[l] + tau5p);
          bm[l] = (bm[l] + eps40) / (bm[l] + tau5m);
        }
        R sump = R(0), summ = R(0);
#pragma unroll
        for (int l = 0; l < 3; ++l) {
          bp[l] = dwe[l] / bp[l];
          bm[l] = dwe[l] / bm[l];
          sump = sump + bp[l];
          summ = summ + bm[l];
        }
        R rsp, rsm;
        recip_pair(sump, summ, rsp, rsm);
#pragma unroll
        for (int l = 0; l < 3; ++l) {
          bp[l] = bp[l] * rsp;
          bm[l] = bm[l] * rsm;
        }
      }
      R vminus = bp[2] * (c0 * VP(i) + c1 * VP(i + 1) + c2 * VP(i + 2)) +
                 bp[1] * (c2 * VP(i - 1) + c1 * VP(i) + c0 * VP(i + 1)) +
                 bp[0] * (c0 * VP(i - 2) + c3 * VP(i - 1) + c4 * VP(i));
      R vplus = bm[2] * (c0 * VM(i + 1) + c1 * VM(i) + c2 * VM(i - 1)) +
                bm[1] * (c2 * VM(i + 2) + c1 * VM(i + 1) + c0 * VM(i)) +
                bm[0] * (c0 * VM(i + 3) + c3 * VM(i + 2) + c4 * VM(i + 1));
      return vminus + vplus;
    }
  }
  if constexpr (WS >= 4) {
    if (ord == 4) {
      const R dwe[4] = {R(1.0) / R(35.0), R(12.0) / R(35.0), R(18.0) / R(35.0), R(4.0) / R(35.0)};
      const R d1 = R(1.0) / R(36.0), d2 = R(13.0) / R(12.0), d3 = R(781.0) / R(720.0);
      auto sq = [](R a) { return a * a; };
      R bp[4], bm[4];
      bp[3] = d1 * sq(-11 * VP(i) + 18 * VP(i + 1) - 9 * VP(i + 2) + 2 * VP(i + 3)) +
              d2 * sq(2 * VP(i) - 5 * VP(i + 1) + 4 * VP(i + 2) - VP(i + 3)) +
              d3 * sq(-VP(i) + 3 * VP(i + 1) - 3 * VP(i + 2) + VP(i + 3));
      bp[2] = d1 * sq(-2 * VP(i - 1) - 3 * VP(i) + 6 * VP(i + 1) - VP(i + 2)) +
              d2 * sq(VP(i - 1) - 2 * VP(i) + VP(i + 1)) + d3 * sq(-VP(i - 1) + 3 * VP(i) - 3 * VP(i + 1) + VP(i + 2));
      bp[1] = d1 * sq(VP(i - 2) - 6 * VP(i - 1) + 3 * VP(i) + 2 * VP(i + 1)) +
              d2 * sq(VP(i - 1) - 2 * VP(i) + VP(i + 1)) + d3 * sq(-VP(i - 2) + 3 * VP(i - 1) - 3 * VP(i) + VP(i + 1));
      bp[0] = d1 * sq(-2 * VP(i - 3) + 9 * VP(i - 2) - 18 * VP(i - 1) + 11 * VP(i)) +
              d2 * sq(-VP(i - 3) + 4 * VP(i - 2) - 5 * VP(i - 1) + 2 * VP(i)) +
              d3 * sq(-VP(i - 3) + 3 * VP(i - 2) - 3 * VP(i - 1) + VP(i));
      bm[3] = d1 * sq(-11 * VM(i + 1) + 18 * VM(i) - 9 * VM(i - 1) + 2 * VM(i - 2)) +
              d2 * sq(2 * VM(i + 1) - 5 * VM(i) + 4 * VM(i - 1) - VM(i - 2)) +
              d3 * sq(-VM(i + 1) + 3 * VM(i) - 3 * VM(i - 1) + VM(i - 2));
      bm[2] = d1 * sq(-2 * VM(i + 2) - 3 * VM(i + 1) + 6 * VM(i) - VM(i - 1)) +
              d2 * sq(VM(i + 2) - 2 * VM(i + 1) + VM(i)) + d3 * sq(-VM(i + 2) + 3 * VM(i + 1) - 3 * VM(i) + VM(i - 1));
      bm[1] = d1 * sq(VM(i + 3) - 6 * VM(i + 2) + 3 * VM(i + 1) + 2 * VM(i)) +
              d2 * sq(VM(i + 2) - 2 * VM(i + 1) + VM(i)) + d3 * sq(-VM(i + 3) + 3 * VM(i + 2) - 3 * VM(i + 1) + VM(i));
      bm[0] = d1 * sq(-2 * VM(i + 4) + 9 * VM(i + 3) - 18 * VM(i + 2) + 11 * VM(i + 1)) +
              d2 * sq(-VM(i + 4) + 4 * VM(i + 3) - 5 * VM(i + 2) + 2 * VM(i + 1)) +
              d3 * sq(-VM(i + 4) + 3 * VM(i + 3) - 3 * VM(i + 2) + VM(i + 1));
      R sump = R(0), summ = R(0);
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        bp[l] = betascale * bp[l];
        bm[l] = betascale * bm[l];
      }
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        R tp = eps6 + bp[l], tm = eps6 + bm[l];
        bp[l] = dwe[l] / (tp * tp);
        bm[l] = dwe[l] / (tm * tm);
        sump = sump + bp[l];
        summ = summ + bm[l];
      }
      R rsp, rsm;
      recip_pair(sump, summ, rsp, rsm);
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        bp[l] = bp[l] * rsp;
        bm[l] = bm[l] * rsm;
      }
      R vminus = bp[3] * (6 * VP(i) + 26 * VP(i + 1) - 10 * VP(i + 2) + 2 * VP(i + 3)) +
                 bp[2] * (-2 * VP(i - 1) + 14 * VP(i) + 14 * VP(i + 1) - 2 * VP(i + 2)) +
                 bp[1] * (2 * VP(i - 2) - 10 * VP(i - 1) + 26 * VP(i) + 6 * VP(i + 1)) +
                 bp[0] * (-6 * VP(i - 3) + 26 * VP(i - 2) - 46 * VP(i - 1) + 50 * VP(i));
      R vplus = bm[3] * (6 * VM(i + 1) + 26 * VM(i) - 10 * VM(i - 1) + 2 * VM(i - 2)) +
                bm[2] * (-2 * VM(i + 2) + 14 * VM(i + 1) + 14 * VM(i) - 2 * VM(i - 1)) +
                bm[1] * (2 * VM(i + 3) - 10 * VM(i + 2) + 26 * VM(i + 1) + 6 * VM(i)) +
                bm[0] * (-6 * VM(i + 4) + 26 * VM(i + 3) - 46 * VM(i + 2) + 50 * VM(i + 1));
      return (vminus + vplus) / R(24);
    }
  }
  return R(0);
}

// Central energy-preserving split-form flux (kernels_cpu.F90:462-612 for x; same in y, z).
// DIR: 0 x, 1 y, 2 z.  Points of st are at offsets -(S-1)..S (index o + S - 1).  KG = false
// instantiates the default nkeep = 0 form at compile time (the general KEEP(n) branch, with its
// divisions, otherwise shapes the register allocation of the whole flux kernel).
template <class R, int DIR, int LB, int S, bool KG = true>
__device__ __forceinline__ void central_flux(const Geom& g, const Stencil<R, S>& st, int lmax, int nkeep_in,
                                             bool zero_flux, R (&fh)[5], R (&fl)[5]) {
  const int nkeep = KG ? nkeep_in : 0;
  const R rgas0 = R(g.rgas0);
  R pp[2 * S], ee[2 * S];
#pragma unroll
  for (int q = 0; q < 2 * S; ++q) {
    pp[q] = st.t[q] * st.rho[q] * rgas0;
    // e = H - p/rho - |u|^2/2 with p/rho = R T taken directly (the reference divides p by rho;
    // the two differ in the last bit only and the division is the costliest operation here)
    ee[q] = st.h[q] - st.t[q] * rgas0 - R(0.5) * (st.u[q] * st.u[q] + st.v[q] * st.v[q] + st.w[q] * st.w[q]);
  }
  R ft1 = 0, ft2 = 0, ft3 = 0, ft4 = 0, ft5 = 0, ft6 = 0;
  R lt1 = 0, lt2 = 0, lt3 = 0, lt4 = 0, lt5 = 0, lt6 = 0;  // compensation (mixed form)
#pragma unroll
  for (int l = 1; l <= LB; ++l) {
    if (l <= lmax) {
      R uvs1 = 0, uvs2 = 0, uvs3 = 0, uvs4 = 0, uvs5 = 0, uvs5_i = 0, uvs5_k = 0, uvs5_p = 0, uvs6 = 0;
#pragma unroll
      for (int m = 0; m < LB; ++m) {
        if (m <= l - 1) {
          const int a = -m + S - 1, b = -m + l + S - 1;
          const R vna = DIR == 0 ? st.u[a] : (DIR == 1 ? st.v[a] : st.w[a]);
          const R vnb = DIR == 0 ? st.u[b] : (DIR == 1 ? st.v[b] : st.w[b]);
          R rhom = st.rho[a] + st.rho[b];
          if (nkeep >= 0) {
            R eem = ee[a] + ee[b];
            R drhof = R(1), deef = R(1);
            if (nkeep != 0) {
              R drho = R(2) * (st.rho[b] - st.rho[a]) / rhom;
              R dee = R(2) * (ee[b] - ee[a]) / eem;
              R t_sumdenrho = (R(0.5) * drho) * (R(0.5) * drho);
              R t_sumdenee = (R(0.5) * dee) * (R(0.5) * dee);
              R t2r = t_sumdenrho, t2e = t_sumdenee;
              R sumdenrho = R(1) + t_sumdenrho / R(3);
              R sumdenee = R(1) + t_sumdenee;
              R sumnumee = R(1) + t_sumdenee / R(3);
              for (int n = 2; n <= nkeep; ++n) {
                R n21 = R(1) + R(2 * n);
                t_sumdenrho = t2r * t_sumdenrho;
                t_sumdenee = t2e * t_sumdenee;
                sumdenrho = sumdenrho + t_sumdenrho / n21;
                sumdenee = sumdenee + t_sumdenee;
                sumnumee = sumnumee + t_sumdenee / n21;
              }
              drhof = R(1) / sumdenrho;
              deef = sumnumee / sumdenee;
            }
            R uv_part = (vna + vnb) * rhom * drhof;
            uvs1 = uvs1 + uv_part * R(2);
            uvs2 = uvs2 + uv_part * (st.u[a] + st.u[b]);
            uvs3 = uvs3 + uv_part * (st.v[a] + st.v[b]);
            uvs4 = uvs4 + uv_part * (st.w[a] + st.w[b]);
            uvs5_i = uvs5_i + uv_part * eem * deef;
            uvs5_k = uvs5_k + uv_part * (st.u[a] * st.u[b] + st.v[a] * st.v[b] + st.w[a] * st.w[b]);
            uvs5_p = uvs5_p + R(4) * (vna * pp[b] + vnb * pp[a]);
            uvs6 = uvs6 + R(2) * (pp[a] + pp[b]);
          } else {
            R uv_part = (vna + vnb) * rhom;
            uvs1 = uvs1 + uv_part * R(2);
            uvs2 = uvs2 + uv_part * (st.u[a] + st.u[b]);
            uvs3 = uvs3 + uv_part * (st.v[a] + st.v[b]);
            uvs4 = uvs4 + uv_part * (st.w[a] + st.w[b]);
            uvs5 = uvs5 + uv_part * (st.h[a] + st.h[b]);
            uvs6 = uvs6 + R(2) * (pp[a] + pp[b]);
          }
        }
      }
      const R cl = R(g.coeff[lmax - 1][l - 1]);
      acc_prod(ft1, lt1, cl, uvs1);
      acc_prod(ft2, lt2, cl, uvs2);
      acc_prod(ft3, lt3, cl, uvs3);
      acc_prod(ft4, lt4, cl, uvs4);
      acc_prod(ft5, lt5, cl, (nkeep >= 0 ? (uvs5_i + uvs5_k + uvs5_p) : uvs5));
      acc_prod(ft6, lt6, cl, uvs6);
    }
  }
  // scaling by 1/4 and 1/2 is exact, so the compensation terms scale with their sums
  fh[0] = R(0.25) * ft1; fl[0] = R(0.25) * lt1;
  fh[1] = R(0.25) * ft2; fl[1] = R(0.25) * lt2;
  fh[2] = R(0.25) * ft3; fl[2] = R(0.25) * lt3;
  fh[3] = R(0.25) * ft4; fl[3] = R(0.25) * lt4;
  fh[4] = R(0.25) * ft5; fl[4] = R(0.25) * lt5;
  if (zero_flux) {
#pragma unroll
    for (int m = 0; m < 5; ++m) fh[m] = fl[m] = R(0);
  }
  acc_add(fh[1 + DIR], fl[1 + DIR], R(0.5) * ft6);
  fl[1 + DIR] = fl[1 + DIR] + R(0.5) * lt6;
}

// Characteristic WENO flux: compute_roe_average (kernels_cpu.F90:3013-3089), eigenvectors_{x,y,z}
// (:2728-2782, :2842-2896, :2956-3010), local Lax-Friedrichs splitting with the stencil maximum
// of |u_n -+ c| (:614-675) and wenorec_1d; back-projection with the right eigenvectors (:677-683).
// TP: thermally perfect gas (Newton for the Roe-averaged temperature, gamma(T) per point; FP64).
// WZ: WENO-Z weights (weno_version = 1) instead of WENO-JS, fixed at compile time.
template <class R, int DIR, int WS, int S, bool TP = false, bool WZ = false>
__device__ __forceinline__ void weno_flux(const Geom& g, const Stencil<R, S>& st, int ord, R (&fh)[5],
                                          R (&fl)[5], R* __restrict__ gs, int gstride, const R* __restrict__ cpt,
                                          long long cstr) {
  static_assert(!TP || sizeof(R) == sizeof(double), "the thermally perfect gas is an FP64 path");
  const R rgas0 = R(g.rgas0);
  const int o0 = S - 1, o1 = S;  // the two points adjacent to the face
  // Roe average
  R uu = st.u[o0], vv = st.v[o0], ww = st.w[o0], h = st.h[o0];
  R r = fdiv(st.rho[o1], st.rho[o0]);
  r = fsqrt_pos(r);
  R rho = r * st.rho[o0];
  R rp1 = fdiv(R(1), r + R(1));
  uu = (r * st.u[o1] + uu) * rp1;
  vv = (r * st.v[o1] + vv) * rp1;
  ww = (r * st.w[o1] + ww) * rp1;
  h = (r * st.h[o1] + h) * rp1;
  R qq = R(0.5) * (uu * uu + vv * vv + ww * ww);
  R hbar = h - qq - R(g.cp_last) * R(g.t0);
  R tt, gamloc;
  if constexpr (TP) {
    // Newton on h(T) from the Roe average of the two temperatures (compute_roe_average)
    const R t_start = (r * st.t[o1] + st.t[o0]) * rp1;
    tt = tp_newton(g, g.cpc, hbar, t_start);
    gamloc = gamloc_of_t(g, tt);
  } else {
    tt = R(g.t0) + fdiv(hbar, R(g.cp0));
    gamloc = R(g.gamloc);
  }
  R cc = gamloc * tt * rgas0;
  R c, ci, b1, b2, b3;
  const R p_rho = tt * rgas0;
  const R etot = h - tt * rgas0;
  if constexpr (TP) {
    const R gm1loc = gamloc - R(1);
    c = sqrt(cc);
    ci = R(1) / c;
    const R p_e = rho * gm1loc;
    b3 = etot - rho * p_rho / p_e;
    b2 = p_e / (rho * cc);
    b1 = p_rho / cc - b2 * (etot - R(2) * qq);
  } else {
    // constant gamma: p_e = rho (gamma - 1), so b2 = (gamma - 1)/c^2 and rho p_rho/p_e =
    // p_rho/(gamma - 1); one reciprocal square root gives c and 1/c (the reference forms three
    // quotients and a square root here: the results differ in the last bits)
    ci = rsqrt(cc);
    c = cc * ci;
    const R ci2 = ci * ci;
    b2 = R(g.gm1) * ci2;
    b1 = p_rho * ci2 - b2 * (etot - R(2) * qq);
    b3 = etot - p_rho * R(g.rgm1);
  }
  const R vn = DIR == 0 ? uu : (DIR == 1 ? vv : ww);
  constexpr int t1 = DIR == 0 ? 1 : 0;
  constexpr int t2 = DIR == 2 ? 1 : 2;
  // stencil maximum of the characteristic speeds (offsets -WS+1 .. WS)
  R ev0 = R(-1), ev1 = R(-1), ev4 = R(-1);
#pragma unroll
  for (int l = 0; l < 2 * WS; ++l) {
    const int q = l + S - WS;
    const R vnq = DIR == 0 ? st.u[q] : (DIR == 1 ? st.v[q] : st.w[q]);
#if SB_CACHE_C
    static_assert(!TP, "the cached sound speed assumes a calorically perfect gas");
    const R cs = st.c[q];
#else
    R cs;
    if constexpr (sizeof(R) == sizeof(double)) {
      cs = __ldg(cpt + q * cstr);  // the aux pass's sound speed of the point (FP64 form)
    } else {
      const R gq = TP ? R(gamloc_of_t(g, double(st.t[q]))) : R(g.gamloc);
      cs = fsqrt_pos(gq * R(g.rgas0) * st.t[q]);
    }
#endif
    ev0 = fmax(fabs(vnq - cs), ev0);
    ev1 = fmax(fabs(vnq), ev1);
    ev4 = fmax(fabs(vnq + cs), ev4);
  }
  const R betascale_a = R(g.wbs_a), betascale_b = R(g.wbs_b);
  // Projection of the stencil's conserved states U and fluxes F onto the five characteristic
  // fields, point by point, using the structure of the left eigenvectors (the reference forms
  // the five dot products el(:,m).U one field at a time): with dq = Roe velocity . X(2:4),
  // s = b1 X1 + b2 (X5 - dq) and a = ci (vn X1 - X(normal momentum)),
  //   P1 = (s + a)/2, P2 = X1 - s, P3 = X(t1) - v_t1 X1, P4 = X(t2) - v_t2 X1, P5 = (s - a)/2.
  // The split values g+- = (P(F) +- lambda_m P(U))/2 of every point and field go to this
  // thread's scratch.  wenorec_1d reads g+ at the points l = 1 .. 2WS-1 and g- at l = 2 .. 2WS
  // whatever its order (vp(i-WS+1 .. i+WS-1), vm(i-WS+2 .. i+WS) with i = WS), so each side keeps
  // 2WS-1 values: gs[((m*(2WS-1) + l)*2 + side) * gstride], l counted from the first point used.
  const R lam[5] = {ev0, ev1, ev1, ev1, ev4};
  const R vel[3] = {uu, vv, ww};
#pragma unroll
  for (int l = 0; l < 2 * WS; ++l) {
    const int q = l + S - WS;
    const R rr = st.rho[q], u1 = st.u[q], v1 = st.v[q], w1 = st.w[q], h1 = st.h[q];
    const R vq[3] = {u1, v1, w1};
    const R rhovn = rr * vq[DIR];
    const R pp = rr * st.t[q] * rgas0;
    R U[5], F[5];
    U[0] = rr; U[1] = rr * u1; U[2] = rr * v1; U[3] = rr * w1; U[4] = rr * h1 - pp;
    F[0] = rhovn; F[1] = u1 * rhovn; F[2] = v1 * rhovn; F[3] = w1 * rhovn; F[4] = h1 * rhovn;
    F[1 + DIR] = F[1 + DIR] + pp;
    R PU[5], PF[5];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const R* X = side == 0 ? U : F;
      R* P = side == 0 ? PU : PF;
      const R dq = uu * X[1] + vv * X[2] + ww * X[3];
      const R sv = b1 * X[0] + b2 * (X[4] - dq);
      const R av = ci * (vn * X[0] - X[1 + DIR]);
      P[0] = R(0.5) * (sv + av);
      P[1] = X[0] - sv;
      P[2] = X[1 + t1] - vel[t1] * X[0];
      P[3] = X[1 + t2] - vel[t2] * X[0];
      P[4] = R(0.5) * (sv - av);
    }
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      const R cm = R(0.5) * (PF[m] + lam[m] * PU[m]);
      if (l < 2 * WS - 1) gs[((m * (2 * WS - 1) + l) * 2) * gstride] = cm;
      if (l > 0) gs[((m * (2 * WS - 1) + l - 1) * 2 + 1) * gstride] = PF[m] - cm;
    }
  }
  // reconstruction, one characteristic field per iteration (rolled: one copy of wenorec)
  R fi[5];
  SB_UNROLL_(SB_WENO_UNROLL)
  for (int m = 0; m < 5; ++m) {
    R gp[2 * WS], gm[2 * WS];
#pragma unroll
    for (int l = 0; l < 2 * WS; ++l) {
      gp[l] = l < 2 * WS - 1 ? gs[((m * (2 * WS - 1) + l) * 2) * gstride] : R(0);
      gm[l] = l > 0 ? gs[((m * (2 * WS - 1) + l - 1) * 2 + 1) * gstride] : R(0);
    }
    const R bs = (m == 2 || m == 3) ? betascale_b : betascale_a;
    const R f = wenorec<R, WS>(gp, gm, ord, WZ ? 1 : 0, bs);
#pragma unroll
    for (int mm = 0; mm < 5; ++mm)
      if (mm == m) fi[mm] = f;
  }
  // back-projection with the right eigenvectors, er(m,:) = (1, u - c n, h - vn c) for m = 1,
  // (1, u, b3) for m = 2, (0, e_t, v_t) for m = 3, 4, (1, u + c n, h + vn c) for m = 5,
  // accumulated term by term (compensated in the mixed form)
#pragma unroll
  for (int m = 0; m < 5; ++m) fh[m] = fl[m] = R(0);
  acc_add(fh[0], fl[0], fi[0]);
  acc_add(fh[0], fl[0], fi[1]);
  acc_add(fh[0], fl[0], fi[4]);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    acc_prod(fh[1 + d], fl[1 + d], vel[d], fi[0]);
    acc_prod(fh[1 + d], fl[1 + d], vel[d], fi[1]);
    acc_prod(fh[1 + d], fl[1 + d], vel[d], fi[4]);
    if (d == DIR) {
      acc_prod(fh[1 + d], fl[1 + d], -c, fi[0]);
      acc_prod(fh[1 + d], fl[1 + d], c, fi[4]);
    }
    if (d == t1) acc_add(fh[1 + d], fl[1 + d], fi[2]);
    if (d == t2) acc_add(fh[1 + d], fl[1 + d], fi[3]);
  }
  acc_prod(fh[4], fl[4], h - vn * c, fi[0]);
  acc_prod(fh[4], fl[4], b3, fi[1]);
  acc_prod(fh[4], fl[4], vel[t1], fi[2]);
  acc_prod(fh[4], fl[4], vel[t2], fi[3]);
  acc_prod(fh[4], fl[4], h + vn * c, fi[4]);
}

// Rusanov (component-wise local Lax-Friedrichs) WENO flux of the *_hybrid_rusanov kernels
// (kernels_cpu.F90:692-941 for x, same in y and z): stencil maximum of |u_n -+ c|, split
// values of the conserved fluxes, wenorec with the scales of wenorec_1d_rusanov (:2325-2523).
template <class R, int DIR, int WS, int S, bool TP = false, bool WZ = false>
__device__ __forceinline__ void rusanov_flux(const Geom& g, const Stencil<R, S>& st, int ord, R (&fh)[5], R (&fl)[5],
                                             const R* __restrict__ cpt, long long cstr) {
  static_assert(!TP || sizeof(R) == sizeof(double), "the thermally perfect gas is an FP64 path");
  const R rgas0 = R(g.rgas0);
  R evmax = R(-1);
#pragma unroll
  for (int l = 0; l < 2 * WS; ++l) {
    const int q = l + S - WS;
    const R un = DIR == 0 ? st.u[q] : (DIR == 1 ? st.v[q] : st.w[q]);
    R c;
    if constexpr (sizeof(R) == sizeof(double)) {
      c = __ldg(cpt + q * cstr);
    } else {
      const R gq = TP ? R(gamloc_of_t(g, double(st.t[q]))) : R(g.gamloc);
      c = fsqrt_pos(gq * rgas0 * st.t[q]);
    }
    const R evm = fmax(fabs(un - c), fabs(un + c));
    evmax = fmax(evm, evmax);
  }
  R bsc[5];
  bsc[0] = R(g.wbs_a);
  bsc[1] = R(g.wbs_b);
  bsc[2] = bsc[1];
  bsc[3] = bsc[1];
  bsc[4] = R(g.wbs_c);
#pragma unroll 1
  for (int m = 0; m < 5; ++m) {
    R gp[2 * WS], gm[2 * WS];
#pragma unroll
    for (int l = 0; l < 2 * WS; ++l) {
      const int q = l + S - WS;
      const R rho = st.rho[q], h = st.h[q];
      const R vel[3] = {st.u[q], st.v[q], st.w[q]};
      const R rhou = rho * vel[DIR];
      const R pp = rho * st.t[q] * rgas0;
      const R rhoevm = rho * evmax;
      R evm, c;
      if (m == 0) {
        evm = rhou;
        c = R(0.5) * (evm + rhoevm);
      } else if (m == 4) {
        evm = h * rhou;
        c = R(0.5) * (evm + evmax * (rho * h - pp));
      } else {
        const R vd = m == 1 ? vel[0] : (m == 2 ? vel[1] : vel[2]);
        evm = vd * rhou;
        if (m == 1 + DIR) evm = evm + pp;
        c = R(0.5) * (evm + rhoevm * vd);
      }
      gp[l] = c;
      gm[l] = evm - c;
    }
    const R bs = m == 0 ? bsc[0] : (m == 4 ? bsc[4] : bsc[1]);
    const R f = wenorec<R, WS>(gp, gm, ord, WZ ? 1 : 0, bs);
#pragma unroll
    for (int mm = 0; mm < 5; ++mm)
      if (mm == m) { fh[mm] = f; fl[mm] = R(0); }
  }
}

}  // namespace sb200
