// Counting scalar of the oracle (measurement infrastructure, not product code).
//
// A double that tallies every floating-point operation applied to it, so that the oracle's own
// face-flux code, instantiated with it, gives the exact FP64 operation count of a central face
// and of a WENO face as the reference's algorithm performs them (kernels_cpu.F90: the hybrid
// flux kernels, compute_roe_average, eigenvectors_*, wenorec_1d).  Conventions: +, -, *, / and
// sqrt count one operation each (an FMA-contracted a*b+c counts two); sign changes, fabs and
// literal constants count nothing; max/min and comparisons are tallied apart (they are not
// floating-point arithmetic); quantities that depend only on the case (gamma of a calorically
// perfect gas, the WENO indicator scales) are constants and count nothing.
#pragma once

#include <algorithm>
#include <cmath>

namespace streams_oracle {

struct FlopTally {
  long long add = 0, mul = 0, div = 0, sqrt = 0, special = 0, cmp = 0;
  long long flops() const { return add + mul + div + sqrt + special; }
};
inline FlopTally& flop_tally() {
  static thread_local FlopTally t;
  return t;
}

struct Counted {
  double v = 0.0;
  Counted() = default;
  Counted(double x) : v(x) {}  // NOLINT: literals and case constants enter uncounted
  explicit operator double() const { return v; }
};

inline Counted operator+(Counted a, Counted b) { ++flop_tally().add; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { ++flop_tally().add; return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { ++flop_tally().mul; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { ++flop_tally().div; return Counted(a.v / b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline bool operator<(Counted a, Counted b) { ++flop_tally().cmp; return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { ++flop_tally().cmp; return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { ++flop_tally().cmp; return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { ++flop_tally().cmp; return a.v >= b.v; }
inline Counted sqrt(Counted a) { ++flop_tally().sqrt; return Counted(std::sqrt(a.v)); }
inline Counted fabs(Counted a) { return Counted(std::fabs(a.v)); }
inline Counted max(Counted a, Counted b) { ++flop_tally().cmp; return Counted(std::max(a.v, b.v)); }
inline Counted pow(Counted a, int l) { ++flop_tally().special; return Counted(std::pow(a.v, l)); }
inline Counted log(Counted a) { ++flop_tally().special; return Counted(std::log(a.v)); }

}  // namespace streams_oracle
