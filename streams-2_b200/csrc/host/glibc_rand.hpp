// Reentrant restatement of glibc's rand() for the seeded fields and random planes.
#pragma once

#include <cstdint>

namespace streams_b200 {

// glibc's rand() (the additive feedback generator behind random(), TYPE_3: degree 31,
// separation 3), restated as a per-call object so that case set-ups running in several threads
// do not share one global sequence.  Seeding: r0 = seed (1 if 0), r_i = 16807 r_{i-1} mod
// (2^31 - 1) for i < 31, r_i = r_{i-31} for i = 31..33; then r_i = r_{i-31} + r_{i-3} (mod 2^32)
// and output k is r_{k+344} >> 1.  crandom.c (code/third-party/crandom/crandom.c:12-29) calls
// srand/rand, so the draws are those of the reference.
class GlibcRand {
 public:
  explicit GlibcRand(unsigned seed) {
    int32_t r[34];
    r[0] = seed == 0 ? 1 : static_cast<int32_t>(seed);
    for (int i = 1; i < 31; ++i) {
      const int32_t hi = r[i - 1] / 127773, lo = r[i - 1] % 127773;
      int32_t word = 16807 * lo - 2836 * hi;
      if (word < 0) word += 2147483647;
      r[i] = word;
    }
    for (int i = 31; i < 34; ++i) r[i] = r[i - 31];
    for (int i = 0; i < 34; ++i) ring_[i] = static_cast<uint32_t>(r[i]);
    pos_ = 34;
    for (int i = 34; i < 344; ++i) next_raw();
  }
  int operator()() { return static_cast<int>(next_raw() >> 1); }
  void discard(long long n) {
    for (long long q = 0; q < n; ++q) next_raw();
  }
  // the 34-word ring and the position (pos mod 34 is the next slot written), for devices that
  // continue the sequence
  const uint32_t* ring() const { return ring_; }
  long long position() const { return pos_; }

 private:
  uint32_t next_raw() {
    const uint32_t v = ring_[(pos_ - 31) % 34] + ring_[(pos_ - 3) % 34];
    ring_[pos_ % 34] = v;
    ++pos_;
    return v;
  }
  uint32_t ring_[34];
  long long pos_;
};

}  // namespace streams_b200
