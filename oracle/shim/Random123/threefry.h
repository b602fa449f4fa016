// Threefry-2x64-20, written from the published description (Salmon, Moraes,
// Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11, and the
// Threefish key schedule of the Skein specification).  The reference pins
// Random123 at commit 9545ff6413f258be2f04c1d319d99aaef7521150
// (third_party/deps.bzl:7-14) but does not vendor it; only this one generator
// is used (utility/threefry.cc:6-15), so this header is enough to compile the
// reference sources into the CPU oracle.
#pragma once

#include <cstdint>

struct threefry2x64_ctr_t {
  uint64_t v[2];
};
typedef threefry2x64_ctr_t threefry2x64_key_t;

static inline threefry2x64_ctr_t threefry2x64(threefry2x64_ctr_t in, threefry2x64_key_t k) {
  static const int rot[8] = {16, 42, 12, 31, 16, 32, 24, 21};
  const uint64_t ks[3] = {k.v[0], k.v[1], 0x1BD11BDAA9FC1A22ull ^ k.v[0] ^ k.v[1]};
  uint64_t x0 = in.v[0] + ks[0], x1 = in.v[1] + ks[1];
  for (int r = 0; r < 20; r++) {
    x0 += x1;
    x1 = (x1 << rot[r & 7]) | (x1 >> (64 - rot[r & 7]));
    x1 ^= x0;
    if ((r & 3) == 3) {
      const int i = (r + 1) >> 2;
      x0 += ks[i % 3];
      x1 += ks[(i + 1) % 3] + uint64_t(i);
    }
  }
  threefry2x64_ctr_t out;
  out.v[0] = x0;
  out.v[1] = x1;
  return out;
}
