// Learned probability model for the rANS coder of solved blocks (stream
// format version 3; the reference has no counterpart and keeps format version
// 2, pentago/shard/arithmetic.cc:456-495, which stays the fallback).
//
// Symbols are the on-disk ternaries of a block, 256 per node in rotation order
// r = i0 + 4 i1 + 16 i2 + 64 i3 (shard/shard.cc:448-449).  A node's symbols are
// coded in 128 steps; step s codes rotations s and s + 128 (i3 two apart, so
// never neighbours).  The block's n nodes are coded by 32 lanes, lane l taking
// the run of nodes l R .. l R + R - 1 (R = ceil(n / 32)) one after another, so
// a node's previous node in its run is coded before it.  The probability of
// symbol r comes from a 3-layer MLP (hidden 64, bf16 weights, fp32
// accumulation) over 124 binary features:
//
//   0..71    stones of the node's board: 18 q + 2 c + colour (colour 0 black,
//            1 white) for cell c of quadrant q;
//   72..87   rotation: 72 + 4 q + i_q;
//   88..119  the 8 neighbouring rotations (i_q + 1 and i_q + 3 in quadrant q,
//            neighbour n = 2 q + (0 | 1)): 88 + 4 n + v, v = that rotation's
//            symbol if it was coded in an earlier step, else 3;
//   120..123 the previous node of the run: 120 + v, v = its symbol of the
//            same rotation, 3 for the first node of a run.
//
// Encoder and decoder must derive identical integer frequencies, so every
// float operation on the coding path is either a separately rounded IEEE
// operation in the fixed order below (no contraction, explicit fma) or exact,
// which also makes the coder reproducible on the CPU:
//
//   node[k] = b1[k], then + W1[f][k] for each stone feature f ascending
//   S1[k]   = sum of W1[f][k] over the 13 rotation, neighbour and previous-node
//             features, exact
//   a1 = node + S1,  hq[k] = rint(min(max(a1 * 16, 0), 255))   (an integer 0..255)
//   a2[j] = fma(C[j], 1/16, b2[j]),  C[j] = sum over k of W2[k][j] hq[k], exact
//   z[c] = b3[c] + ((P_0 + P_1) + (P_2 + P_3)), P_t = fma chain from 0 over
//          the columns j with (j >> 1) & 3 = t ascending of W3[j][c] relu(a2[j])
//
// then lm_freqs turns the logits into 15-bit frequencies (each at least 1,
// summing to 2^15).  S1 and C are exact because a model's W1 rows 72..123 and
// its W2 lie on grids: every column (hidden unit k of W1 rows 72..123, output
// j of W2) is integers of magnitude at most 127 times 2^-e (lm_grid_exp), so
// each term and partial sum is a multiple of 2^-e below 2^21 2^-e and an fp32
// sum in any order is exact.  The coder forms both sums on the tensor cores
// (bf16 inputs: one-hot features and integer activations, fp32
// accumulation); models are checked for the grids when loaded.  Training may
// run the same network in any order; only the coder needs this one.
#pragma once
#include "superscore.cuh"
#include <cmath>
#include <cstdint>
#include <cstring>

namespace pg {

constexpr int kLmIn = 124, kLmHidden = 64, kLmOut = 3;
constexpr int kLmRot = 72, kLmCtx = 88, kLmPrev = 120;
// Parameter layout (fp32 master copy and bf16 model alike)
constexpr int kLmW1 = 0;
constexpr int kLmB1 = kLmW1 + kLmIn * kLmHidden;
constexpr int kLmW2 = kLmB1 + kLmHidden;
constexpr int kLmB2 = kLmW2 + kLmHidden * kLmHidden;
constexpr int kLmW3 = kLmB2 + kLmHidden;
constexpr int kLmB3 = kLmW3 + kLmHidden * kLmOut;
constexpr int kLmParams = kLmB3 + kLmOut;  // 12355
// Serialized model: magic "PGLM", version 3, parameter count, bf16 parameters
constexpr uint32_t kLmMagic = 0x4d4c4750u;
constexpr uint32_t kLmModelVersion = 3;
// Activations entering layer 2: integers 0..kLmActMax, a1 scaled by kLmActScale
constexpr float kLmActScale = 16.f, kLmActInv = 0.0625f, kLmActMax = 255.f;
constexpr int kLmModelHeader = 12;
constexpr int64_t kLmModelBytes = kLmModelHeader + 2 * int64_t(kLmParams);
// Coder: 32-bit states, 16-bit words, 15-bit probabilities, 32 lanes
constexpr uint32_t kLmProbBits = 15, kLmProbTotal = 1u << kLmProbBits;
constexpr uint32_t kLmLower = 1u << 16;
constexpr int kLmLanes = 32;
constexpr uint32_t kLmVersion = 3;
// Stream: version u32 | model hash u64 | nodes u32 | words u32 | 32 lane states u32 | words u16.
// Lane l codes its run of nodes l R .. l R + R - 1 in order, each node step by
// step (rotation s, then s + 128).
constexpr int kLmStreamHeader = 20 + 4 * kLmLanes;

PG_HD float f_add(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
PG_HD float f_mul(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
PG_HD float f_div(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fdiv_rn(a, b);
#else
  return a / b;
#endif
}
PG_HD float f_fma(float a, float b, float c) {
#ifdef __CUDA_ARCH__
  return __fmaf_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}
PG_HD float f_bits(uint32_t u) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}
PG_HD uint32_t f_raw(float f) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
#endif
}
PG_HD float bf16_value(uint16_t h) { return f_bits(uint32_t(h) << 16); }
// Round to nearest even (parameters are finite).
PG_HD uint16_t bf16_round(float f) {
  const uint32_t u = f_raw(f);
  return uint16_t((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}
PG_HD float relu(float a) { return a > 0.f ? a : 0.f; }

// rint(v) for 0 <= v <= 2^22: adding 2^23 rounds to an integer (ties to even).
PG_HD float f_rint_small(float v) { return f_add(f_add(v, 8388608.f), -8388608.f); }

// The quantized activation hq of a1: rint(min(max(a1 * 16, 0), 255)), an
// integer 0..255 as a float.
PG_HD float lm_act_q(float a) {
  float v = f_mul(a, kLmActScale);
  v = v > 0.f ? v : 0.f;
  return f_rint_small(v < kLmActMax ? v : kLmActMax);
}

// Round to nearest, ties to even (v finite, |v| < 2^31).
PG_HD float f_rint(float v) {
#ifdef __CUDA_ARCH__
  return __int2float_rn(__float2int_rn(v));
#else
  return std::nearbyint(v);
#endif
}

// 2^e as a float, for -126 <= e <= 127.
PG_HD float f_pow2(int e) { return f_bits(uint32_t(127 + e) << 23); }

// The grid of a column whose largest magnitude is m > 0 (finite): its
// weights are integers of magnitude at most 127 times 2^-e, with
// e = 7 - x for m = f 2^x, f in [0.5, 1).  Returns e.
PG_HD int lm_grid_exp(float m) {
  int s = 0;
  if (m < f_pow2(-126)) {   // subnormal: scale into the normal range first (exact)
    m = f_mul(m, f_pow2(64));
    s = 64;
  }
  const int x = int(f_raw(m) >> 23 & 0xff) - 126;   // m = f 2^x with f in [0.5, 1)
  return 7 - (x - s);
}
// w on grid e: the nearest multiple of 2^-e (ties to even), clamped to
// +-127 2^-e.  Computed as w 2^e in two power-of-two steps (exact) so e may
// exceed 127.
PG_HD float lm_grid_quantize(float w, int e) {
  const int e1 = e / 2, e2 = e - e1;
  float q = f_rint(f_mul(f_mul(w, f_pow2(e1)), f_pow2(e2)));
  q = q > 127.f ? 127.f : q < -127.f ? -127.f : q;
  return f_mul(f_mul(q, f_pow2(-e1)), f_pow2(-e2));
}
// A column of n finite weights w[0], w[stride], ... moved onto its grid, in
// place.  A column on its grid is left unchanged (its largest magnitude
// keeps the grid).
PG_HD void lm_grid_column(float* w, int n, int stride) {
  float m = 0.f;
  for (int k = 0; k < n; k++) m = fmaxf(m, fabsf(w[k * stride]));
  if (!(m > 0.f)) {
    for (int k = 0; k < n; k++) w[k * stride] = 0.f;
    return;
  }
  const int e = lm_grid_exp(m);
  for (int k = 0; k < n; k++) w[k * stride] = lm_grid_quantize(w[k * stride], e);
}
// Every grid column of a parameter vector (fp32 layout of kLmParams), in place.
PG_HD void lm_grid_params(float* p) {
  for (int k = 0; k < kLmHidden; k++) lm_grid_column(p + kLmW1 + kLmRot * kLmHidden + k, kLmIn - kLmRot, kLmHidden);
  for (int j = 0; j < kLmHidden; j++) lm_grid_column(p + kLmW2 + j, kLmHidden, kLmHidden);
}

// 2^d for d <= 0, 0 below -24: d = n + t with n = floor(d), t in [0, 1); 2^t
// from its Taylor series (coefficients ln(2)^i / i!, degree 7, Horner), then
// an exact power-of-two scale.  Accuracy is irrelevant to correctness; only
// determinism matters, and every step is an exactly specified IEEE operation.
PG_HD float lm_exp2(float d) {
  if (!(d >= -24.f)) return 0.f;
  const float n = floorf(d);
  const float t = f_add(d, -n);
  float p = 1.5252734e-05f;
  p = f_fma(p, t, 1.5403530e-04f);
  p = f_fma(p, t, 1.3333558e-03f);
  p = f_fma(p, t, 9.6181291e-03f);
  p = f_fma(p, t, 5.5504109e-02f);
  p = f_fma(p, t, 2.4022651e-01f);
  p = f_fma(p, t, 6.9314718e-01f);
  p = f_fma(p, t, 1.0f);
  return f_mul(p, f_bits(uint32_t(127 + int(n)) << 23));
}

struct lm_freq_t {
  uint32_t f[3], cum[3];
};

// Logits -> frequencies: e_c = 2^((z_c - max z) log2 e), f_c = 1 + trunc(e_c /
// (e_0 + e_1 + e_2) * 32765), the remainder to the largest (first on ties).
// Any logits, NaN and infinities included, give a valid table.
PG_HD lm_freq_t lm_freqs(const float* z) {
  float m = z[0];
  if (z[1] > m) m = z[1];
  if (z[2] > m) m = z[2];
  float e[3];
  for (int c = 0; c < 3; c++) e[c] = lm_exp2(f_mul(f_add(z[c], -m), 1.44269504f));
  const float s = f_add(f_add(e[0], e[1]), e[2]);
  lm_freq_t t;
  for (int c = 0; c < 3; c++) {
    const float q = f_mul(f_div(e[c], s), float(kLmProbTotal - 3));
    t.f[c] = 1 + (q >= 1.f ? uint32_t(q) : 0u);
  }
  int big = 0;
  if (t.f[1] > t.f[big]) big = 1;
  if (t.f[2] > t.f[big]) big = 2;
  t.f[big] += kLmProbTotal - (t.f[0] + t.f[1] + t.f[2]);
  t.cum[0] = 0;
  t.cum[1] = t.f[0];
  t.cum[2] = t.f[0] + t.f[1];
  return t;
}

// Rotation index r' of neighbour n (quadrant q = n / 2 turned one step further
// for even n, one step back for odd n).
PG_HD int lm_neighbour(int r, int n) {
  const int q = n >> 1, s = 2 * q;
  const int i = (r >> s) & 3;
  const int j = (i + ((n & 1) ? 3 : 1)) & 3;
  return r + ((j - i) << s);
}

// Per-stream block geometry, resolved on the host: the block's node shape and
// where its quadrant coordinates start in the rotation-minimal quadrant list.
struct lm_block_t {
  int64_t nodes;
  int32_t qbase[4];  // rmin_off[bucket] + 8 * block[q]
  int32_t shape[4];  // nodes along each quadrant axis (C order, axis 3 fastest)
};

// Quadrant ids of node i of a block (C order over shape).
PG_HD void lm_node_quadrants(const lm_block_t& B, int64_t i, const uint16_t* rmin_flat, uint16_t* qid) {
  for (int q = 3; q >= 0; q--) {
    const int idx = int(i % B.shape[q]);
    i /= B.shape[q];
    qid[q] = rmin_flat[B.qbase[q] + idx];
  }
}

// Stone features of a node, ascending.  Returns the count (at most 36).
PG_HD int lm_node_features(const uint16_t* qid, const uint16_t* unpack, uint8_t* f) {
  int n = 0;
  for (int q = 0; q < 4; q++) {
    const uint32_t b = unpack[2 * qid[q]], w = unpack[2 * qid[q] + 1];
    for (int c = 0; c < 9; c++) {
      if (b >> c & 1) f[n++] = uint8_t(18 * q + 2 * c);
      if (w >> c & 1) f[n++] = uint8_t(18 * q + 2 * c + 1);
    }
  }
  return n;
}

// Rotation a was coded in an earlier step than rotation r.
PG_HD bool lm_before(int a, int r) { return (a & 127) < (r & 127); }

// Context of symbol r: per quadrant axis q, u_q = v_{2q} + 4 v_{2q+1}.
PG_HD void lm_context(const uint8_t* sym, int r, int* u) {
  for (int q = 0; q < 4; q++) {
    const int a = lm_neighbour(r, 2 * q), b = lm_neighbour(r, 2 * q + 1);
    const int va = lm_before(a, r) ? sym[a] : 3, vb = lm_before(b, r) ? sym[b] : 3;
    u[q] = va + 4 * vb;
  }
}

}  // namespace pg
