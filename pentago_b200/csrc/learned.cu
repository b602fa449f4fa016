// Learned-model rANS for solved blocks (stream format version 3) and the
// kernels that train its network.  The model and the exact arithmetic of the
// coding path are specified in learned.cuh.
//
// Coder layout: one warp per stream; node i of the block is coded by lane
// i % 32, whose own rANS state walks the steps (round i / 32, rotation r) in
// order.  The encoder runs the steps backward; at each step the lanes that
// renormalize append one 16-bit word each, in lane order, to the stream's
// shared word array, so the decoder (running forward) finds the words of its
// step as the last unread ones.  The network runs once per symbol on every
// lane, from tables staged in shared memory (stone rows of W1, pair sums of
// the rotation and neighbour rows, W2, W3).
//
// Training: one thread per sample (stream, node, rotation) computes the
// forward pass and the backward pass of the softmax cross entropy with the
// bf16-rounded weights; the CTA accumulates the gradient of its samples in
// shared memory and registers, partial sums per CTA are added in a fixed
// order, and an Adam step updates the fp32 master parameters.
#include "learned.cuh"
#include "lines.h"
#include "runtime.h"
#include "tables.h"
#include "../../include/pentago_b200.h"
#include <algorithm>
#include <vector>

namespace pg {

// Format-2 coder (rans.cu); the decoder can be restricted to version-2 streams.
int64_t rans_stream_bound(int64_t n);
int launch_rans_encode(const uint8_t* symbols, const int64_t* offsets, int nstreams, uint8_t* out,
                       const int64_t* out_offsets, int64_t* sizes, const int64_t* expect, cudaStream_t stream);
int launch_rans_decode(const uint8_t* in, const int64_t* in_offsets, const int64_t* in_sizes, int nstreams,
                       uint8_t* symbols, const int64_t* sym_offsets, const int64_t* sym_caps, int64_t* status,
                       int only_v2, cudaStream_t stream);

constexpr int kLmWarps = 4;
constexpr int kLmThreads = 32 * kLmWarps;
constexpr int kW1Pad = 65;  // stone rows padded so lanes reading different rows use different banks

// Coding tables in shared memory.
struct lm_tables {
  float w1s[72 * kW1Pad];
  float ra[kLmHidden][16], rb[kLmHidden][16];  // [k][i0 + 4 i1], [k][i2 + 4 i3]
  float pt[4][kLmHidden][16];                  // [q][k][va + 4 vb]
  float w2[kLmHidden][kLmHidden];              // [k][j]
  float b1[kLmHidden], b2[kLmHidden];
  float w3[kLmHidden][4];                      // [j][c]
  float b3[4];
};

__device__ void lm_build_tables(lm_tables& S, const uint16_t* __restrict__ P, int tid, int nt) {
  auto w = [&](int i) { return bf16_value(P[i]); };
  for (int i = tid; i < 72 * kLmHidden; i += nt) S.w1s[(i / kLmHidden) * kW1Pad + i % kLmHidden] = w(kLmW1 + i);
  for (int i = tid; i < kLmHidden * 16; i += nt) {
    const int k = i / 16, u = i % 16, a = u & 3, b = u >> 2;
    S.ra[k][u] = f_add(w(kLmW1 + (kLmRot + a) * kLmHidden + k), w(kLmW1 + (kLmRot + 4 + b) * kLmHidden + k));
    S.rb[k][u] = f_add(w(kLmW1 + (kLmRot + 8 + a) * kLmHidden + k), w(kLmW1 + (kLmRot + 12 + b) * kLmHidden + k));
    for (int q = 0; q < 4; q++)
      S.pt[q][k][u] = f_add(w(kLmW1 + (kLmCtx + 8 * q + a) * kLmHidden + k),
                            w(kLmW1 + (kLmCtx + 8 * q + 4 + b) * kLmHidden + k));
  }
  for (int i = tid; i < kLmHidden * kLmHidden; i += nt) S.w2[i / kLmHidden][i % kLmHidden] = w(kLmW2 + i);
  for (int i = tid; i < kLmHidden; i += nt) {
    S.b1[i] = w(kLmB1 + i);
    S.b2[i] = w(kLmB2 + i);
    for (int c = 0; c < 3; c++) S.w3[i][c] = w(kLmW3 + i * kLmOut + c);
    S.w3[i][3] = 0.f;
  }
  if (tid < 3) S.b3[tid] = w(kLmB3 + tid);
  if (tid == 3) S.b3[3] = 0.f;
}

// node[k] = b1[k] + stone rows, ascending.
__device__ __forceinline__ void lm_node_sum(const lm_tables& S, const uint8_t* feats, int nf, float* node) {
#pragma unroll
  for (int k = 0; k < kLmHidden; k++) node[k] = S.b1[k];
  for (int i = 0; i < nf; i++) {
    const float* row = S.w1s + feats[i] * kW1Pad;
#pragma unroll
    for (int k = 0; k < kLmHidden; k++) node[k] = f_add(node[k], row[k]);
  }
}

// Logits of one symbol (the order of learned.cuh).
__device__ __forceinline__ void lm_logits(const lm_tables& S, const float* node, int r, const int* u, float* z) {
  const int ua = r & 15, ub = r >> 4;
  float a2[kLmHidden];
#pragma unroll
  for (int j = 0; j < kLmHidden; j++) a2[j] = S.b2[j];
#pragma unroll
  for (int k = 0; k < kLmHidden; k++) {
    const float rot = f_add(S.ra[k][ua], S.rb[k][ub]);
    const float ctx = f_add(f_add(S.pt[0][k][u[0]], S.pt[1][k][u[1]]), f_add(S.pt[2][k][u[2]], S.pt[3][k][u[3]]));
    const float h = relu(f_add(f_add(node[k], rot), ctx));
    const float4* w = reinterpret_cast<const float4*>(S.w2[k]);
#pragma unroll
    for (int j4 = 0; j4 < kLmHidden / 4; j4++) {
      const float4 v = w[j4];
      a2[4 * j4 + 0] = f_fma(v.x, h, a2[4 * j4 + 0]);
      a2[4 * j4 + 1] = f_fma(v.y, h, a2[4 * j4 + 1]);
      a2[4 * j4 + 2] = f_fma(v.z, h, a2[4 * j4 + 2]);
      a2[4 * j4 + 3] = f_fma(v.w, h, a2[4 * j4 + 3]);
    }
  }
  z[0] = S.b3[0];
  z[1] = S.b3[1];
  z[2] = S.b3[2];
#pragma unroll
  for (int j = 0; j < kLmHidden; j++) {
    const float h = relu(a2[j]);
    const float4 v = *reinterpret_cast<const float4*>(S.w3[j]);
    z[0] = f_fma(v.x, h, z[0]);
    z[1] = f_fma(v.y, h, z[1]);
    z[2] = f_fma(v.z, h, z[2]);
  }
}

// Logits of the two symbols of step s (rotations s and s + 128) of one node,
// whose node sums are node[k * 32] (the lane's column of its warp's block).
// Each logit follows the order of learned.cuh exactly; the pair shares the
// node sums, the RA lookup and the W2 rows.
__device__ __forceinline__ void lm_logits2(const lm_tables& S, const float* node, int s, const int* uA,
                                           const int* uB, float* zA, float* zB) {
  const int ua = s & 15, ubA = s >> 4, ubB = ubA + 8;
  float a2A[kLmHidden], a2B[kLmHidden];
#pragma unroll
  for (int j = 0; j < kLmHidden; j++) { a2A[j] = S.b2[j]; a2B[j] = S.b2[j]; }
#pragma unroll 4
  for (int k = 0; k < kLmHidden; k++) {
    const float nk = node[32 * k], ra = S.ra[k][ua];
    const float ctxA = f_add(f_add(S.pt[0][k][uA[0]], S.pt[1][k][uA[1]]), f_add(S.pt[2][k][uA[2]], S.pt[3][k][uA[3]]));
    const float ctxB = f_add(f_add(S.pt[0][k][uB[0]], S.pt[1][k][uB[1]]), f_add(S.pt[2][k][uB[2]], S.pt[3][k][uB[3]]));
    const float hA = relu(f_add(f_add(nk, f_add(ra, S.rb[k][ubA])), ctxA));
    const float hB = relu(f_add(f_add(nk, f_add(ra, S.rb[k][ubB])), ctxB));
    const float4* w = reinterpret_cast<const float4*>(S.w2[k]);
#pragma unroll
    for (int j4 = 0; j4 < kLmHidden / 4; j4++) {
      const float4 v = w[j4];
      a2A[4 * j4 + 0] = f_fma(v.x, hA, a2A[4 * j4 + 0]);
      a2A[4 * j4 + 1] = f_fma(v.y, hA, a2A[4 * j4 + 1]);
      a2A[4 * j4 + 2] = f_fma(v.z, hA, a2A[4 * j4 + 2]);
      a2A[4 * j4 + 3] = f_fma(v.w, hA, a2A[4 * j4 + 3]);
      a2B[4 * j4 + 0] = f_fma(v.x, hB, a2B[4 * j4 + 0]);
      a2B[4 * j4 + 1] = f_fma(v.y, hB, a2B[4 * j4 + 1]);
      a2B[4 * j4 + 2] = f_fma(v.z, hB, a2B[4 * j4 + 2]);
      a2B[4 * j4 + 3] = f_fma(v.w, hB, a2B[4 * j4 + 3]);
    }
  }
  zA[0] = zB[0] = S.b3[0];
  zA[1] = zB[1] = S.b3[1];
  zA[2] = zB[2] = S.b3[2];
#pragma unroll
  for (int j = 0; j < kLmHidden; j++) {
    const float4 v = *reinterpret_cast<const float4*>(S.w3[j]);
    const float hA = relu(a2A[j]), hB = relu(a2B[j]);
    zA[0] = f_fma(v.x, hA, zA[0]);
    zA[1] = f_fma(v.y, hA, zA[1]);
    zA[2] = f_fma(v.z, hA, zA[2]);
    zB[0] = f_fma(v.x, hB, zB[0]);
    zB[1] = f_fma(v.y, hB, zB[1]);
    zB[2] = f_fma(v.z, hB, zB[2]);
  }
}

// node[k * 32] = b1[k] + stone rows ascending, for this lane's node.
__device__ __forceinline__ void lm_node_store(const lm_tables& S, const uint8_t* feats, int nf, float* node) {
#pragma unroll
  for (int kc = 0; kc < kLmHidden; kc += 16) {
    float acc[16];
#pragma unroll
    for (int i = 0; i < 16; i++) acc[i] = S.b1[kc + i];
    for (int f = 0; f < nf; f++) {
      const float* row = S.w1s + feats[f] * kW1Pad + kc;
#pragma unroll
      for (int i = 0; i < 16; i++) acc[i] = f_add(acc[i], row[i]);
    }
#pragma unroll
    for (int i = 0; i < 16; i++) node[32 * (kc + i)] = acc[i];
  }
}

__device__ __forceinline__ void lm_context_clamped(const uint8_t* sym, int r, int* u) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int a = lm_neighbour(r, 2 * q), b = lm_neighbour(r, 2 * q + 1);
    const int va = lm_before(a, r) ? (sym[a] & 3) : 3, vb = lm_before(b, r) ? (sym[b] & 3) : 3;
    u[q] = va + 4 * vb;
  }
}

__device__ __forceinline__ int lm_load_node(const lm_block_t& B, int64_t i, const dev_tables_t& T, uint8_t* feats) {
  uint16_t qid[4];
  lm_node_quadrants(B, i, T.rmin_flat, qid);
  return lm_node_features(qid, T.unpack, feats);
}

__device__ __forceinline__ void put16(uint8_t* p, uint16_t v) { p[0] = uint8_t(v); p[1] = uint8_t(v >> 8); }
__device__ __forceinline__ uint16_t get16(const uint8_t* p) { return uint16_t(p[0] | p[1] << 8); }
__device__ __forceinline__ void put32(uint8_t* p, uint32_t v) { for (int i = 0; i < 4; i++) p[i] = uint8_t(v >> (8 * i)); }
__device__ __forceinline__ uint32_t get32(const uint8_t* p) {
  return uint32_t(p[0]) | uint32_t(p[1]) << 8 | uint32_t(p[2]) << 16 | uint32_t(p[3]) << 24;
}

// Dynamic shared memory of the coding kernels: the tables, then each warp's
// node sums (64 x 32 floats, one column per lane).
constexpr size_t kLmNodeFloats = kLmHidden * 32;
constexpr size_t kLmCodeSmem = sizeof(lm_tables) + sizeof(float) * kLmNodeFloats * kLmWarps;

// Append one 16-bit word per renormalizing lane, in lane order (encoder).
__device__ __forceinline__ void lm_put_state(uint32_t& x, const lm_freq_t& F, int v, bool active, uint8_t* words,
                                             uint32_t& len, unsigned below) {
  const bool emit = active && x >= (F.f[v] << 17);
  const unsigned mask = __ballot_sync(0xffffffffu, emit);
  if (emit) {
    put16(words + 2 * (len + __popc(mask & below)), uint16_t(x));
    x >>= 16;
  }
  len += __popc(mask);
  if (active) x = ((x / F.f[v]) << kLmProbBits) + x % F.f[v] + F.cum[v];
}

// Decode one symbol per active lane and take this step's words (decoder).
__device__ __forceinline__ int lm_get_symbol(uint32_t& x, const lm_freq_t& F, bool active, const uint8_t* words,
                                             int64_t& ptr, unsigned above, int& bad) {
  int v = 0;
  if (active) {
    const uint32_t slot = x & (kLmProbTotal - 1);
    v = slot < F.cum[1] ? 0 : slot < F.cum[2] ? 1 : 2;
    x = F.f[v] * (x >> kLmProbBits) + slot - F.cum[v];
  }
  const bool need = active && x < kLmLower;
  const unsigned mask = __ballot_sync(0xffffffffu, need);
  const int64_t at = ptr - 1 - __popc(mask & above);
  if (need) {
    if (at >= 0) x = (x << 16) | get16(words + 2 * at);
    else bad = 1;
  }
  ptr -= __popc(mask);
  return v;
}

// One warp per stream (grid-stride over streams).  sizes[s] = stream bytes, or
// PG_ERR_ARG for a symbol above 2 or a symbol count that does not match.
__global__ void __launch_bounds__(kLmThreads)
lm_encode_kernel(const uint16_t* __restrict__ P, uint64_t hash, const lm_block_t* __restrict__ blocks, int nstreams,
                 const uint8_t* __restrict__ symbols, const int64_t* __restrict__ offsets, uint8_t* __restrict__ out,
                 const int64_t* __restrict__ out_offsets, int64_t* __restrict__ sizes, const dev_tables_t T) {
  extern __shared__ __align__(16) unsigned char lm_smem_raw[];
  lm_tables& S = *reinterpret_cast<lm_tables*>(lm_smem_raw);
  lm_build_tables(S, P, threadIdx.x, blockDim.x);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* node = reinterpret_cast<float*>(lm_smem_raw + sizeof(lm_tables)) + kLmNodeFloats * warp + lane;
  const unsigned below = (1u << lane) - 1;
  for (int s = blockIdx.x * kLmWarps + warp; s < nstreams; s += gridDim.x * kLmWarps) {
    const lm_block_t B = blocks[s];
    const int64_t n = B.nodes;
    uint8_t* base = out + out_offsets[s];
    if (offsets[s + 1] - offsets[s] != 256 * n) {
      if (lane == 0) sizes[s] = PG_ERR_ARG;
      continue;
    }
    const uint8_t* sym0 = symbols + offsets[s];
    uint8_t* words = base + kLmStreamHeader;
    uint32_t x = kLmLower;
    uint32_t len = 0;
    int bad = 0;
    const int64_t rounds = (n + 31) / 32;
    for (int64_t round = rounds - 1; round >= 0; round--) {
      const int64_t i = 32 * round + lane;
      const bool active = i < n;
      uint8_t feats[36];
      const int nf = active ? lm_load_node(B, i, T, feats) : 0;
      lm_node_store(S, feats, nf, node);
      const uint8_t* sym = sym0 + 256 * (active ? i : 0);
      for (int st = 127; st >= 0; st--) {
        lm_freq_t FA = {}, FB = {};
        int vA = 0, vB = 0;
        if (active) {
          int uA[4], uB[4];
          lm_context_clamped(sym, st, uA);
          lm_context_clamped(sym, st + 128, uB);
          float zA[3], zB[3];
          lm_logits2(S, node, st, uA, uB, zA, zB);
          FA = lm_freqs(zA);
          FB = lm_freqs(zB);
          vA = sym[st];
          vB = sym[st + 128];
          if (vA > 2) { bad = 1; vA = 0; }
          if (vB > 2) { bad = 1; vB = 0; }
        }
        // the decoder takes s then s + 128, so the encoder puts s + 128 first
        lm_put_state(x, FB, vB, active, words, len, below);
        lm_put_state(x, FA, vA, active, words, len, below);
      }
    }
    put32(base + 20 + 4 * lane, x);
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
      put32(base, kLmVersion);
      put32(base + 4, uint32_t(hash));
      put32(base + 8, uint32_t(hash >> 32));
      put32(base + 12, uint32_t(n));
      put32(base + 16, len);
      sizes[s] = bad ? PG_ERR_ARG : kLmStreamHeader + 2 * int64_t(len);
    }
  }
}

// status[s] = symbols decoded, or PG_ERR_FORMAT / PG_ERR_CAPACITY.  Version-2
// streams are left to the format-2 decoder (and streams too short to carry a
// version, which it rejects).
__global__ void __launch_bounds__(kLmThreads)
lm_decode_kernel(const uint16_t* __restrict__ P, uint64_t hash, const lm_block_t* __restrict__ blocks, int nstreams,
                 const uint8_t* __restrict__ in, const int64_t* __restrict__ in_offsets,
                 const int64_t* __restrict__ in_sizes, uint8_t* __restrict__ symbols,
                 const int64_t* __restrict__ sym_offsets, const int64_t* __restrict__ sym_caps,
                 int64_t* __restrict__ status, const dev_tables_t T) {
  extern __shared__ __align__(16) unsigned char lm_smem_raw[];
  lm_tables& S = *reinterpret_cast<lm_tables*>(lm_smem_raw);
  lm_build_tables(S, P, threadIdx.x, blockDim.x);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* node = reinterpret_cast<float*>(lm_smem_raw + sizeof(lm_tables)) + kLmNodeFloats * warp + lane;
  const unsigned above = lane == 31 ? 0u : ~0u << (lane + 1);
  for (int s = blockIdx.x * kLmWarps + warp; s < nstreams; s += gridDim.x * kLmWarps) {
    const lm_block_t B = blocks[s];
    const int64_t n = B.nodes;
    const uint8_t* base = in + in_offsets[s];
    const int64_t size = in_sizes[s];
    if (size < 4) continue;
    const uint32_t version = get32(base);
    if (version == 2) continue;
    const uint64_t h = uint64_t(get32(base + 4)) | uint64_t(get32(base + 8)) << 32;
    const uint32_t len = size >= kLmStreamHeader ? get32(base + 16) : 0;
    if (version != kLmVersion || size < kLmStreamHeader || h != hash || get32(base + 12) != uint64_t(n) ||
        int64_t(len) * 2 + kLmStreamHeader != size) {
      if (lane == 0) status[s] = PG_ERR_FORMAT;
      continue;
    }
    if (sym_caps[s] < 256 * n) {
      if (lane == 0) status[s] = PG_ERR_CAPACITY;
      continue;
    }
    const uint8_t* words = base + kLmStreamHeader;
    uint8_t* out0 = symbols + sym_offsets[s];
    uint32_t x = get32(base + 20 + 4 * lane);
    int64_t ptr = len;  // words [0, ptr) are unread
    int bad = 0;
    const int64_t rounds = (n + 31) / 32;
    for (int64_t round = 0; round < rounds; round++) {
      const int64_t i = 32 * round + lane;
      const bool active = i < n;
      uint8_t feats[36];
      const int nf = active ? lm_load_node(B, i, T, feats) : 0;
      lm_node_store(S, feats, nf, node);
      uint8_t* sym = out0 + 256 * (active ? i : 0);
      for (int st = 0; st < 128; st++) {
        lm_freq_t FA = {}, FB = {};
        if (active) {
          int uA[4], uB[4];
          lm_context_clamped(sym, st, uA);
          lm_context_clamped(sym, st + 128, uB);
          float zA[3], zB[3];
          lm_logits2(S, node, st, uA, uB, zA, zB);
          FA = lm_freqs(zA);
          FB = lm_freqs(zB);
        }
        const int vA = lm_get_symbol(x, FA, active, words, ptr, above, bad);
        const int vB = lm_get_symbol(x, FB, active, words, ptr, above, bad);
        if (active) {
          sym[st] = uint8_t(vA);
          sym[st + 128] = uint8_t(vB);
        }
      }
    }
    // A well-formed stream ends with every word read and every lane back at
    // the encoder's initial state.
    bad |= x != kLmLower;
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) status[s] = (bad || ptr != 0) ? PG_ERR_FORMAT : 256 * n;
  }
}

// Frequencies of given samples (for checking the coding path against the CPU).
__global__ void __launch_bounds__(kLmThreads)
lm_freqs_kernel(const uint16_t* __restrict__ P, const lm_block_t* __restrict__ blocks, int nstreams,
                const uint8_t* __restrict__ symbols, const int64_t* __restrict__ offsets,
                const int64_t* __restrict__ samples, int64_t n, uint32_t* __restrict__ freqs, const dev_tables_t T) {
  extern __shared__ __align__(16) unsigned char lm_smem_raw[];
  lm_tables& S = *reinterpret_cast<lm_tables*>(lm_smem_raw);
  lm_build_tables(S, P, threadIdx.x, blockDim.x);
  __syncthreads();
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t smp = samples[t];
    const int64_t s = smp >> 24, i = (smp >> 8) & 0xffff;
    const int r = int(smp & 255);
    uint32_t* f = freqs + 3 * t;
    if (s < 0 || s >= nstreams || i >= blocks[s].nodes) { f[0] = f[1] = f[2] = 0; continue; }
    uint8_t feats[36];
    const int nf = lm_load_node(blocks[s], i, T, feats);
    float node[kLmHidden];
    lm_node_sum(S, feats, nf, node);
    int u[4];
    lm_context_clamped(symbols + offsets[s] + 256 * i, r, u);
    float z[3];
    lm_logits(S, node, r, u, z);
    const lm_freq_t F = lm_freqs(z);
    f[0] = F.f[0];
    f[1] = F.f[1];
    f[2] = F.f[2];
  }
}

// Keep the smaller of the learned and format-2 streams.
__global__ void lm_choose_kernel(int nstreams, uint8_t* __restrict__ out, const int64_t* __restrict__ out_offsets,
                                 int64_t* __restrict__ sizes, const uint8_t* __restrict__ alt,
                                 const int64_t* __restrict__ alt_offsets, const int64_t* __restrict__ alt_sizes) {
  const int s = blockIdx.x;
  if (s >= nstreams) return;
  const int64_t a = sizes[s], b = alt_sizes[s];
  if (a < 0 || b < 0 || b >= a) return;
  uint8_t* d = out + out_offsets[s];
  const uint8_t* src = alt + alt_offsets[s];
  for (int64_t k = threadIdx.x; k < b; k += blockDim.x) d[k] = src[k];
  if (threadIdx.x == 0) sizes[s] = b;
}

// ---------------------------------------------------------------------------
// Training

constexpr int kGradThreads = 128;
constexpr int kMaxFeats = 48;  // 36 stones + 4 rotation + 8 neighbours

struct lm_grad_smem {
  float w1[kLmIn * kW1Pad];
  float w2[kLmHidden][kLmHidden];
  float w3[kLmHidden][4];
  float b1[kLmHidden], b2[kLmHidden], b3[4];
  float h1[kGradThreads][kW1Pad];   // relu(a1)
  float d2[kGradThreads][kW1Pad];   // dL/da2
  float x[kGradThreads][kW1Pad];    // relu(a2), then dL/da1
  float dz[kGradThreads][4];
  float loss[kGradThreads];
  uint8_t feats[kGradThreads][kMaxFeats];
  int nfeat[kGradThreads];
  float gw1[kLmIn][kLmHidden];
};

__device__ __forceinline__ float bf16_of(const float* p, int i) { return bf16_value(bf16_round(p[i])); }

__global__ void __launch_bounds__(kGradThreads)
lm_grad_kernel(const float* __restrict__ params, const lm_block_t* __restrict__ blocks, int nstreams,
               const uint8_t* __restrict__ symbols, const int64_t* __restrict__ offsets,
               const int64_t* __restrict__ samples, int64_t n, float* __restrict__ partial, const dev_tables_t T) {
  extern __shared__ __align__(16) unsigned char lm_smem_raw[];
  lm_grad_smem& G = *reinterpret_cast<lm_grad_smem*>(lm_smem_raw);
  const int tid = threadIdx.x;
  for (int i = tid; i < kLmIn * kLmHidden; i += kGradThreads) {
    G.w1[(i / kLmHidden) * kW1Pad + i % kLmHidden] = bf16_of(params, kLmW1 + i);
    G.gw1[i / kLmHidden][i % kLmHidden] = 0.f;
  }
  for (int i = tid; i < kLmHidden * kLmHidden; i += kGradThreads) G.w2[i / kLmHidden][i % kLmHidden] = bf16_of(params, kLmW2 + i);
  if (tid < kLmHidden) {
    G.b1[tid] = bf16_of(params, kLmB1 + tid);
    G.b2[tid] = bf16_of(params, kLmB2 + tid);
    for (int c = 0; c < 3; c++) G.w3[tid][c] = bf16_of(params, kLmW3 + tid * kLmOut + c);
    G.w3[tid][3] = 0.f;
  }
  if (tid < 3) G.b3[tid] = bf16_of(params, kLmB3 + tid);
  // Per-thread gradient accumulators: dW2 rows k = tid / 2, columns 32 (tid & 1) + 0..31;
  // b1/b2 for tid < 64; W3 row tid for tid < 64; b3 for 64 <= tid < 67.
  float gw2[32];
#pragma unroll
  for (int j = 0; j < 32; j++) gw2[j] = 0.f;
  float gb1 = 0.f, gb2 = 0.f, gw3[3] = {0.f, 0.f, 0.f}, gb3 = 0.f, gloss = 0.f;
  __syncthreads();
  const int64_t tiles = (n + kGradThreads - 1) / kGradThreads;
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    // Forward and local backward, one sample per thread
    const int64_t t = tile * kGradThreads + tid;
    int nf = 0, y = -1;
    if (t < n) {
      const int64_t smp = samples[t];
      const int64_t s = smp >> 24, i = (smp >> 8) & 0xffff;
      const int r = int(smp & 255);
      if (s >= 0 && s < nstreams && i < blocks[s].nodes) {
        const uint8_t* sym = symbols + offsets[s] + 256 * i;
        if (sym[r] <= 2) {
          y = sym[r];
          nf = lm_load_node(blocks[s], i, T, G.feats[tid]);
          for (int q = 0; q < 4; q++) G.feats[tid][nf++] = uint8_t(kLmRot + 4 * q + ((r >> (2 * q)) & 3));
          for (int nb = 0; nb < 8; nb++) {
            const int a = lm_neighbour(r, nb);
            G.feats[tid][nf++] = uint8_t(kLmCtx + 4 * nb + (lm_before(a, r) ? (sym[a] & 3) : 3));
          }
        }
      }
    }
    G.nfeat[tid] = nf;
    float a2[kLmHidden];
    float z[3] = {0.f, 0.f, 0.f};
    if (y >= 0) {
      for (int k = 0; k < kLmHidden; k++) {
        float a = G.b1[k];
        for (int f = 0; f < nf; f++) a += G.w1[G.feats[tid][f] * kW1Pad + k];
        G.h1[tid][k] = relu(a);
      }
#pragma unroll
      for (int j = 0; j < kLmHidden; j++) a2[j] = G.b2[j];
      for (int k = 0; k < kLmHidden; k++) {
        const float h = G.h1[tid][k];
#pragma unroll
        for (int j = 0; j < kLmHidden; j++) a2[j] = fmaf(G.w2[k][j], h, a2[j]);
      }
      z[0] = G.b3[0];
      z[1] = G.b3[1];
      z[2] = G.b3[2];
#pragma unroll
      for (int j = 0; j < kLmHidden; j++) {
        const float h = relu(a2[j]);
        G.x[tid][j] = h;
        z[0] = fmaf(G.w3[j][0], h, z[0]);
        z[1] = fmaf(G.w3[j][1], h, z[1]);
        z[2] = fmaf(G.w3[j][2], h, z[2]);
      }
      const float m = fmaxf(z[0], fmaxf(z[1], z[2]));
      float e[3], es = 0.f;
      for (int c = 0; c < 3; c++) { e[c] = expf(z[c] - m); es += e[c]; }
      G.loss[tid] = (logf(es) - (z[y] - m)) * 1.44269504f;  // bits
      float dzc[3];
      for (int c = 0; c < 3; c++) {
        dzc[c] = e[c] / es - (c == y ? 1.f : 0.f);
        G.dz[tid][c] = dzc[c];
      }
#pragma unroll
      for (int j = 0; j < kLmHidden; j++)
        G.d2[tid][j] = a2[j] > 0.f ? G.w3[j][0] * dzc[0] + G.w3[j][1] * dzc[1] + G.w3[j][2] * dzc[2] : 0.f;
    } else {
      for (int k = 0; k < kLmHidden; k++) { G.h1[tid][k] = 0.f; G.x[tid][k] = 0.f; G.d2[tid][k] = 0.f; }
      for (int c = 0; c < 3; c++) G.dz[tid][c] = 0.f;
      G.loss[tid] = 0.f;
    }
    __syncthreads();
    // W3, b3 and the loss (fixed sample order)
    if (tid < kLmHidden) {
      for (int q = 0; q < kGradThreads; q++) {
        const float h = G.x[q][tid];
        gw3[0] += h * G.dz[q][0];
        gw3[1] += h * G.dz[q][1];
        gw3[2] += h * G.dz[q][2];
      }
    } else if (tid < kLmHidden + 3) {
      for (int q = 0; q < kGradThreads; q++) gb3 += G.dz[q][tid - kLmHidden];
    } else if (tid == kLmHidden + 3) {
      for (int q = 0; q < kGradThreads; q++) gloss += G.loss[q];
    }
    __syncthreads();
    // dL/da1 into x
    if (y >= 0) {
      for (int k = 0; k < kLmHidden; k++) {
        float d = 0.f;
        if (G.h1[tid][k] > 0.f)
          for (int j = 0; j < kLmHidden; j++) d = fmaf(G.w2[k][j], G.d2[tid][j], d);
        G.x[tid][k] = d;
      }
    }
    __syncthreads();
    // W2, b1, b2
    {
      const int k = tid >> 1, j0 = 32 * (tid & 1);
      for (int q = 0; q < kGradThreads; q++) {
        const float h = G.h1[q][k];
#pragma unroll
        for (int j = 0; j < 32; j++) gw2[j] = fmaf(h, G.d2[q][j0 + j], gw2[j]);
      }
      if (tid < kLmHidden) {
        for (int q = 0; q < kGradThreads; q++) { gb1 += G.x[q][tid]; gb2 += G.d2[q][tid]; }
      }
    }
    // W1: thread owns column k for the features of its half
    {
      const int k = tid & (kLmHidden - 1), lo = tid < kLmHidden ? 0 : kLmIn / 2, hi = lo + kLmIn / 2;
      for (int q = 0; q < kGradThreads; q++) {
        const float d = G.x[q][k];
        for (int f = 0; f < G.nfeat[q]; f++) {
          const int ft = G.feats[q][f];
          if (ft >= lo && ft < hi) G.gw1[ft][k] += d;
        }
      }
    }
    __syncthreads();
  }
  // Partial sums of this CTA
  float* out = partial + int64_t(blockIdx.x) * (kLmParams + 1);
  for (int i = tid; i < kLmIn * kLmHidden; i += kGradThreads) out[kLmW1 + i] = G.gw1[i / kLmHidden][i % kLmHidden];
  {
    const int k = tid >> 1, j0 = 32 * (tid & 1);
    for (int j = 0; j < 32; j++) out[kLmW2 + k * kLmHidden + j0 + j] = gw2[j];
  }
  if (tid < kLmHidden) {
    out[kLmB1 + tid] = gb1;
    out[kLmB2 + tid] = gb2;
    for (int c = 0; c < 3; c++) out[kLmW3 + tid * kLmOut + c] = gw3[c];
  } else if (tid < kLmHidden + 3) {
    out[kLmB3 + tid - kLmHidden] = gb3;
  } else if (tid == kLmHidden + 3) {
    out[kLmParams] = gloss;
  }
}

__global__ void lm_reduce_kernel(const float* __restrict__ partial, int nparts, float* __restrict__ grad,
                                 float* __restrict__ loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > kLmParams) return;
  float s = 0.f;
  for (int c = 0; c < nparts; c++) s += partial[int64_t(c) * (kLmParams + 1) + p];
  if (p < kLmParams) grad[p] = s;
  else if (loss) *loss = s;
}

__global__ void lm_adam_kernel(float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
                               const float* __restrict__ grad, float lr, float scale, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kLmParams) return;
  const float g = grad[p] * scale;
  const float mm = 0.9f * m[p] + 0.1f * g;
  const float vv = 0.999f * v[p] + 0.001f * g * g;
  m[p] = mm;
  v[p] = vv;
  params[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + 1e-8f);
}

__device__ __forceinline__ uint64_t splitmix(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void lm_samples_kernel(const int64_t* __restrict__ cand, int64_t ncand, uint64_t seed, int64_t step,
                                  int64_t batch, int64_t* __restrict__ out) {
  const int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (k >= batch) return;
  const uint64_t h = splitmix(seed ^ splitmix(uint64_t(step) * 0x100000001b3ull + uint64_t(k)));
  const int64_t c = cand[(h & 0xffffffffffull) % uint64_t(ncand)];
  out[k] = (c << 8) | int64_t(h >> 56);
}

// ---------------------------------------------------------------------------
// Host side

static uint64_t fnv1a(const uint8_t* p, int64_t n) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (int64_t i = 0; i < n; i++) h = (h ^ p[i]) * 0x100000001b3ull;
  return h;
}

static bool check_model(const uint8_t* model, std::string& err) {
  if (!model) { err = "null model"; return false; }
  uint32_t h[3];
  memcpy(h, model, 12);
  if (h[0] != kLmMagic || h[1] != 1 || h[2] != uint32_t(kLmParams)) { err = "not a version-1 PGLM model"; return false; }
  return true;
}

static bool resolve_blocks(const pg_block_ref_t* refs, int n, std::vector<lm_block_t>& out, std::string& err) {
  const auto& T = tables();
  out.resize(n);
  for (int s = 0; s < n; s++) {
    const section_t sec = section_t::from_sig(refs[s].section);
    if (!sec.valid() || sec.sum() > 36) { err = "invalid section in block " + std::to_string(s); return false; }
    lm_block_t& B = out[s];
    B.nodes = 1;
    for (int q = 0; q < 4; q++) {
      const int k = rmin_bucket(sec.c[q][0], sec.c[q][1]);
      const int size = T.rmin_off[k + 1] - T.rmin_off[k];
      const int b = refs[s].block[q];
      if (b < 0 || 8 * b >= size) { err = "block out of range in block " + std::to_string(s); return false; }
      B.qbase[q] = T.rmin_off[k] + 8 * b;
      B.shape[q] = std::min(8, size - 8 * b);
      B.nodes *= B.shape[q];
    }
  }
  return true;
}

struct lm_launch {
  uint16_t* params = nullptr;
  lm_block_t* blocks = nullptr;
  uint64_t hash = 0;
  cudaStream_t stream = nullptr;
  ~lm_launch() {
    if (params) cudaFreeAsync(params, stream);
    if (blocks) cudaFreeAsync(blocks, stream);
  }
};

static int lm_prepare(const uint8_t* model, const pg_block_ref_t* refs, int n, cudaStream_t stream, lm_launch& L,
                      std::vector<lm_block_t>* host_blocks = nullptr) {
  std::string err;
  L.stream = stream;
  if (model) {
    if (!check_model(model, err)) return fail(PG_ERR_FORMAT, err);
    L.hash = fnv1a(model, kLmModelBytes);
    PG_CUDA(cudaMallocAsync(&L.params, 2 * kLmParams, stream));
    PG_CUDA(cudaMemcpyAsync(L.params, model + kLmModelHeader, 2 * kLmParams, cudaMemcpyHostToDevice, stream));
  }
  std::vector<lm_block_t> B;
  if (!resolve_blocks(refs, n, B, err)) return fail(PG_ERR_ARG, err);
  PG_CUDA(cudaMallocAsync(&L.blocks, sizeof(lm_block_t) * std::max(n, 1), stream));
  PG_CUDA(cudaMemcpyAsync(L.blocks, B.data(), sizeof(lm_block_t) * n, cudaMemcpyHostToDevice, stream));
  if (host_blocks) *host_blocks = std::move(B);
  return PG_OK;
}

template<class K> static int lm_smem_opt_in(K kernel, size_t bytes) {
  PG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
  return PG_OK;
}

static int lm_grid(int nstreams) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return std::max(1, std::min((nstreams + kLmWarps - 1) / kLmWarps, 4 * sms));
}

}  // namespace pg

using namespace pg;

extern "C" int64_t pg_learned_model_bytes(void) { return kLmModelBytes; }

extern "C" int64_t pg_rans_learned_bound(int64_t nodes) {
  if (nodes < 0 || nodes > (int64_t(1) << 32)) return PG_ERR_ARG;
  return std::max<int64_t>(kLmStreamHeader + 2 * 256 * nodes, rans_stream_bound(256 * nodes));
}

extern "C" int pg_learned_export(const float* params, uint8_t* model) {
  if (!params || !model) return fail(PG_ERR_ARG, "null argument");
  const uint32_t h[3] = {kLmMagic, 1u, uint32_t(kLmParams)};
  memcpy(model, h, 12);
  for (int i = 0; i < kLmParams; i++) {
    if (!std::isfinite(params[i])) return fail(PG_ERR_ARG, "non-finite parameter " + std::to_string(i));
    const uint16_t b = bf16_round(params[i]);
    model[kLmModelHeader + 2 * i] = uint8_t(b);
    model[kLmModelHeader + 2 * i + 1] = uint8_t(b >> 8);
  }
  return PG_OK;
}

extern "C" int pg_rans_learned_encode(const uint8_t* model, const pg_block_ref_t* blocks, int nstreams,
                                      const uint8_t* symbols, const int64_t* offsets, uint8_t* out,
                                      const int64_t* out_offsets, int64_t* sizes, void* stream) {
  if (nstreams < 0 || (nstreams && !blocks)) return fail(PG_ERR_ARG, "bad stream list");
  if (!nstreams) return PG_OK;
  const cudaStream_t st = (cudaStream_t)stream;
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  lm_launch L;
  std::vector<lm_block_t> hb;
  if (int rc = lm_prepare(model, blocks, nstreams, st, L, &hb)) return rc;
  if (int rc = lm_smem_opt_in(lm_encode_kernel, kLmCodeSmem)) return rc;
  lm_encode_kernel<<<lm_grid(nstreams), kLmThreads, kLmCodeSmem, st>>>(L.params, L.hash, L.blocks, nstreams,
                                                                              symbols, offsets, out, out_offsets,
                                                                              sizes, *T);
  PG_CUDA(cudaGetLastError());
  // Format-2 streams of the same symbols; the smaller one is kept
  // alt_off[s] = slot of stream s; alt_off[nstreams + s] = its symbol count
  std::vector<int64_t> alt_off(2 * nstreams);
  int64_t total = 0;
  for (int s = 0; s < nstreams; s++) {
    alt_off[s] = total;
    alt_off[nstreams + s] = 256 * hb[s].nodes;
    total += (rans_stream_bound(256 * hb[s].nodes) + 15) & ~15;
  }
  // Scratch for the format-2 streams
  stream_scratch X(st);
  uint8_t* alt = nullptr;
  int64_t *alt_off_d = nullptr, *alt_sizes = nullptr;
  PG_CUDA(X.alloc(&alt, std::max<int64_t>(total, 16)));
  PG_CUDA(X.alloc(&alt_off_d, sizeof(int64_t) * 2 * nstreams));
  PG_CUDA(X.alloc(&alt_sizes, sizeof(int64_t) * nstreams));
  PG_CUDA(cudaMemcpyAsync(alt_off_d, alt_off.data(), sizeof(int64_t) * 2 * nstreams, cudaMemcpyHostToDevice, st));
  if (int rc = launch_rans_encode(symbols, offsets, nstreams, alt, alt_off_d, alt_sizes, alt_off_d + nstreams, st))
    return rc;
  lm_choose_kernel<<<nstreams, 256, 0, st>>>(nstreams, out, out_offsets, sizes, alt, alt_off_d, alt_sizes);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

extern "C" int pg_rans_learned_decode(const uint8_t* model, const pg_block_ref_t* blocks, int nstreams,
                                      const uint8_t* in, const int64_t* in_offsets, const int64_t* in_sizes,
                                      uint8_t* symbols, const int64_t* sym_offsets, const int64_t* sym_caps,
                                      int64_t* status, void* stream) {
  if (nstreams < 0 || (nstreams && !blocks)) return fail(PG_ERR_ARG, "bad stream list");
  if (!nstreams) return PG_OK;
  const cudaStream_t st = (cudaStream_t)stream;
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  lm_launch L;
  if (int rc = lm_prepare(model, blocks, nstreams, st, L)) return rc;
  if (int rc = launch_rans_decode(in, in_offsets, in_sizes, nstreams, symbols, sym_offsets, sym_caps, status, 1, st))
    return rc;
  if (int rc = lm_smem_opt_in(lm_decode_kernel, kLmCodeSmem)) return rc;
  lm_decode_kernel<<<lm_grid(nstreams), kLmThreads, kLmCodeSmem, st>>>(L.params, L.hash, L.blocks, nstreams, in,
                                                                              in_offsets, in_sizes, symbols,
                                                                              sym_offsets, sym_caps, status, *T);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

extern "C" int pg_learned_freqs(const uint8_t* model, const pg_block_ref_t* blocks, int nstreams,
                                const uint8_t* symbols, const int64_t* offsets, const int64_t* samples, int64_t n,
                                uint32_t* freqs, void* stream) {
  if (nstreams < 0 || n < 0 || (nstreams && !blocks)) return fail(PG_ERR_ARG, "bad arguments");
  if (!n) return PG_OK;
  const cudaStream_t st = (cudaStream_t)stream;
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  lm_launch L;
  if (int rc = lm_prepare(model, blocks, nstreams, st, L)) return rc;
  if (int rc = lm_smem_opt_in(lm_freqs_kernel, sizeof(lm_tables))) return rc;
  const int grid = int(std::min<int64_t>((n + kLmThreads - 1) / kLmThreads, 1024));
  lm_freqs_kernel<<<grid, kLmThreads, sizeof(lm_tables), st>>>(L.params, L.blocks, nstreams, symbols, offsets, samples,
                                                                n, freqs, *T);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

extern "C" int pg_learned_samples(const int64_t* candidates, int64_t ncand, uint64_t seed, int64_t step,
                                  int64_t batch, int64_t* samples, void* stream) {
  if (ncand <= 0 || batch < 0 || step < 0) return fail(PG_ERR_ARG, "bad arguments");
  if (!batch) return PG_OK;
  lm_samples_kernel<<<unsigned((batch + 255) / 256), 256, 0, (cudaStream_t)stream>>>(candidates, ncand, seed, step,
                                                                                    batch, samples);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

extern "C" int pg_learned_grad(const float* params, const pg_block_ref_t* blocks, int nstreams, const uint8_t* symbols,
                               const int64_t* offsets, const int64_t* samples, int64_t n, float* grad, float* loss,
                               void* stream) {
  if (nstreams < 0 || n < 0 || (nstreams && !blocks) || !params || !grad) return fail(PG_ERR_ARG, "bad arguments");
  const cudaStream_t st = (cudaStream_t)stream;
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  lm_launch L;
  if (int rc = lm_prepare(nullptr, blocks, nstreams, st, L)) return rc;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = int(std::max<int64_t>(1, std::min<int64_t>((n + kGradThreads - 1) / kGradThreads, sms)));
  stream_scratch X(st);
  float* partial = nullptr;
  PG_CUDA(X.alloc(&partial, sizeof(float) * grid * (kLmParams + 1)));
  if (int rc = lm_smem_opt_in(lm_grad_kernel, sizeof(lm_grad_smem))) return rc;
  lm_grad_kernel<<<grid, kGradThreads, sizeof(lm_grad_smem), st>>>(params, L.blocks, nstreams, symbols, offsets,
                                                                    samples, n, partial, *T);
  PG_CUDA(cudaGetLastError());
  lm_reduce_kernel<<<(kLmParams + 1 + 255) / 256, 256, 0, st>>>(partial, grid, grad, loss);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

extern "C" int pg_learned_adam(float* params, float* m, float* v, const float* grad, int64_t step, float lr,
                               float scale, void* stream) {
  if (!params || !m || !v || !grad || step < 1) return fail(PG_ERR_ARG, "bad arguments");
  const float c1 = 1.f - std::pow(0.9f, float(step)), c2 = 1.f - std::pow(0.999f, float(step));
  lm_adam_kernel<<<(kLmParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, m, v, grad, lr, scale, c1, c2);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}
