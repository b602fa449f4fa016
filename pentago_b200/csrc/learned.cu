// Learned-model rANS for solved blocks (stream format version 3) and the
// kernels that train its network.  The model and the exact arithmetic of the
// coding path are specified in learned.cuh.
//
// Coder layout: one warp per stream; lane l codes the run of nodes l R ..
// l R + R - 1 (R = ceil(n / 32)), node l R + k in round k, its own rANS
// state walking the steps (round, rotation) in order.  The encoder runs the
// steps backward; at each step the lanes that renormalize append one 16-bit
// word each, in lane order, to the stream's shared word array, so the decoder
// (running forward) finds the words of its step as the last unread ones.
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
constexpr int kLmCtxRows = kLmIn - kLmRot;   // W1 rows 72..123: the rotation, neighbour and previous-node features

// Coding tables in shared memory.  The tensor cores' B operands are stored
// transposed, one row of 64 bf16 (8 chunks of 16 bytes) per output unit:
// w1t row k holds W1[72 + 8 c .. 72 + 8 c + 7][k] in chunk c (c < 6), w2t
// row j holds W2[8 c .. 8 c + 7][j], chunk c at c ^ (row & 7) so that the
// eight rows an ldmatrix phase reads fall in different banks.
struct lm_tables {
  uint4 w1t[kLmHidden][8];
  uint4 w2t[kLmHidden][8];
  float b1[kLmHidden], b2[kLmHidden];
  float w3[kLmHidden][4];        // [j][c]
  float b3[4];
};

__device__ __forceinline__ int swz(int row, int chunk) { return chunk ^ (row & 7); }

__device__ void lm_build_tables(lm_tables& S, const uint16_t* __restrict__ P, int tid, int nt) {
  auto w = [&](int i) { return bf16_value(P[i]); };
  for (int i = tid; i < kLmHidden * 8; i += nt) {
    const int j = i >> 3, c = i & 7;
    uint32_t v[4], u[4];
    for (int e = 0; e < 4; e++) {
      const int f = 8 * c + 2 * e;   // feature rows 72 + f, 72 + f + 1 (zero past the 48)
      u[e] = f < kLmCtxRows ? uint32_t(P[kLmW1 + (kLmRot + f) * kLmHidden + j]) |
                                  uint32_t(P[kLmW1 + (kLmRot + f + 1) * kLmHidden + j]) << 16
                            : 0u;
      v[e] = uint32_t(P[kLmW2 + (8 * c + 2 * e) * kLmHidden + j]) |
             uint32_t(P[kLmW2 + (8 * c + 2 * e + 1) * kLmHidden + j]) << 16;
    }
    S.w1t[j][swz(j, c)] = make_uint4(u[0], u[1], u[2], u[3]);
    S.w2t[j][swz(j, c)] = make_uint4(v[0], v[1], v[2], v[3]);
  }
  for (int i = tid; i < kLmHidden; i += nt) {
    S.b1[i] = w(kLmB1 + i);
    S.b2[i] = w(kLmB2 + i);
    for (int c = 0; c < 3; c++) S.w3[i][c] = w(kLmW3 + i * kLmOut + c);
    S.w3[i][3] = 0.f;
  }
  if (tid < 3) S.b3[tid] = w(kLmB3 + tid);
  if (tid == 3) S.b3[3] = 0.f;
}

// Element k of row t of a transposed table (bf16 -> float).
__device__ __forceinline__ float lm_tab(const uint4 (*tab)[8], int row, int k) {
  const uint4 ch = tab[row][swz(row, k >> 3)];
  const uint32_t pr = (k & 7) < 2 ? ch.x : (k & 7) < 4 ? ch.y : (k & 7) < 6 ? ch.z : ch.w;
  return f_bits(k & 1 ? pr & 0xffff0000u : pr << 16);
}

// node[k] = b1[k] + stone rows, ascending (registers of one thread); the
// stone rows are read from the model (bf16, global memory: a lane reads them
// once per node).
__device__ __forceinline__ void lm_node_sum(const lm_tables& S, const uint16_t* __restrict__ P, const uint8_t* feats,
                                            int nf, float* node) {
#pragma unroll
  for (int k = 0; k < kLmHidden; k++) node[k] = S.b1[k];
  for (int i = 0; i < nf; i++) {
    const uint4* row = reinterpret_cast<const uint4*>(P + kLmW1 + feats[i] * kLmHidden);
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const uint4 v = ldg(row + c);
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int e = 0; e < 4; e++) {
        node[8 * c + 2 * e] = f_add(node[8 * c + 2 * e], f_bits(w[e] << 16));
        node[8 * c + 2 * e + 1] = f_add(node[8 * c + 2 * e + 1], f_bits(w[e] & 0xffff0000u));
      }
    }
  }
}

// The 4 rotation, 8 neighbour and 1 previous-node features of symbol r
// (indices into W1 rows 72..123): 4 q + i_q, then 16 + 4 n + v_n with
// u[q] = v_2q + 4 v_2q+1, then 48 + the previous node's symbol (3: none).
__device__ __forceinline__ void lm_ctx_features(int r, const int* u, int prev, int* f) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    f[q] = 4 * q + ((r >> (2 * q)) & 3);
    f[4 + 2 * q] = 16 + 8 * q + (u[q] & 3);
    f[5 + 2 * q] = 20 + 8 * q + (u[q] >> 2);
  }
  f[12] = kLmPrev - kLmRot + prev;
}

// Logits of one symbol, one thread (the frequency check kernel): S1 and C by
// fp32 chains, exact on a model whose grid columns are on their grids, and layer 3 in the order of
// learned.cuh.
__device__ __forceinline__ void lm_logits(const lm_tables& S, const float* node, int r, const int* u, int prev,
                                          float* z) {
  int f[13];
  lm_ctx_features(r, u, prev, f);
  float hq[kLmHidden];
  for (int k = 0; k < kLmHidden; k++) {
    float s1 = 0.f;
    for (int i = 0; i < 13; i++) s1 = f_add(s1, lm_tab(S.w1t, k, f[i]));
    hq[k] = lm_act_q(f_add(node[k], s1));
  }
  float part[4][3];
#pragma unroll
  for (int t = 0; t < 4; t++) part[t][0] = part[t][1] = part[t][2] = 0.f;
  for (int j = 0; j < kLmHidden; j++) {
    float c = 0.f;
    for (int k = 0; k < kLmHidden; k++) c = f_fma(lm_tab(S.w2t, j, k), hq[k], c);
    const float h = relu(f_fma(c, kLmActInv, S.b2[j]));
    const int t = (j >> 1) & 3;
    for (int cc = 0; cc < 3; cc++) part[t][cc] = f_fma(S.w3[j][cc], h, part[t][cc]);
  }
  for (int cc = 0; cc < 3; cc++)
    z[cc] = f_add(S.b3[cc], f_add(f_add(part[0][cc], part[1][cc]), f_add(part[2][cc], part[3][cc])));
}

// Tensor-core pieces (mma.sync m16n8k16, bf16 inputs, fp32 accumulation).
__device__ __forceinline__ void ldsm_x4(uint32_t* r, const void* p) {
  const unsigned a = unsigned(__cvta_generic_to_shared(p));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(a));
}
__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
               "{%8, %9}, {%0, %1, %2, %3};\n"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// out[n] += A x B for the eight n-tiles of a transposed table, k-tile kt.
__device__ __forceinline__ void mma_row(float (*acc)[4], const uint32_t* a, const uint4 (*tab)[8], int kt, int lane) {
#pragma unroll
  for (int np = 0; np < 4; np++) {
    const int row = 16 * np + 8 * (lane >> 4) + (lane & 7), chunk = 2 * kt + ((lane >> 3) & 1);
    uint32_t b[4];
    ldsm_x4(b, &tab[row][swz(row, chunk)]);
    mma_bf16(acc[2 * np], a, b[0], b[1]);
    mma_bf16(acc[2 * np + 1], a, b[2], b[3]);
  }
}

// bf16 1.0 at the element of value v among the pair (base, base + 1).
__device__ __forceinline__ uint32_t onehot2(int v, int base) {
  return v == base ? 0x00003f80u : v == base + 1 ? 0x3f800000u : 0u;
}

// The warp's 64 rows per step: row lane is symbol s of the lane's node, row
// 32 + lane symbol s + 128; tile m holds rows 16 m .. 16 m + 15, and lane
// (g, t) = (lane / 4, lane % 4) holds rows 16 m + g and 16 m + g + 8 of each
// tile, that is the nodes of lanes 16 (m & 1) + 8 h + g (h = 0, 1), and
// columns 8 n + 2 t + e (e = 0, 1) of each n-tile.  lm_nodefrag is the node
// sums at those places (constant over a node's 128 steps).
struct lm_nodefrag {
  float v[2][2][8][2];   // [m & 1][h][n][e]
};

// Chunk kc (hidden units 16 kc .. 16 kc + 15) of the lane's own node sums,
// own[i] for unit 16 kc + i, spread to the warp's fragment places.
__device__ __forceinline__ void lm_node_frag(const float* own, int kc, int lane, lm_nodefrag& F) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int i = 0; i < 16; i++) {
    const int k = 16 * kc + i;
#pragma unroll
    for (int mm = 0; mm < 2; mm++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const float x = __shfl_sync(0xffffffffu, own[i], 16 * mm + 8 * h + g);
        if (((k >> 1) & 3) == t) F.v[mm][h][k >> 3][k & 1] = x;
      }
  }
}

// Logits of the two symbols of step s (rotations s and s + 128) of every
// lane's node.  ctx[0], ctx[1] are the lane's contexts of the two symbols:
// 4 bits u_q = v_2q + 4 v_2q+1 per quadrant q (bits 0-15), the previous
// node's symbol (bits 16-17).  Layer 1's rotation, neighbour and
// previous-node rows and layer 2 run on the tensor cores; layer 1's results
// stay in registers as layer 2's A operand.
__device__ __forceinline__ void lm_step_logits(const lm_tables& S, const lm_nodefrag& N, int lane, int s,
                                               const uint32_t* ctx, float* zA, float* zB) {
  const int g = lane >> 2, t = lane & 3;
  uint32_t cx[2][2][2];   // [m & 1][h][symbol]
#pragma unroll
  for (int mm = 0; mm < 2; mm++)
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int sb = 0; sb < 2; sb++) cx[mm][h][sb] = __shfl_sync(0xffffffffu, ctx[sb], 16 * mm + 8 * h + g);
  // Row lane is in tile lane / 16 (symbol s) and tile 2 + lane / 16 (s + 128),
  // half (lane / 8) & 1 of quad lane & 7.
  const int src = 4 * (lane & 7), mine = lane >> 4, half = (lane >> 3) & 1;
  // Tile m = 2 sb + mm: one tile at a time (the loop over sb is not unrolled,
  // so the tiles' registers are not live together)
#pragma unroll
  for (int mm = 0; mm < 2; mm++) {
#pragma unroll 1
    for (int sb = 0; sb < 2; sb++) {
      const int r = s + 128 * sb;
      // Layer 1 A operand: one-hot features.  k-tile 0 is the rotation
      // (feature 4 q + i_q; the lane's columns 2 t, 2 t + 1 and 8 + 2 t,
      // 9 + 2 t are quadrants t / 2 and 2 + t / 2), the same for every node;
      // k-tiles 1 and 2 are neighbours n = 4 (kt - 1) + t / 2 and n + 2;
      // k-tile 3 is the previous node's symbol (columns 0-3: lanes t < 2).
      const int base = 2 * (t & 1);
      uint32_t a1[4][4];
      a1[0][0] = a1[0][1] = onehot2((r >> (2 * (t >> 1))) & 3, base);
      a1[0][2] = a1[0][3] = onehot2((r >> (2 * (2 + (t >> 1)))) & 3, base);
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const uint32_t u = sb ? cx[mm][h][1] : cx[mm][h][0];
#pragma unroll
        for (int kt = 1; kt < 3; kt++) {
          const int n0 = 4 * (kt - 1) + (t >> 1);
          a1[kt][h] = onehot2(int(u >> (2 * n0)) & 3, base);
          a1[kt][2 + h] = onehot2(int(u >> (2 * (n0 + 2))) & 3, base);
        }
        a1[3][h] = t < 2 ? onehot2(int(u >> 16) & 3, 2 * t) : 0u;
        a1[3][2 + h] = 0u;
      }
      float acc[8][4];
#pragma unroll
      for (int n = 0; n < 8; n++) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
#pragma unroll
      for (int kt = 0; kt < 4; kt++) mma_row(acc, a1[kt], S.w1t, kt, lane);
      // a1 = node + S1, quantized: n-tiles 2 k and 2 k + 1 of layer 1 are the
      // k-tile k of layer 2's A operand
      uint32_t a2[4][4];
#pragma unroll
      for (int n = 0; n < 8; n++) {
        const float q00 = lm_act_q(f_add(N.v[mm][0][n][0], acc[n][0]));
        const float q01 = lm_act_q(f_add(N.v[mm][0][n][1], acc[n][1]));
        const float q10 = lm_act_q(f_add(N.v[mm][1][n][0], acc[n][2]));
        const float q11 = lm_act_q(f_add(N.v[mm][1][n][1], acc[n][3]));
        a2[n >> 1][2 * (n & 1)] = __byte_perm(f_raw(q00), f_raw(q01), 0x7632);
        a2[n >> 1][2 * (n & 1) + 1] = __byte_perm(f_raw(q10), f_raw(q11), 0x7632);
      }
#pragma unroll
      for (int n = 0; n < 8; n++) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
#pragma unroll
      for (int kt = 0; kt < 4; kt++) mma_row(acc, a2[kt], S.w2t, kt, lane);
      // Layer 3 on the accumulators: the lane's columns make its P_t
      float p0[3] = {0.f, 0.f, 0.f}, p1[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int n = 0; n < 8; n++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int j = 8 * n + 2 * t + e;
          const float4 w3 = *reinterpret_cast<const float4*>(S.w3[j]);
          const float b2 = S.b2[j];
          const float h0 = relu(f_fma(acc[n][e], kLmActInv, b2)), h1 = relu(f_fma(acc[n][2 + e], kLmActInv, b2));
          p0[0] = f_fma(w3.x, h0, p0[0]);
          p0[1] = f_fma(w3.y, h0, p0[1]);
          p0[2] = f_fma(w3.z, h0, p0[2]);
          p1[0] = f_fma(w3.x, h1, p1[0]);
          p1[1] = f_fma(w3.y, h1, p1[1]);
          p1[2] = f_fma(w3.z, h1, p1[2]);
        }
#pragma unroll
      for (int c = 0; c < 3; c++) {
        // (P0 + P1) + (P2 + P3); addition commutes, so every lane of the
        // quad ends with the same bits; then to the row's own lane
        float q0 = f_add(p0[c], __shfl_xor_sync(0xffffffffu, p0[c], 1));
        float q1 = f_add(p1[c], __shfl_xor_sync(0xffffffffu, p1[c], 1));
        q0 = f_add(S.b3[c], f_add(q0, __shfl_xor_sync(0xffffffffu, q0, 2)));
        q1 = f_add(S.b3[c], f_add(q1, __shfl_xor_sync(0xffffffffu, q1, 2)));
        const float v0 = __shfl_sync(0xffffffffu, q0, src), v1 = __shfl_sync(0xffffffffu, q1, src);
        if (mm == mine) {
          const float v = half ? v1 : v0;
          if (sb) zB[c] = v;
          else zA[c] = v;
        }
      }
    }
  }
}

// Neighbour context of symbol r from the node's symbols (those of earlier
// steps; later ones read as 3), packed as 4 bits per quadrant.
__device__ __forceinline__ uint32_t lm_context_packed(const uint8_t* sym, int r) {
  uint32_t p = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int a = lm_neighbour(r, 2 * q), b = lm_neighbour(r, 2 * q + 1);
    const int va = lm_before(a, r) ? (sym[a] & 3) : 3, vb = lm_before(b, r) ? (sym[b] & 3) : 3;
    p |= uint32_t(va + 4 * vb) << (4 * q);
  }
  return p;
}
__device__ __forceinline__ void lm_context_clamped(const uint8_t* sym, int r, int* u) {
  const uint32_t p = lm_context_packed(sym, r);
#pragma unroll
  for (int q = 0; q < 4; q++) u[q] = int(p >> (4 * q)) & 15;
}

__device__ __forceinline__ int lm_load_node(const lm_block_t& B, int64_t i, const dev_tables_t& T, uint8_t* feats) {
  uint16_t qid[4];
  lm_node_quadrants(B, i, T.rmin_flat, qid);
  return lm_node_features(qid, T.unpack, feats);
}

// The lane's node: its node sums (b1 + stone rows ascending), 16 units at a
// time, spread to the warp's fragment places.
__device__ __forceinline__ void lm_round_nodes(const lm_tables& S, const uint16_t* __restrict__ P,
                                               const lm_block_t& B, int64_t i, bool active, const dev_tables_t& T,
                                               int lane, lm_nodefrag& N) {
  uint8_t feats[36];
  const int nf = active ? lm_load_node(B, i, T, feats) : 0;
#pragma unroll
  for (int kc = 0; kc < 4; kc++) {
    float own[16];
#pragma unroll
    for (int u = 0; u < 16; u++) own[u] = S.b1[16 * kc + u];
    for (int f = 0; f < nf; f++) {
      const uint4* row = reinterpret_cast<const uint4*>(P + kLmW1 + feats[f] * kLmHidden + 16 * kc);
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const uint4 v = ldg(row + c);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int e = 0; e < 4; e++) {
          own[8 * c + 2 * e] = f_add(own[8 * c + 2 * e], f_bits(w[e] << 16));
          own[8 * c + 2 * e + 1] = f_add(own[8 * c + 2 * e + 1], f_bits(w[e] & 0xffff0000u));
        }
      }
    }
    lm_node_frag(own, kc, lane, N);
  }
}

// A run's previous node (its symbols, 2 bits each, 17 words a lane so that
// lanes reading the same rotation use different banks); 3 for every
// rotation before a run's first node.
constexpr int kLmPrevWords = 17;
__device__ __forceinline__ int lm_prev_sym(const uint32_t* prev, int r) { return int(prev[r >> 4] >> (2 * (r & 15))) & 3; }
__device__ __forceinline__ void lm_prev_none(uint32_t* prev) {
  for (int w = 0; w < 16; w++) prev[w] = 0xffffffffu;
}
__device__ __forceinline__ void lm_prev_from(uint32_t* prev, const uint8_t* sym) {
  for (int w = 0; w < 16; w++) {
    uint32_t v = 0;
    for (int k = 0; k < 16; k++) v |= uint32_t(sym[16 * w + k] & 3) << (2 * k);
    prev[w] = v;
  }
}

__device__ __forceinline__ void put16(uint8_t* p, uint16_t v) { p[0] = uint8_t(v); p[1] = uint8_t(v >> 8); }
__device__ __forceinline__ uint16_t get16(const uint8_t* p) { return uint16_t(p[0] | p[1] << 8); }
__device__ __forceinline__ void put32(uint8_t* p, uint32_t v) { for (int i = 0; i < 4; i++) p[i] = uint8_t(v >> (8 * i)); }
__device__ __forceinline__ uint32_t get32(const uint8_t* p) {
  return uint32_t(p[0]) | uint32_t(p[1]) << 8 | uint32_t(p[2]) << 16 | uint32_t(p[3]) << 24;
}

// Dynamic shared memory of the coding kernels: the tables, then per warp its
// lanes' nodes' symbols (one row of 256 bytes a lane, rows 260 bytes apart
// so that lanes reading the same rotation use different banks), their
// previous nodes' symbols (packed) and, for the decoder, a window of the
// stream's next words.
constexpr int kLmSymRow = 260;
constexpr int kLmWordWin = 1024;   // the decoder's window of upcoming stream words, per warp
constexpr size_t kLmWarpSmem = size_t(32) * kLmSymRow + size_t(32) * 4 * kLmPrevWords + 2 * kLmWordWin;
constexpr size_t kLmCodeSmem = sizeof(lm_tables) + kLmWarpSmem * kLmWarps;
static_assert(sizeof(lm_tables) % 16 == 0 && kLmWarpSmem % 16 == 0, "coding rows stay 16-byte aligned");

// A node's 256 symbols between global memory and its shared-memory row.
__device__ __forceinline__ int lm_row_in(uint8_t* row, const uint8_t* g) {
  int bad = 0;
  if ((reinterpret_cast<uintptr_t>(g) & 3) == 0) {
    for (int w = 0; w < 64; w++) {
      const uint32_t v = reinterpret_cast<const uint32_t*>(g)[w];
      bad |= (v & 0xfcfcfcfcu) != 0 || (v & v >> 1 & 0x01010101u) != 0;   // a byte above 2
      reinterpret_cast<uint32_t*>(row)[w] = v;
    }
  } else {
    for (int k = 0; k < 256; k++) {
      const uint8_t v = g[k];
      bad |= v > 2;
      row[k] = v;
    }
  }
  return bad;
}
__device__ __forceinline__ void lm_row_out(const uint8_t* row, uint8_t* g) {
  if ((reinterpret_cast<uintptr_t>(g) & 3) == 0) {
    for (int w = 0; w < 64; w++) reinterpret_cast<uint32_t*>(g)[w] = reinterpret_cast<const uint32_t*>(row)[w];
  } else {
    for (int k = 0; k < 256; k++) g[k] = row[k];
  }
}

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
// Words [wlo, wlo + kLmWordWin) are also in win.
__device__ __forceinline__ int lm_get_symbol(uint32_t& x, const lm_freq_t& F, bool active, const uint8_t* words,
                                             const uint16_t* win, int64_t wlo, int64_t& ptr, unsigned above,
                                             int& bad) {
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
    if (at >= wlo) x = (x << 16) | win[at - wlo];
    else if (at >= 0) x = (x << 16) | get16(words + 2 * at);
    else bad = 1;
  }
  ptr -= __popc(mask);
  return v;
}

// The next stream of a launch, largest first: streams are handed to warps
// one at a time through a counter, in the order the host sorted them.
__device__ __forceinline__ int lm_next_stream(int* next, const int32_t* order, int nstreams, int lane) {
  int k = 0;
  if (lane == 0) k = atomicAdd(next, 1);
  k = __shfl_sync(0xffffffffu, k, 0);
  return k < nstreams ? order[k] : -1;
}

// One warp per stream (grid-stride over streams).  sizes[s] = stream bytes, or
// PG_ERR_ARG for a symbol above 2 or a symbol count that does not match.
// Coding kernels are compiled for three CTAs (12 warps) per SM.
constexpr int kLmCodeCtas = 3;

__global__ void __launch_bounds__(kLmThreads, kLmCodeCtas)
lm_encode_kernel(const uint16_t* __restrict__ P, uint64_t hash, const lm_block_t* __restrict__ blocks, int nstreams,
                 const int32_t* __restrict__ order, int* __restrict__ next, const uint8_t* __restrict__ symbols,
                 const int64_t* __restrict__ offsets, uint8_t* __restrict__ out,
                 const int64_t* __restrict__ out_offsets, int64_t* __restrict__ sizes, const dev_tables_t T) {
  extern __shared__ __align__(16) unsigned char lm_smem_raw[];
  lm_tables& S = *reinterpret_cast<lm_tables*>(lm_smem_raw);
  lm_build_tables(S, P, threadIdx.x, blockDim.x);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint8_t* row = lm_smem_raw + sizeof(lm_tables) + kLmWarpSmem * warp + kLmSymRow * lane;
  uint32_t* prev = reinterpret_cast<uint32_t*>(lm_smem_raw + sizeof(lm_tables) + kLmWarpSmem * warp +
                                               32 * kLmSymRow) + kLmPrevWords * lane;
  const unsigned below = (1u << lane) - 1;
  for (int s; (s = lm_next_stream(next, order, nstreams, lane)) >= 0;) {
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
    const int64_t R = (n + 31) / 32;   // the run of nodes of each lane
    for (int64_t round = R - 1; round >= 0; round--) {
      const int64_t i = R * lane + round;
      const bool active = i < n;
      lm_nodefrag N;
      lm_round_nodes(S, P, B, i, active, T, lane, N);
      if (active) bad |= lm_row_in(row, sym0 + 256 * i);
      if (active && round > 0) lm_prev_from(prev, sym0 + 256 * (i - 1));
      else lm_prev_none(prev);
      for (int st = 127; st >= 0; st--) {
        uint32_t ctx[2] = {0u, 0u};
        if (active) {
          ctx[0] = lm_context_packed(row, st) | uint32_t(lm_prev_sym(prev, st)) << 16;
          ctx[1] = lm_context_packed(row, st + 128) | uint32_t(lm_prev_sym(prev, st + 128)) << 16;
        }
        float zA[3], zB[3];
        lm_step_logits(S, N, lane, st, ctx, zA, zB);
        lm_freq_t FA = {}, FB = {};
        int vA = 0, vB = 0;
        if (active) {
          FA = lm_freqs(zA);
          FB = lm_freqs(zB);
          vA = row[st] & 3;
          vB = row[st + 128] & 3;
          if (vA > 2) vA = 0;   // (flagged when the row was read)
          if (vB > 2) vB = 0;
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
__global__ void __launch_bounds__(kLmThreads, kLmCodeCtas)
lm_decode_kernel(const uint16_t* __restrict__ P, uint64_t hash, const lm_block_t* __restrict__ blocks, int nstreams,
                 const int32_t* __restrict__ order, int* __restrict__ next, const uint8_t* __restrict__ in,
                 const int64_t* __restrict__ in_offsets,
                 const int64_t* __restrict__ in_sizes, uint8_t* __restrict__ symbols,
                 const int64_t* __restrict__ sym_offsets, const int64_t* __restrict__ sym_caps,
                 int64_t* __restrict__ status, const dev_tables_t T) {
  extern __shared__ __align__(16) unsigned char lm_smem_raw[];
  lm_tables& S = *reinterpret_cast<lm_tables*>(lm_smem_raw);
  lm_build_tables(S, P, threadIdx.x, blockDim.x);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint8_t* row = lm_smem_raw + sizeof(lm_tables) + kLmWarpSmem * warp + kLmSymRow * lane;
  uint32_t* prev = reinterpret_cast<uint32_t*>(lm_smem_raw + sizeof(lm_tables) + kLmWarpSmem * warp +
                                               32 * kLmSymRow) + kLmPrevWords * lane;
  uint16_t* win = reinterpret_cast<uint16_t*>(lm_smem_raw + sizeof(lm_tables) + kLmWarpSmem * warp +
                                              32 * kLmSymRow + 32 * 4 * kLmPrevWords);
  const unsigned above = lane == 31 ? 0u : ~0u << (lane + 1);
  for (int s; (s = lm_next_stream(next, order, nstreams, lane)) >= 0;) {
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
    const int64_t R = (n + 31) / 32;   // the run of nodes of each lane
    for (int64_t round = 0; round < R; round++) {
      const int64_t i = R * lane + round;
      const bool active = i < n;
      lm_nodefrag N;
      lm_round_nodes(S, P, B, i, active, T, lane, N);
      // the previous node of the run is the row of the last round
      if (round > 0) lm_prev_from(prev, row);
      else lm_prev_none(prev);
      for (int w = 0; w < 64; w++) reinterpret_cast<uint32_t*>(row)[w] = 0u;
      // the round's words are the last unread ones: stage up to kLmWordWin of them
      const int64_t wlo = ptr > kLmWordWin ? ptr - kLmWordWin : 0;
      __syncwarp();
      for (int64_t w = wlo + lane; w < ptr; w += 32) win[w - wlo] = get16(words + 2 * w);
      __syncwarp();
      for (int st = 0; st < 128; st++) {
        uint32_t ctx[2] = {0u, 0u};
        if (active) {
          ctx[0] = lm_context_packed(row, st) | uint32_t(lm_prev_sym(prev, st)) << 16;
          ctx[1] = lm_context_packed(row, st + 128) | uint32_t(lm_prev_sym(prev, st + 128)) << 16;
        }
        float zA[3], zB[3];
        lm_step_logits(S, N, lane, st, ctx, zA, zB);
        lm_freq_t FA = {}, FB = {};
        if (active) {
          FA = lm_freqs(zA);
          FB = lm_freqs(zB);
        }
        const int vA = lm_get_symbol(x, FA, active, words, win, wlo, ptr, above, bad);
        const int vB = lm_get_symbol(x, FB, active, words, win, wlo, ptr, above, bad);
        row[st] = uint8_t(vA);
        row[st + 128] = uint8_t(vB);
      }
      if (active) lm_row_out(row, out0 + 256 * i);
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
    lm_node_sum(S, P, feats, nf, node);
    int u[4];
    const uint8_t* sym = symbols + offsets[s] + 256 * i;
    lm_context_clamped(sym, r, u);
    const int64_t R = (blocks[s].nodes + 31) / 32;   // lanes' runs: the previous node is i - 1 inside a run
    const int prev = i % R ? (sym[r - 256] & 3) : 3;
    float z[3];
    lm_logits(S, node, r, u, prev, z);
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
constexpr int kW1Pad = 65;  // rows of 64 floats padded so lanes reading different rows use different banks
constexpr int kMaxFeats = 49;  // 36 stones + 4 rotation + 8 neighbours + the previous node

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
  __syncthreads();
  // W1's rotation and neighbour rows and W2 on their column grids, as the
  // exported model holds them (lm_grid_params)
  if (tid < kLmHidden) {
    float col[kLmHidden];
    for (int f = 0; f < kLmCtxRows; f++) col[f] = params[kLmW1 + (kLmRot + f) * kLmHidden + tid];
    lm_grid_column(col, kLmCtxRows, 1);
    for (int f = 0; f < kLmCtxRows; f++) G.w1[(kLmRot + f) * kW1Pad + tid] = col[f];
    for (int k = 0; k < kLmHidden; k++) col[k] = params[kLmW2 + k * kLmHidden + tid];
    lm_grid_column(col, kLmHidden, 1);
    for (int k = 0; k < kLmHidden; k++) G.w2[k][tid] = col[k];
  }
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
          const int64_t R = (blocks[s].nodes + 31) / 32;   // the coder's runs of nodes
          G.feats[tid][nf++] = uint8_t(kLmPrev + (i % R ? (sym[r - 256] & 3) : 3));
        }
      }
    }
    G.nfeat[tid] = nf;
    float a2[kLmHidden];
    float z[3] = {0.f, 0.f, 0.f};
    if (y >= 0) {
      // h1 holds the quantized activations hq / 16 (learned.cuh): the stone
      // rows summed in order, the last 13 (rotation, neighbour and
      // previous-node rows, on their grids) summed exactly, then added
      const int ns = nf - 13;
      for (int k = 0; k < kLmHidden; k++) {
        float a = G.b1[k], s1 = 0.f;
        for (int f = 0; f < ns; f++) a += G.w1[G.feats[tid][f] * kW1Pad + k];
        for (int f = ns; f < nf; f++) s1 += G.w1[G.feats[tid][f] * kW1Pad + k];
        G.h1[tid][k] = f_mul(lm_act_q(f_add(a, s1)), kLmActInv);
      }
      // the layer-2 sums are exact on the grid, so a2 = b2 + sum rounds once
#pragma unroll
      for (int j = 0; j < kLmHidden; j++) a2[j] = 0.f;
      for (int k = 0; k < kLmHidden; k++) {
        const float h = G.h1[tid][k];
#pragma unroll
        for (int j = 0; j < kLmHidden; j++) a2[j] = fmaf(G.w2[k][j], h, a2[j]);
      }
#pragma unroll
      for (int j = 0; j < kLmHidden; j++) a2[j] = f_add(G.b2[j], a2[j]);
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
    // dL/da1 into x: the quantizer passes the gradient straight through
    // where the activation is neither cut by relu nor clamped at the top
    if (y >= 0) {
      for (int k = 0; k < kLmHidden; k++) {
        float d = 0.f;
        const float h = G.h1[tid][k];
        if (h > 0.f && h < kLmActMax * kLmActInv)
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
  if (h[0] != kLmMagic || h[1] != kLmModelVersion || h[2] != uint32_t(kLmParams)) {
    err = "not a version-3 PGLM model";
    return false;
  }
  // W1's rotation and neighbour rows and W2 must lie on their column grids,
  // or the tensor cores' sums would not be exact
  std::vector<float> w(kLmParams), q;
  for (int i = 0; i < kLmParams; i++) {
    const int b = kLmModelHeader + 2 * i;
    w[i] = bf16_value(uint16_t(model[b] | model[b + 1] << 8));
    if (!std::isfinite(w[i])) { err = "non-finite parameter " + std::to_string(i); return false; }
  }
  q = w;
  lm_grid_params(q.data());
  for (int i = 0; i < kLmParams; i++)
    if (q[i] != w[i]) { err = "parameter " + std::to_string(i) + " is not on its grid"; return false; }
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
  int32_t* order = nullptr;   // streams by node count, largest first (after the blocks)
  int* next = nullptr;        // the coding kernels' stream counter, zeroed (after the order)
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
  // One buffer: the blocks, the processing order and the counter
  std::vector<int32_t> order(n);
  for (int s = 0; s < n; s++) order[s] = s;
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return B[a].nodes > B[b].nodes; });
  const size_t bb = sizeof(lm_block_t) * std::max(n, 1), ob = (sizeof(int32_t) * std::max(n, 1) + 15) & ~size_t(15);
  char* buf = nullptr;
  PG_CUDA(cudaMallocAsync(&buf, bb + ob + 16, stream));
  L.blocks = reinterpret_cast<lm_block_t*>(buf);
  L.order = reinterpret_cast<int32_t*>(buf + bb);
  L.next = reinterpret_cast<int*>(buf + bb + ob);
  PG_CUDA(cudaMemcpyAsync(L.blocks, B.data(), sizeof(lm_block_t) * n, cudaMemcpyHostToDevice, stream));
  PG_CUDA(cudaMemcpyAsync(L.order, order.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream));
  PG_CUDA(cudaMemsetAsync(L.next, 0, sizeof(int), stream));
  if (host_blocks) *host_blocks = std::move(B);
  return PG_OK;
}

template<class K> static int lm_smem_opt_in(K kernel, size_t bytes) {
  PG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
  return PG_OK;
}

// The coding kernels: as many CTAs as are resident at once (the streams are
// handed out dynamically), no more than there are streams for.
template<class K> static int lm_code_grid(K kernel, int nstreams) {
  int dev = 0, sms = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kLmThreads, kLmCodeSmem) != cudaSuccess || per < 1)
    per = 1;
  return std::max(1, std::min((nstreams + kLmWarps - 1) / kLmWarps, per * sms));
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
  const uint32_t h[3] = {kLmMagic, kLmModelVersion, uint32_t(kLmParams)};
  memcpy(model, h, 12);
  std::vector<float> p(params, params + kLmParams);
  for (int i = 0; i < kLmParams; i++)
    if (!std::isfinite(p[i])) return fail(PG_ERR_ARG, "non-finite parameter " + std::to_string(i));
  lm_grid_params(p.data());
  for (int i = 0; i < kLmParams; i++) {
    const uint16_t b = bf16_round(p[i]);
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
  lm_encode_kernel<<<lm_code_grid(lm_encode_kernel, nstreams), kLmThreads, kLmCodeSmem, st>>>(
      L.params, L.hash, L.blocks, nstreams, L.order, L.next, symbols, offsets, out, out_offsets, sizes, *T);
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
  lm_decode_kernel<<<lm_code_grid(lm_decode_kernel, nstreams), kLmThreads, kLmCodeSmem, st>>>(
      L.params, L.hash, L.blocks, nstreams, L.order, L.next, in, in_offsets, in_sizes, symbols, sym_offsets, sym_caps,
      status, *T);
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
