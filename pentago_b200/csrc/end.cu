// End-engine block-line compute on the GPU: the replacement for
// schedule_compute_line / compute_microline (pentago/end/compute.cc:219-404).
//
// One CTA computes one microline (a 1-D run of parent nodes along the line's
// dimension at one cross-section position).  It works in two phases:
//
//  1. child phase: every child node j of the microline is loaded once and
//     turned into Q_j = T_{b * L_j}(rmax(~child_j)), the child's contribution
//     already moved into the parent's frame, for both the win and the
//     not-lost halves.  rmax commutes with every symmetry (rmax(C) = C + R
//     with R = {+-e_q}, which every conjugation phi_g preserves), so this is
//     the reference's rmax(transform_super(s, ~child)) with the per-move part
//     of s factored out.  Q lives in shared memory.
//  2. parent phase: each parent node ORs, over its empty cells, the
//     immediate wins of the move plus Q_j translated along the line's own
//     axis by the move's rotation (the leftmost factor local((ir&3)<<2dim) of
//     the reference's symmetry, compute.cc:336-338), then applies the
//     immediate-win masks of compute.cc:353-355.
//
// 35-stone sections have no children (compute_microline<true>): the child
// result is the immediate one, compute.cc:329-333.
#include "superscore.cuh"
#include "lines.h"
#include "runtime.h"
#include "../../include/pentago_b200.h"
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

namespace pg {

PG_HD int pow3(int b) {  // 3^b for 0 <= b < 9, the radix-3 weight of quadrant cell b
  return ((b & 1) ? 3 : 1) * ((b & 2) ? 9 : 1) * ((b & 4) ? 81 : 1) * ((b & 8) ? 6561 : 1);
}

PG_HD int ladd(int a, int b) {
  return (((a & 0x33) + (b & 0x33)) & 0x33) + (((a & 0xcc) + (b & 0xcc)) & 0xcc);
}

// Per-device error word for device-side bounds checks (bit 0: child index
// out of range).  Read and cleared by pg_end_check.
__device__ unsigned int d_end_errors;
__device__ void record_errors(unsigned e) { atomicOr(&d_end_errors, e); }

struct microline_geom {
  int64_t input_base, last_input_base, output_base, last_output_base;
  int input_stride, output_stride;
  int base_l;
};

PG_HD void row_strides(const int* shape, int* st) {
  st[3] = 1;
  st[2] = shape[3];
  st[1] = shape[3] * shape[2];
  st[0] = shape[3] * shape[2] * shape[1];
}

// Index bookkeeping of compute_microline (compute.cc:224-281): addressing
// and the base translation (no global loads; the cross quadrants' stones
// come from the line's cross records).
template<int DIM>
PG_HD microline_geom microline_addressing(const line_dev_t& L, int m) {
  microline_geom G;
  int fb[4];
  const int c1 = L.cross[1], c2 = L.cross[2];
  fb[DIM] = 0;
#pragma unroll
  for (int i = 0, k = 0; i < 4; i++) {
    if (i == DIM) continue;
    fb[i] = k == 0 ? m / (c1 * c2) : k == 1 ? m / c2 % c1 : m % c2;
    k++;
  }
  // Output addressing
  int obs[4], ost[4];
#pragma unroll
  for (int i = 0; i < 4; i++) obs[i] = i == DIM ? 8 : L.out_shape[i];
  row_strides(obs, ost);
  G.output_stride = ost[DIM];
  G.output_base = int64_t(ost[0]) * fb[0] + ost[1] * fb[1] + ost[2] * fb[2] + ost[3] * fb[3];
  // Input addressing, in the standardized child section
  int ibs[4], ist[4], fcb[4], rcb[4];
#pragma unroll
  for (int i = 0; i < 4; i++) ibs[i] = obs[L.perm[i]];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    fcb[i] = fb[L.perm[i]];
    const int fcn = 8 * L.first_child_block[i] + fcb[i];
    rcb[i] = fcb[i] ^ int(i != L.child_dim && fcn < L.refl_moves[i]);
  }
  row_strides(ibs, ist);
  G.input_stride = ist[L.child_dim];
  G.input_base = int64_t(ist[0]) * rcb[0] + ist[1] * rcb[1] + ist[2] * rcb[2] + ist[3] * rcb[3];
  // Last blocks are shorter along the line
  obs[DIM] = (L.nparent & 7) ? (L.nparent & 7) : 8;
  row_strides(obs, ost);
  G.last_output_base = int64_t(ost[0]) * fb[0] + ost[1] * fb[1] + ost[2] * fb[2] + ost[3] * fb[3];
  ibs[L.child_dim] = (L.nchild & 7) ? (L.nchild & 7) : 8;
  row_strides(ibs, ist);
  G.last_input_base = int64_t(ist[0]) * rcb[0] + ist[1] * rcb[1] + ist[2] * rcb[2] + ist[3] * rcb[3];
  // Base transform = inverse_transform * (reflection locals of the cross dims)
  int local = 0;
#pragma unroll
  for (int i = 0; i < 4; i++)
    if (i != L.child_dim) local += L.xsym[i][fcb[i] & 7];
  G.base_l = ladd(L.inv_l, local);
  return G;
}

// Per-microline context: the geometry (the win tables live beside it).
struct micro_ctx {
  microline_geom G;
};

constexpr int kMaxPat = 126;  // C(9,4): most stone patterns of one count in a quadrant
constexpr int kTerms = 17;    // win patterns touching one quadrant
constexpr int kTab = 80;      // subset tables: terms 0-3, 4-7, 8-11 (16 entries each), 12-16 (32)

// Chunk of subset-table entry e (the first three tables fill one 128-byte
// row of shared-memory banks each, so their lookups never conflict).
PG_HD int table_chunk(int e) { return e < 48 ? e >> 4 : 3; }

// super_wins with the line quadrant DIM varying and the other three fixed,
// as subset tables.  Each win pattern touching DIM ("term" t) wins at the
// rotations where DIM's coverage bit r_DIM and the fixed quadrants' product
// f_t(other rotations) are both set, so for each r_DIM the answer is the OR
// of f_t over the terms that quadrant DIM covers at r_DIM (term_sub), read
// from three tables of ORs over subsets of terms.  The f_t live in the frame
// where axes DIM and 3 are swapped, so that one r_DIM is two whole words.

// 4-bit coverage c of the quadrant on frame axis a, broadcast over the other
// two axes of a 64-bit slice (bit i0 + 4 i1 + 16 i2).
PG_HD uint64_t axis_broadcast(int a, uint32_t c) {
  if (a == 0) return uint64_t(c) * 0x1111111111111111ull;
  if (a == 1) return uint64_t(spread4(c)) * 0x0001000100010001ull;
  uint64_t f = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) f |= uint64_t(c >> k & 1) * (uint64_t(0xffff) << (16 * k));
  return f;
}

// The cross quadrants' state indices (in their sections' rotation-minimal
// lists) of microline m.
template<int DIM>
PG_HD void cross_index(const line_dev_t& L, int m, int* xq) {
  const int c1 = L.cross[1], c2 = L.cross[2];
#pragma unroll
  for (int q = 0, k = 0; q < 4; q++) {
    if (q == DIM) { xq[q] = 0; continue; }
    const int f = k == 0 ? m / (c1 * c2) : k == 1 ? m / c2 % c1 : m % c2;
    k++;
    xq[q] = 8 * L.block0[q] + f;
  }
}

// The factor of lane t of a table warp for one side of a microline: for
// t < 17 term t's f_t, else the product of missed pattern t - 17, in the
// line frame, from the side's cross records of the microline's cross
// quadrant states (xe[c]: the c-th quadrant other than DIM).
template<int DIM>
PG_HD uint64_t lane_factor(const line_dev_t& L, const uint4* xe, int t) {
  const bool term = t < kTerms;
  const int u = term ? t : t - kTerms;
  const int p = term ? L.term_pat[u] : L.miss_pat[u];
  const int nq = term ? 2 : 3;
  uint64_t f = ~uint64_t(0);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (k >= nq) break;
    const int q = term ? L.term_q[u][k] : L.miss_q[u][k];
    if (q > 3) break;
    const uint4 e = xe[q - (q > DIM)];
    const uint32_t w = (p >> 3) == 0 ? e.x : (p >> 3) == 1 ? e.y : (p >> 3) == 2 ? e.z : e.w;
    f &= axis_broadcast(q == 3 ? DIM : q, w >> (4 * (p & 7)) & 15);
  }
  return f;
}

// Where the cross record of one side of a microline's c-th cross quadrant
// state lies.
template<int DIM>
PG_HD const uint4* cross_entry(const line_dev_t& L, const int* xq, int side, int c) {
  const int q = c + (c >= DIM);
  return reinterpret_cast<const uint4*>(L.xrecs) + L.xoff[q] + 2 * xq[q] + side;
}

// Entry e of the subset tables from the 17 f_t; the first table also carries
// c0, the OR of the patterns that miss DIM, so every evaluation includes it.
PG_HD uint2 table_entry(const uint2* f, uint64_t c0, int e) {
  const int c = table_chunk(e), s = e - 16 * c;
  uint32_t lo = c ? 0u : uint32_t(c0), hi = c ? 0u : uint32_t(c0 >> 32);
#pragma unroll
  for (int b = 0; b < 5; b++)
    if (s >> b & 1) { lo |= f[4 * c + b].x; hi |= f[4 * c + b].y; }
  return make_uint2(lo, hi);
}

// super_wins from the tables and the covered terms per rotation of DIM, in
// the line frame: axes DIM and 3 exchanged, so that rotation p of the line
// quadrant is word pair p (words 2p, 2p + 1) and a translation along the
// line's axis is a choice of pairs, not arithmetic.
PG_HD super8 table_eval(const uint2* tab, const uint4 sub) {
  super8 r;
  const uint32_t S[4] = {sub.x, sub.y, sub.z, sub.w};
#pragma unroll
  for (int d = 0; d < 4; d++) {
    const uint2 a = tab[S[d] & 15], b = tab[16 + (S[d] >> 4 & 15)], c = tab[32 + (S[d] >> 8 & 15)],
                e = tab[48 + (S[d] >> 12 & 31)];
    r.w[2 * d] = a.x | b.x | c.x | e.x;
    r.w[2 * d + 1] = a.y | b.y | c.y | e.y;
  }
  return r;
}

// Standard frame <-> line frame (exchanging axes DIM and 3 is its own
// inverse).  For DIM 2 the exchange of index bits 4 and 6 moves 16-bit
// halves between words (byte permutes) and that of bits 5 and 7 renames words.
template<int DIM> PG_HD void s_line_frame(super8& s) {
  if constexpr (DIM == 2) {
#ifdef __CUDA_ARCH__
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int w = (k & 1) | (k & 2) << 1;  // 0, 1, 4, 5
      const uint32_t lo = s.w[w], hi = s.w[w | 2];
      s.w[w] = __byte_perm(lo, hi, 0x5410);
      s.w[w | 2] = __byte_perm(lo, hi, 0x7632);
    }
    uint32_t t = s.w[1]; s.w[1] = s.w[4]; s.w[4] = t;
    t = s.w[3]; s.w[3] = s.w[6]; s.w[6] = t;
#else
    s_swap_axes<2, 3>(s);
#endif
  } else if constexpr (DIM < 2) {
    s_swap_axes<DIM, 3>(s);
  }
}

// x = k n + i with 0 <= i < n, for 0 <= x < 2^20 and m = floor((2^32 - 1) / n):
// the high product gives k exactly or one short.
PG_HD void split(int x, int n, uint32_t m, int& k, int& i) {
#ifdef __CUDA_ARCH__
  k = int(__umulhi(uint32_t(x), m));
#else
  k = int((uint64_t(uint32_t(x)) * m) >> 32);
#endif
  i = x - k * n;
  if (i >= n) { i -= n; k++; }
}

// Per-microline results live in shared memory as structures of arrays, word
// pair by word pair (lanes reading different entries then spread over the
// banks).  Pattern results: rotation class e (the mover's classes, then the
// opponent's: pp in all) has pair p at p * pp + e.  Children: pair p of Q_j
// with its not-lost pair, one uint4, at p * nchild + j.
PG_HD void pattern_store(uint2* pat, int e, int pp, const super8& w) {
#pragma unroll
  for (int p = 0; p < 4; p++) pat[p * pp + e] = make_uint2(w.w[2 * p], w.w[2 * p + 1]);
}
// super_wins of class e's representative rotated left rho times: rotating the
// line quadrant shifts the rotation sets along its axis, so pair p of the
// result is pair p + rho of the representative's.
PG_HD super8 pattern_rotated(const uint2* pat, int e, int pp, int rho) {
  super8 r;
#pragma unroll
  for (int p = 0; p < 4; p++) {
    const uint2 a = pat[((p + rho) & 3) * pp + e];
    r.w[2 * p] = a.x;
    r.w[2 * p + 1] = a.y;
  }
  return r;
}

// What the children of a line need from its descriptor, read once per thread.
struct child_src {
  const uint64_t* input;
  const int64_t* in_off;
  int line_moves, last_block;
  bool wide;  // 32-byte aligned input: 256-bit loads
};
PG_HD child_src child_source(const line_dev_t& L) {
  return child_src{L.input, L.in_off, L.line_moves, L.input_blocks - 1,
                   (reinterpret_cast<uintptr_t>(L.input) & 31) == 0};
}
// One half of a child node (32 bytes at p, 32-byte aligned when C.wide).
PG_HD super8 child_load(const child_src& C, const uint64_t* p) { return C.wide ? s_load_nc32(p) : s_load_ldg(p); }

// Address of child j of a microline in the line's input.
PG_HD const uint64_t* child_addr(const child_src& C, const microline_geom& G, int j) {
  const int jj = j ^ int(j < C.line_moves);
  const int blk = j >> 3;
  const int64_t idx = C.in_off[blk] + (blk == C.last_block ? G.last_input_base : G.input_base) +
                      int64_t(G.input_stride) * (jj & 7);
  return C.input + 8 * idx;
}

// ---------------------------------------------------------------------------
// The children's transform, line frame first.  A child's contribution is
// Q = swap_DIM3(phi_g(T_l(y))) with y = rmax(~child).  Writing phi_g as
// s * sigma (sigma an axis permutation, s = -1 when g holds the reflection),
// Q[u] = Z[s u + sigma(l)] with Z = swap_DIM3(sigma(y)): a fixed axis
// permutation, then on each line-frame axis a rotation (s = 1) or a
// reflection (s = -1) by the matching component of sigma(l).  Axis 3 of the
// line frame is the child's own line axis: its map is applied by the
// addresses the word pairs are stored at.

// Cost in word operations of exchanging axes a < b (delta swaps within
// words, between words, or renaming words).
constexpr int swap_cost(int a, int b) {
  return (a == 2 && b == 3) ? 20 : b == 3 ? 40 : (a == 0 && b == 1) ? 64 : 52;
}
// The cheapest sequence of at most four axis exchanges giving p.
struct swap_seq { int n, a[4], b[4]; };
constexpr swap_seq cheapest_swaps(axis_perm target) {
  const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {1, 2, 3, 2, 3, 3};
  swap_seq best{-1, {0, 0, 0, 0}, {0, 0, 0, 0}};
  int best_cost = 1 << 30;
  for (int n = 0; n <= 4; n++) {
    int total = 1;
    for (int i = 0; i < n; i++) total *= 6;
    for (int code = 0; code < total; code++) {
      axis_perm p = perm_id();
      int cost = 0, c = code;
      swap_seq s{n, {0, 0, 0, 0}, {0, 0, 0, 0}};
      for (int i = 0; i < n; i++, c /= 6) {
        s.a[i] = pa[c % 6];
        s.b[i] = pb[c % 6];
        p = perm_swap(p, s.a[i], s.b[i]);
        cost += swap_cost(s.a[i], s.b[i]);
      }
      bool same = true;
      for (int q = 0; q < 4; q++) same = same && p.to[q] == target.to[q];
      if (same && cost < best_cost) { best = s; best_cost = cost; }
    }
  }
  return best;
}
template<int DIM, int G> PG_HD void line_permute(super8& s) {
  constexpr swap_seq q = cheapest_swaps(line_sigma(DIM, G));
  static_assert(q.n >= 0, "every axis permutation is a product of at most four exchanges");
  if constexpr (q.n > 0) s_swap_axes<q.a[0], q.b[0]>(s);
  if constexpr (q.n > 1) s_swap_axes<q.a[1], q.b[1]>(s);
  if constexpr (q.n > 2) s_swap_axes<q.a[2], q.b[2]>(s);
  if constexpr (q.n > 3) s_swap_axes<q.a[3], q.b[3]>(s);
}

PG_HD uint32_t byte_perm(uint32_t x, uint32_t y, uint32_t s) {
#ifdef __CUDA_ARCH__
  return __byte_perm(x, y, s);
#else
  const uint64_t v = uint64_t(y) << 32 | x;
  uint32_t r = 0;
  for (int i = 0; i < 4; i++) r |= uint32_t(v >> (8 * (s >> (4 * i) & 7)) & 0xff) << (8 * i);
  return r;
#endif
}

// Maps of line-frame axes 0-2 with amounts c0, c1, c2: out[u] = in[u + c]
// (rotations) or out[u] = in[c - u] (reflections), per axis.
template<bool REFL> PG_HD void axis_maps(super8& s, int c0, int c1, int c2) {
  if constexpr (REFL) {
    // axis 0 (bits of a nibble): c - u is u ^ c for odd c
    if (c0 & 1) {
#pragma unroll
      for (int i = 0; i < 8; i++) s.w[i] = ((s.w[i] >> 1) & 0x55555555u) | ((s.w[i] << 1) & 0xaaaaaaaau);
      if (c0 & 2)
#pragma unroll
        for (int i = 0; i < 8; i++) s.w[i] = ((s.w[i] >> 2) & 0x33333333u) | ((s.w[i] << 2) & 0xccccccccu);
    } else {
      const uint32_t m = c0 ? 0x11111111u : 0x22222222u;   // positions 0, 2 or 1, 3 exchanged
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const uint32_t t = ((s.w[i] >> 2) ^ s.w[i]) & m;
        s.w[i] ^= t ^ (t << 2);
      }
    }
    // axis 1 (nibbles of a 16-bit half)
    if (c1 & 1) {
#pragma unroll
      for (int i = 0; i < 8; i++) s.w[i] = ((s.w[i] >> 4) & 0x0f0f0f0fu) | ((s.w[i] << 4) & 0xf0f0f0f0u);
      if (c1 & 2)
#pragma unroll
        for (int i = 0; i < 8; i++) s.w[i] = byte_perm(s.w[i], 0, 0x2301);
    } else {
      const uint32_t m = c1 ? 0x000f000fu : 0x00f000f0u;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const uint32_t t = ((s.w[i] >> 8) ^ s.w[i]) & m;
        s.w[i] ^= t ^ (t << 8);
      }
    }
  } else {
    const uint32_t m0 = (0xfu >> c0) * 0x11111111u, m1 = (0xffffu >> (4 * c1)) * 0x10001u;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      uint32_t x = s.w[i];
      x = ((x >> c0) & m0) | ((x << (4 - c0)) & ~m0);
      x = ((x >> (4 * c1)) & m1) | ((x << (16 - 4 * c1)) & ~m1);
      s.w[i] = x;
    }
  }
  // axis 2 (half of a word, then word of a pair): byte permutes per pair,
  // selectors for c = 0..3 packed 16 bits each
  const uint64_t klo = REFL ? 0x5476325410327610ull : 0x1076765454323210ull;
  const uint64_t khi = REFL ? 0x1032761054763254ull : 0x5432321010767654ull;
  const uint32_t slo = uint32_t(klo >> (16 * c2)) & 0xffff, shi = uint32_t(khi >> (16 * c2)) & 0xffff;
#pragma unroll
  for (int p = 0; p < 4; p++) {
    const uint32_t lo = s.w[2 * p], hi = s.w[2 * p + 1];
    s.w[2 * p] = byte_perm(lo, hi, slo);
    s.w[2 * p + 1] = byte_perm(lo, hi, shi);
  }
}

template<int DIM, int G> PG_HD void child_map(super8& a, int c) {
  line_permute<DIM, G>(a);
  axis_maps<(G >= 4)>(a, c & 3, c >> 2 & 3, c >> 4 & 3);
}

PG_HD uint32_t select4(const uint4 v, int i) {
  return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

// Child j -> Q_j in the line frame, both halves already moved into the
// parent's frame: Q_j = swap(phi_g(rmax(~child) - l_j)), done as a fixed
// axis permutation of rmax(~child) and a rotation or reflection of each
// line-frame axis (see axis_maps); the map of axis 3, the child's own line
// axis, is applied by the addresses of the stored word pairs.  The win half
// also carries W_j = super_wins of the mover's stones once the move is made
// (csub: the terms they cover per rotation): a move that makes the child
// wins at once, and super_wins of the moved quadrant is W_j translated by the
// move's rotation exactly as the child's value is, so a parent ORs one
// translated Q_j for both.
//
// The two halves are independent and computed by adjacent threads: half 0
// is the win half (x = the child's not-lost super, with W_j), half 1 the
// not-lost half (x = its win super).  q2 holds pair p of Q_j as the uint2
// halves 2 (p nc + j) + half.
template<int DIM, int G>
PG_HD void child_half(const line_dev_t& L, const microline_geom& geom, const uint2* tab0, uint2* q2, int j, int nc,
                      int half, const super8& x, const uint4 csub) {
  super8 z = s_rmax(s_not(x));
  const int c = ladd(geom.base_l, int(L.csym[j]) << 6);   // the translation, axes moved to the line frame
  child_map<DIM, G>(z, c);
  // Pair k goes to pair p(k) = k - c3 (rotation) or c3 - k (reflection), and
  // W_j's pair p(k) is evaluated beside it.
  const int c3 = c >> 6 & 3, sgn = G >= 4 ? -1 : 1;
  int pk[4];
#pragma unroll
  for (int k = 0; k < 4; k++) pk[k] = (sgn * (k - c3)) & 3;
#ifdef __CUDA_ARCH__
  // On the device the two threads of a child each evaluate two of W_j's four
  // word pairs (the not-lost half's pairs 2 and 3 reach the win half by
  // shuffles), so neither idles while the other does the lookups.  Both
  // threads of a child are always active together.
  {
    uint32_t w[4];
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
      const uint32_t S = select4(csub, (sgn * (2 * half + kk - c3)) & 3);
      const uint2 a = tab0[S & 15], b = tab0[16 + (S >> 4 & 15)], d = tab0[32 + (S >> 8 & 15)],
                  e = tab0[48 + (S >> 12 & 31)];
      w[2 * kk] = a.x | b.x | d.x | e.x;
      w[2 * kk + 1] = a.y | b.y | d.y | e.y;
    }
    const unsigned mask = __activemask();
    uint32_t o[4];
#pragma unroll
    for (int t = 0; t < 4; t++) o[t] = __shfl_xor_sync(mask, w[t], 1);
    if (half == 0) {
#pragma unroll
      for (int t = 0; t < 4; t++) {
        z.w[t] |= w[t];
        z.w[4 + t] |= o[t];
      }
    }
  }
#else
  if (half == 0)
    z = s_or(z, table_eval(tab0, make_uint4(select4(csub, pk[0]), select4(csub, pk[1]), select4(csub, pk[2]),
                                            select4(csub, pk[3]))));
#endif
#pragma unroll
  for (int k = 0; k < 4; k++) q2[2 * (pk[k] * nc + j) + half] = make_uint2(z.w[2 * k], z.w[2 * k + 1]);
}

// Parent i of a microline (compute.cc:308-356), in the line frame until its
// store.  h is the first 16 bytes of its record, rec the record.
template<int DIM>
PG_HD void parent_node(const line_dev_t& L, const microline_geom& G, const uint2* tab0, const uint4* qs,
                       const uint2* pats, const uint4 h, const uint4* rec, int i, unsigned* errors) {
  const int p0 = L.npat[0], pp = p0 + L.npat[1];
  // Where the result goes.  Node offsets are multiples of 64 bytes, so a
  // 32-byte aligned output base allows one 256-bit access per super.  When
  // accumulating, the node is prefetched into L1 first, so the read of its
  // previous value at the end does not wait on memory.
  const int blk = i >> 3;
  const int64_t oidx = L.out_off[blk] + (blk == L.length - 1 ? G.last_output_base : G.output_base) +
                       int64_t(G.output_stride) * (i & 7);
  uint64_t* out = L.output + 8 * oidx;
  const bool wide = (reinterpret_cast<uintptr_t>(L.output) & 31) == 0;
  const bool accumulate = L.flags & PG_LINE_OR;
#ifdef __CUDA_ARCH__
  if (accumulate) asm volatile("prefetch.global.L1 [%0];" ::"l"(out));
#endif
  // super_wins of both sides, from their rotation classes
  const super8 wins0 = pattern_rotated(pats, int(h.x & 0xff), pp, int(h.x >> 16 & 3));
  const super8 wins1 = pattern_rotated(pats, p0 + int(h.x >> 8 & 0xff), pp, int(h.x >> 18 & 3));
  super8 wins, not_loss;
  if (L.slice35) {
    // The board is full after the move: the child's value is immediate
    // (compute.cc:329-333); the union over the empty cells of super_wins
    // after the move is one table evaluation of the union of the covered
    // terms, and rmax is OR-linear, so the union over moves works.
    const super8 moved = table_eval(tab0, ldg(rec + 2));
    wins = s_or(moved, s_rmax(s_andnot(moved, wins1)));
    not_loss = s_rmax(s_or(moved, s_not(wins1)));
  } else {
    wins = not_loss = s_zero();
    const int nmoves = int(h.x >> 24);
    const uint4 h2 = nmoves > 6 ? ldg(rec + 1) : make_uint4(0, 0, 0, 0);
    const uint32_t mvw[5] = {h.y, h.z, h.w, h2.x, h2.y};
    // A move's entry is the slot r nc + j of the child's pair r; pair p + r
    // follows nc p slots later, wrapping around the 4 nc slots.
    const int nc = L.nchild, all = 4 * nc;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      if (k >= nmoves) break;
      const int a0 = int(mvw[k >> 1] >> (16 * (k & 1)) & 0xffff);
      if (a0 >= all) { *errors |= 1u; continue; }
#pragma unroll
      for (int p = 0; p < 4; p++) {
        const int ap = a0 + p * nc;
        const uint4 a = qs[ap >= all ? ap - all : ap];
        wins.w[2 * p] |= a.x;
        wins.w[2 * p + 1] |= a.y;
        not_loss.w[2 * p] |= a.z;
        not_loss.w[2 * p + 1] |= a.w;
      }
    }
  }
  const super8 immediate = s_or(wins0, wins1);
  super8 r0 = s_or(s_andnot(wins, immediate), s_andnot(wins0, wins1));
  super8 r1 = s_or(s_andnot(not_loss, immediate), wins0);
  s_line_frame<DIM>(r0);
  s_line_frame<DIM>(r1);
  if (accumulate) {
    r0 = s_or(wide ? s_load32(out) : s_load(out), r0);
    r1 = s_or(wide ? s_load32(out + 4) : s_load(out + 4), r1);
  }
  if (wide) {
    s_store32(out, r0);
    s_store32(out + 4, r1);
  } else {
    s_store(out, r0);
    s_store(out + 4, r1);
  }
}

// The subset tables of one side of a microline (sd: that side's stones in
// the fixed quadrants), built by one warp: lane t < 17 computes term t,
// lanes 17-31 the patterns that miss the line quadrant (ORed into c0).
template<int DIM>
__device__ __forceinline__ void warp_tables(const line_dev_t& L, const uint4* xe, uint2* tab, int lane) {
  const uint64_t f = lane_factor<DIM>(L, xe, lane);
  uint64_t c0 = lane < kTerms ? 0 : f;
#pragma unroll
  for (int o = 16; o; o >>= 1) c0 |= __shfl_xor_sync(0xffffffffu, c0, o);
#pragma unroll
  for (int j = 0; j < (kTab + 31) / 32; j++) {
    const int e = lane + 32 * j, c = table_chunk(e), sub = e - 16 * c;
    uint64_t v = c ? 0 : c0;
#pragma unroll
    for (int b = 0; b < 5; b++) {
      const uint64_t fb = __shfl_sync(0xffffffffu, f, 4 * c + b < kTerms ? 4 * c + b : 0);
      if (sub >> b & 1) v |= fb;
    }
    if (e < kTab) tab[e] = make_uint2(uint32_t(v), uint32_t(v >> 32));
  }
}

constexpr int kLineThreads = 256;
// CTAs per SM the line kernels are compiled for (64 registers a thread): a
// CTA's set-up and phase changes are latency chains, which other CTAs cover.
constexpr int kLineCtasPerSm = 4;
// 16-byte asynchronous copies from global to shared memory (no registers
// held while they fly); a thread waits only for its own.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned a = unsigned(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ void record_errors(unsigned e);

// Static shared memory of a CTA of MICRO microlines: per microline its
// geometry, the mover's subset tables (the children and the 35-stone parents
// evaluate them again) and its cross records ([microline][side][cross
// quadrant]).
template<int MICRO> struct cta_smem {
  micro_ctx ctx[MICRO];
  uint2 tab[MICRO][kTab];
  uint4 xs[MICRO][2][3];
};

// Stage the cross records of microlines m0 .. m0 + M - 1 (6 per microline).
template<int DIM, int MICRO>
__device__ __forceinline__ void stage_cross(const line_dev_t& L, cta_smem<MICRO>& S, int m0, int M, int tid) {
  if (tid < 6 * M) {
    const int k = tid / 6, r = tid - 6 * k, side = r / 3, c = r - 3 * side;
    int xq[4];
    cross_index<DIM>(L, m0 + k, xq);
    cp_async16(&S.xs[k][side][c], cross_entry<DIM>(L, xq, side, c));
  }
  cp_async_commit();
}

// Dynamic shared memory of a CTA of `micro` microlines: the stone-pattern
// results of every microline (micro x 4 pp uint2), the pattern set-up (the
// covered terms of every pattern class, pp uint4, and the opponent's subset
// tables, micro x kTab uint2), then the children (micro x 4 nchild uint4).
// The set-up has its own space, so patterns and children are computed in one
// phase.  Sized per launch for its largest line.
PG_HD size_t pattern_bytes(int pp, int micro) { return size_t(micro) * pp * 32; }
PG_HD size_t setup_bytes(int pp, int micro) { return size_t(pp) * 16 + size_t(micro) * kTab * 8; }
inline size_t line_smem_bytes(int pp, int nchild, int micro) {
  return pattern_bytes(pp, micro) + setup_bytes(pp, micro) + size_t(micro) * nchild * 64;
}
const size_t kMaxLineSmem = line_smem_bytes(2 * kMaxPat, kMaxLine, 4);

// Microlines per CTA for a launch whose lines have at most np parents, pp
// pattern classes and nc children per microline: 8 when a microline is short
// (so a CTA's threads have about as many parents as on long lines, and its
// set-up is spread over as much work) and 8 still fit 4 CTAs to an SM, else 4.
inline int line_micro(int np, int pp, int nc) {
  return np <= 192 && line_smem_bytes(pp, nc, 8) <= (size_t(48) << 10) ? 8 : 4;
}

// Microlines m0 .. m0 + M - 1 (M <= MICRO) of a line.  Set-up: the covered
// terms of the pattern classes and the microlines' cross records are staged,
// and the microlines' addressing worked out (no loads); barrier; each
// thread's first child requested, and warp w builds the subset tables of
// side w & 1 of microline w >> 1 (and w + 8 and so on) from the staged
// records; barrier; super_wins of every pattern class, then all children
// into shared memory; each thread's first parent record requested; barrier;
// all parents.
template<int DIM, int G, int MICRO>
__device__ __forceinline__ void cta_microlines(const line_dev_t& L, cta_smem<MICRO>& S, uint4* dyn, int m0, int M,
                                               int tid, int nt) {
  const int nc = L.nchild, np = L.nparent;
  const int p0 = L.npat[0], pp = p0 + L.npat[1];
  uint2* pats = reinterpret_cast<uint2*>(dyn);         // microline k at 4 pp k
  uint4* psub = dyn + MICRO * 2 * pp;                  // pattern set-up
  uint2* tab1 = reinterpret_cast<uint2*>(psub + pp);   // opponent's tables, microline k at kTab k
  uint4* q_smem = psub + pp + MICRO * kTab / 2;        // microline k at 4 nc k
  const int warp = tid >> 5, lane = tid & 31;
  const child_src C = child_source(L);
  const uint4* crecs = reinterpret_cast<const uint4*>(L.crecs);
  const uint4* recs = reinterpret_cast<const uint4*>(L.recs);
  const uint32_t mc = L.split_m[1];
  stage_cross<DIM>(L, S, m0, M, tid);
  for (int x = tid; x < pp; x += nt) psub[x] = ldg(reinterpret_cast<const uint4*>(L.precs) + x);
  // The last warp's first M lanes work out the microlines' addressing while
  // the records fly.
  if (tid >= nt - 32 && lane < M) S.ctx[lane].G = microline_addressing<DIM>(L, m0 + lane);
  cp_async_wait_all();
  __syncthreads();
  // Each thread's first child half is requested before the tables are built
  // and the patterns evaluated; adjacent threads take the two halves of a
  // child.
  const int half = tid & 1;
  super8 cx;
  uint4 cs = make_uint4(0, 0, 0, 0);
  const bool children = !L.slice35 && tid < 2 * M * nc;
  if (children) {
    int k, j;
    split(tid >> 1, nc, mc, k, j);
    cx = child_load(C, child_addr(C, S.ctx[k].G, j) + 4 * (1 - half));
    cs = ldg(crecs + j);
  }
  for (int w = warp; w < 2 * M; w += nt >> 5) {
    const int k = w >> 1;
    warp_tables<DIM>(L, S.xs[k][w & 1], w & 1 ? tab1 + k * kTab : S.tab[k], lane);
  }
  __syncthreads();
  for (int x = tid; x < M * pp; x += nt) {
    int k, e;
    split(x, pp, L.split_m[2], k, e);
    const super8 w = table_eval(e >= p0 ? tab1 + k * kTab : S.tab[k], psub[e]);
    pattern_store(pats + 4 * pp * k, e, pp, w);
  }
  if (children) {
    // Each thread's next child half is loaded while it transforms the
    // current one (nt is even, so a thread keeps its half).
    for (int x = tid; x < 2 * M * nc; x += nt) {
      int k, j;
      split(x >> 1, nc, mc, k, j);
      const super8 v = cx;
      const uint4 s = cs;
      if (x + nt < 2 * M * nc) {
        int kn, jn;
        split((x + nt) >> 1, nc, mc, kn, jn);
        cx = child_load(C, child_addr(C, S.ctx[kn].G, jn) + 4 * (1 - half));
        cs = ldg(crecs + jn);
      }
      child_half<DIM, G>(L, S.ctx[k].G, S.tab[k], reinterpret_cast<uint2*>(q_smem + 4 * k * nc), j, nc, half, v, s);
    }
  }
  // Each thread's first record header is requested before the barrier, the
  // next one while it computes the current parent.
  uint4 h = make_uint4(0, 0, 0, 0);
  if (tid < M * np) {
    int k, i;
    split(tid, np, L.split_m[0], k, i);
    h = ldg(recs + 3 * i);
  }
  __syncthreads();
  unsigned errors = 0;
  for (int x = tid; x < M * np; x += nt) {
    int k, i;
    split(x, np, L.split_m[0], k, i);
    const uint4 a = h;
    if (x + nt < M * np) {
      int kn, in;
      split(x + nt, np, L.split_m[0], kn, in);
      h = ldg(recs + 3 * in);
    }
    parent_node<DIM>(L, S.ctx[k].G, S.tab[k], q_smem + 4 * k * nc, pats + 4 * pp * k, a, recs + 3 * i, i, &errors);
  }
  if (errors) record_errors(errors);
}

// One CTA computes MICRO consecutive microlines of one line (fewer at the
// line's end).  All lines of a launch have line axis DIM and children
// standardized by global symmetry G.
template<int DIM, int G, int MICRO>
__global__ void __launch_bounds__(kLineThreads, kLineCtasPerSm)
end_line_kernel(const line_dev_t* __restrict__ lines, const dev_tables_t T) {
  const line_dev_t& D = lines[blockIdx.y];
  const int nmicro = D.cross[0] * D.cross[1] * D.cross[2];
  const int m0 = blockIdx.x * MICRO;
  if (m0 >= nmicro) return;
  // The descriptor is read throughout; shared memory keeps those reads short.
  __shared__ __align__(16) line_dev_t L;
  __shared__ cta_smem<MICRO> S;
  extern __shared__ uint4 dyn_smem[];
  {
    const uint4* src = reinterpret_cast<const uint4*>(&D);
    uint4* dst = reinterpret_cast<uint4*>(&L);
    for (int i = threadIdx.x; i < int(sizeof(line_dev_t) / 16); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  cta_microlines<DIM, G, MICRO>(L, S, dyn_smem, m0, min(MICRO, nmicro - m0), threadIdx.x, blockDim.x);
}

// The same microline code run sequentially on the host, for CPU self-tests of
// the kernel arithmetic.  Never used by the device entry points.
template<int DIM, int G> static unsigned host_line(const line_dev_t& L, const dev_tables_t& T) {
  const int pp = L.npat[0] + L.npat[1];
  std::vector<uint4> q(4 * std::max(L.nchild, 1));
  std::vector<uint2> pat(4 * std::max(pp, 1));
  unsigned errors = 0;
  uint2 fterm[kTerms], tab[2][kTab];
  for (int m = 0; m < L.cross[0] * L.cross[1] * L.cross[2]; m++) {
    const microline_geom geom = microline_addressing<DIM>(L, m);
    int xq[4];
    cross_index<DIM>(L, m, xq);
    for (int side = 0; side < 2; side++) {
      uint4 xe[3];
      for (int c = 0; c < 3; c++) xe[c] = *cross_entry<DIM>(L, xq, side, c);
      uint64_t c0 = 0;
      for (int u = 0; u < 15; u++) c0 |= lane_factor<DIM>(L, xe, kTerms + u);
      for (int t = 0; t < kTerms; t++) {
        const uint64_t f = lane_factor<DIM>(L, xe, t);
        fterm[t] = make_uint2(uint32_t(f), uint32_t(f >> 32));
      }
      for (int e = 0; e < kTab; e++) tab[side][e] = table_entry(fterm, c0, e);
      for (int r = 0; r < L.npat[side]; r++) {
        const int e = side ? L.npat[0] + r : r;
        const super8 w = table_eval(tab[side], reinterpret_cast<const uint4*>(L.precs)[e]);
        pattern_store(pat.data(), e, pp, w);
      }
    }
    if (!L.slice35)
      for (int j = 0; j < L.nchild; j++) {
        const uint64_t* a = child_addr(child_source(L), geom, j);
        for (int half = 0; half < 2; half++)
          child_half<DIM, G>(L, geom, tab[0], reinterpret_cast<uint2*>(q.data()), j, L.nchild, half,
                             s_load_ldg(a + 4 * (1 - half)), reinterpret_cast<const uint4*>(L.crecs)[j]);
      }
    for (int i = 0; i < L.nparent; i++) {
      const uint4* rp = reinterpret_cast<const uint4*>(L.recs + i);
      parent_node<DIM>(L, geom, tab[0], q.data(), pat.data(), rp[0], rp, i, &errors);
    }
  }
  return errors;
}

// The records of the (section, dimension) pairs of a set of lines, back to
// back in one buffer of 16-byte words (each pair once).
// Where the records of one (section, dimension) start, in 16-byte words.
struct rec_loc {
  size_t parent, child, cross, cls;
  int32_t xoff[4];
};

struct record_set {
  std::vector<uint4> words;
  std::vector<std::pair<uint64_t, rec_loc>> seen;
  rec_loc add(uint64_t section, int dim) {
    const uint64_t key = section << 2 | uint64_t(dim);
    for (const auto& kv : seen) if (kv.first == key) return kv.second;
    line_rec_set R;
    line_records(section, dim, R);
    rec_loc at;
    auto put = [&](const void* p, size_t n16) {
      const size_t o = words.size();
      const uint4* w = static_cast<const uint4*>(p);
      words.insert(words.end(), w, w + n16);
      return o;
    };
    at.parent = put(R.recs.data(), 3 * R.recs.size());
    at.child = put(R.crecs.data(), R.crecs.size());
    at.cross = put(R.xrecs.data(), R.xrecs.size());
    at.cls = put(R.precs.data(), R.precs.size());
    for (int q = 0; q < 4; q++) at.xoff[q] = R.xoff[q];
    seen.emplace_back(key, at);
    return at;
  }
};

static void bind_line_records(line_dev_t& L, const uint4* base, const rec_loc& at) {
  L.recs = reinterpret_cast<const parent_rec*>(base + at.parent);
  L.crecs = reinterpret_cast<const child_rec*>(base + at.child);
  L.xrecs = reinterpret_cast<const cross_rec*>(base + at.cross);
  L.precs = reinterpret_cast<const class_rec*>(base + at.cls);
  for (int q = 0; q < 4; q++) L.xoff[q] = at.xoff[q];
}

// A set of planned lines, grouped by dimension, with their descriptors on the device.
struct end_plan {
  std::vector<line_dev_t> host[4];
  line_dev_t* dev[4] = {nullptr, nullptr, nullptr, nullptr};
  int maxchild[4] = {0, 0, 0, 0};
  int maxpat[4] = {0, 0, 0, 0};         // most stone-pattern classes (both sides) of a line
  int maxparent[4] = {0, 0, 0, 0};      // most parents of a microline
  int order[4] = {3, 2, 1, 0};          // launch order: longest CTAs (most parents per microline) first
  // records of every (section, dimension) used
  record_set recs;
  std::vector<rec_loc> rec_off[4];       // per planned line: where its records start
  uint4* recs_dev = nullptr;
  // When the dimensions' lines are independent (dims_independent), the
  // launches of all but the first dimension run on side streams, forked from
  // and joined back into the caller's stream.
  bool concurrent = false;
  cudaStream_t side[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t fork = nullptr, join[3] = {nullptr, nullptr, nullptr};
};

// Every (line axis, child symmetry) pair the kernels are instantiated for.
#define PG_FOR_DIM_G(X) \
  X(0, 0) X(0, 1) X(0, 2) X(0, 3) X(0, 4) X(0, 5) X(0, 6) X(0, 7) \
  X(1, 0) X(1, 1) X(1, 2) X(1, 3) X(1, 4) X(1, 5) X(1, 6) X(1, 7) \
  X(2, 0) X(2, 1) X(2, 2) X(2, 3) X(2, 4) X(2, 5) X(2, 6) X(2, 7) \
  X(3, 0) X(3, 1) X(3, 2) X(3, 3) X(3, 4) X(3, 5) X(3, 6) X(3, 7)

template<int DIM, int G, int MICRO> static int set_smem_attr() {
  return cudaFuncSetAttribute(end_line_kernel<DIM, G, MICRO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kMaxLineSmem) == cudaSuccess ? 0 : PG_ERR_CUDA;
}
template<int DIM, int G, int MICRO> static int set_smem_limit() {
  return per_device_once((const void*)&set_smem_attr<DIM, G, MICRO>, set_smem_attr<DIM, G, MICRO>);
}
// A launch of end_line_kernel<DIM, G, MICRO>.
template<int DIM, int G, int MICRO>
static int launch_lines(const line_dev_t* lines, int n, size_t smem, cudaStream_t stream, const dev_tables_t& T) {
  if (int rc = set_smem_limit<DIM, G, MICRO>()) return rc;
  end_line_kernel<DIM, G, MICRO><<<dim3(512 / MICRO, unsigned(n)), kLineThreads, smem, stream>>>(lines, T);
  return 0;
}

// The planned lines of one dimension, sorted by child symmetry: one launch
// per symmetry, so each kernel holds only its own children's transform.
static int launch_group(const end_plan& P, int dim, cudaStream_t stream, const dev_tables_t& T) {
  const int n = int(P.host[dim].size());
  const int micro = line_micro(P.maxparent[dim], P.maxpat[dim], P.maxchild[dim]);
  const size_t smem = line_smem_bytes(P.maxpat[dim], P.maxchild[dim], micro);
  for (int a = 0, b = 0; a < n; a = b) {
    const int g = P.host[dim][a].g;
    while (b < n && P.host[dim][b].g == g) b++;
    const line_dev_t* lines = P.dev[dim] + a;
    int rc = PG_ERR_ARG;
    switch (dim * 8 + g) {
#define PG_CASE(D, G) case D * 8 + G: \
      rc = micro == 8 ? launch_lines<D, G, 8>(lines, b - a, smem, stream, T) \
                      : launch_lines<D, G, 4>(lines, b - a, smem, stream, T); \
      break;
      PG_FOR_DIM_G(PG_CASE)
#undef PG_CASE
    }
    if (rc) return fail(rc, "cudaFuncSetAttribute failed");
    PG_CUDA(cudaGetLastError());
  }
  return PG_OK;
}

static line_in_t to_in(const pg_line_t& l) {
  line_in_t in;
  in.section = l.section;
  in.dim = l.dimension;
  in.length = l.length;
  for (int i = 0; i < 3; i++) in.block_base[i] = l.block_base[i];
  in.flags = l.flags;
  in.input = l.input;
  in.output = l.output;
  in.input_offsets = l.input_block_offsets;
  in.output_offsets = l.output_block_offsets;
  in.input_stride = l.input_block_stride;
  in.output_stride = l.output_block_stride;
  return in;
}

}  // namespace pg

using namespace pg;

extern "C" int pg_line_info(const pg_line_t* line, pg_line_info_t* info) {
  if (!line || !info) return fail(PG_ERR_ARG, "null argument");
  line_shapes_t s;
  std::string err;
  if (!line_shapes(to_in(*line), s, err)) return fail(PG_ERR_ARG, err);
  info->input_nodes = int64_t(s.in_shape[0]) * s.in_shape[1] * s.in_shape[2] * s.in_shape[3];
  info->output_nodes = int64_t(s.out_shape[0]) * s.out_shape[1] * s.out_shape[2] * s.out_shape[3];
  info->input_blocks = s.input_blocks;
  info->block_stride = s.block_stride;
  info->child_section = s.child_std.sig();
  info->child_dimension = s.child_dim;
  for (int i = 0; i < 4; i++) { info->input_shape[i] = s.in_shape[i]; info->output_shape[i] = s.out_shape[i]; }
  return PG_OK;
}

static int plan_lines(const pg_line_t* lines, int n, end_plan& P) {
  std::string err;
  for (int i = 0; i < n; i++) {
    line_dev_t d;
    if (!plan_line(to_in(lines[i]), d, err)) return fail(PG_ERR_ARG, "line " + std::to_string(i) + ": " + err);
    if (!d.output || (!d.slice35 && !d.input)) return fail(PG_ERR_ARG, "null line buffer");
    const auto off = P.recs.add(lines[i].section, lines[i].dimension);
    P.maxchild[d.dim] = std::max(P.maxchild[d.dim], d.nchild);
    P.maxpat[d.dim] = std::max(P.maxpat[d.dim], d.npat[0] + d.npat[1]);
    P.maxparent[d.dim] = std::max(P.maxparent[d.dim], d.nparent);
    P.host[d.dim].push_back(d);
    P.rec_off[d.dim].push_back(off);
  }
  for (int dim = 0; dim < 4; dim++) {
    std::vector<size_t> order(P.host[dim].size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return P.host[dim][a].g < P.host[dim][b].g; });
    std::vector<line_dev_t> h;
    std::vector<rec_loc> r;
    for (size_t i : order) { h.push_back(P.host[dim][i]); r.push_back(P.rec_off[dim][i]); }
    P.host[dim].swap(h);
    P.rec_off[dim].swap(r);
  }
  std::stable_sort(P.order, P.order + 4, [&](int a, int b) { return P.maxparent[a] > P.maxparent[b]; });
  return PG_OK;
}

// Point every planned line at its records, given their device copy.
// Byte range [lo, hi) that a line's blocks can touch in one of its buffers:
// block b at node offset off[b] holds the cross-section's nodes times 8 along
// the line (fewer in the last block, `last` nodes along the line).
static void line_span(const void* base, const int64_t* off, int nblocks, int64_t cross, int last,
                      uintptr_t& lo, uintptr_t& hi) {
  int64_t a = off[0], b = 0;
  for (int i = 0; i < nblocks; i++) {
    a = std::min(a, off[i]);
    b = std::max(b, off[i] + cross * (i == nblocks - 1 ? last : 8));
  }
  lo = reinterpret_cast<uintptr_t>(base) + uintptr_t(a) * 64;
  hi = reinterpret_cast<uintptr_t>(base) + uintptr_t(b) * 64;
}

// Whether the launches of different dimensions may run at the same time: no
// line ORs into its output, and no line's output range meets a range (input
// or output) of a line of another dimension.  Plans of more than 4096 lines
// are not checked and run one dimension after another.
static bool dims_independent(const end_plan& P) {
  struct span_t { uintptr_t lo, hi; int dim; bool out; };
  std::vector<span_t> v;
  for (int d = 0; d < 4; d++)
    for (const line_dev_t& L : P.host[d]) {
      if (L.flags & PG_LINE_OR) return false;
      const int64_t cross = int64_t(L.cross[0]) * L.cross[1] * L.cross[2];
      span_t s{0, 0, d, true};
      line_span(L.output, L.out_off, L.length, cross, (L.nparent & 7) ? (L.nparent & 7) : 8, s.lo, s.hi);
      v.push_back(s);
      if (!L.slice35) {
        span_t t{0, 0, d, false};
        line_span(L.input, L.in_off, L.input_blocks, cross, (L.nchild & 7) ? (L.nchild & 7) : 8, t.lo, t.hi);
        v.push_back(t);
      }
    }
  if (v.size() > 8192) return false;
  for (const span_t& a : v) {
    if (!a.out) continue;
    for (const span_t& b : v)
      if (b.dim != a.dim && a.lo < b.hi && b.lo < a.hi) return false;
  }
  return true;
}

static void release_plan(end_plan* P) {
  for (auto* d : P->dev) if (d) cudaFree(d);
  if (P->recs_dev) cudaFree(P->recs_dev);
  for (auto s : P->side) if (s) cudaStreamDestroy(s);
  for (auto e : P->join) if (e) cudaEventDestroy(e);
  if (P->fork) cudaEventDestroy(P->fork);
  delete P;
}

static void bind_records(end_plan& P, uint4* recs_dev) {
  P.recs_dev = recs_dev;
  for (int dim = 0; dim < 4; dim++)
    for (size_t k = 0; k < P.host[dim].size(); k++) bind_line_records(P.host[dim][k], recs_dev, P.rec_off[dim][k]);
}

extern "C" int pg_end_compute_lines(const pg_line_t* lines, int n, void* stream_) {
  if (n < 0 || (n && !lines)) return fail(PG_ERR_ARG, "bad line array");
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  cudaStream_t stream = (cudaStream_t)stream_;
  end_plan P;
  if (int rc = plan_lines(lines, n, P)) return rc;
  if (P.recs.words.empty()) return PG_OK;
  stream_scratch X(stream);
  const size_t rbytes = sizeof(uint4) * P.recs.words.size();
  uint4* recs = nullptr;
  PG_CUDA(X.alloc(&recs, rbytes));
  PG_CUDA(cudaMemcpyAsync(recs, P.recs.words.data(), rbytes, cudaMemcpyHostToDevice, stream));
  bind_records(P, recs);
  int rc = PG_OK;
  for (int dim = 0; dim < 4 && !rc; dim++) {
    if (P.host[dim].empty()) continue;
    const size_t bytes = sizeof(line_dev_t) * P.host[dim].size();
    PG_CUDA(X.alloc(&P.dev[dim], bytes));
    PG_CUDA(cudaMemcpyAsync(P.dev[dim], P.host[dim].data(), bytes, cudaMemcpyHostToDevice, stream));
    rc = launch_group(P, dim, stream, *T);
    P.dev[dim] = nullptr;  // released with the scratch, not by end_plan
  }
  return rc;
}

extern "C" int pg_end_plan_create(const pg_line_t* lines, int n, pg_end_plan_t* plan) {
  if (!plan || n < 0 || (n && !lines)) return fail(PG_ERR_ARG, "bad plan arguments");
  if (!device_tables()) return PG_ERR_CUDA;
  auto* P = new end_plan;
  if (int rc = plan_lines(lines, n, *P)) { delete P; return rc; }
  if (!P->recs.words.empty()) {
    const size_t rbytes = sizeof(uint4) * P->recs.words.size();
    uint4* recs = nullptr;
    cudaError_t e = cudaMalloc(&recs, rbytes);
    if (e == cudaSuccess) e = cudaMemcpy(recs, P->recs.words.data(), rbytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { if (recs) cudaFree(recs); delete P; return cuda_fail(e, "pg_end_plan_create"); }
    bind_records(*P, recs);
  }
  int ndims = 0;
  for (int dim = 0; dim < 4; dim++) {
    if (P->host[dim].empty()) continue;
    ndims++;
    const size_t bytes = sizeof(line_dev_t) * P->host[dim].size();
    cudaError_t e = cudaMalloc(&P->dev[dim], bytes);
    if (e == cudaSuccess) e = cudaMemcpy(P->dev[dim], P->host[dim].data(), bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      release_plan(P);
      return cuda_fail(e, "pg_end_plan_create");
    }
  }
  if (ndims > 1 && dims_independent(*P)) {
    cudaError_t e = cudaEventCreateWithFlags(&P->fork, cudaEventDisableTiming);
    for (int k = 0; k < ndims - 1 && e == cudaSuccess; k++) {
      e = cudaStreamCreateWithFlags(&P->side[k], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->join[k], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
      release_plan(P);
      return cuda_fail(e, "pg_end_plan_create");
    }
    P->concurrent = true;
  }
  *plan = reinterpret_cast<pg_end_plan_t>(P);
  return PG_OK;
}

extern "C" int pg_end_plan_run(pg_end_plan_t plan, void* stream_) {
  if (!plan) return fail(PG_ERR_ARG, "null plan");
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  const end_plan& P = *reinterpret_cast<end_plan*>(plan);
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!P.concurrent) {
    for (int dim = 0; dim < 4; dim++)
      if (int rc = launch_group(P, dim, stream, *T)) return rc;
    return PG_OK;
  }
  // One launch per dimension, each on its own stream, so that the tail of
  // one launch's last wave overlaps the next launch instead of idling SMs.
  // The dimensions with the longest CTAs go first, so that a step ends on
  // short CTAs.
  PG_CUDA(cudaEventRecord(P.fork, stream));
  int k = -1;
  for (int d = 0; d < 4; d++) {
    const int dim = P.order[d];
    if (P.host[dim].empty()) continue;
    if (k < 0) {
      if (int rc = launch_group(P, dim, stream, *T)) return rc;
    } else {
      PG_CUDA(cudaStreamWaitEvent(P.side[k], P.fork, 0));
      if (int rc = launch_group(P, dim, P.side[k], *T)) return rc;
      PG_CUDA(cudaEventRecord(P.join[k], P.side[k]));
      PG_CUDA(cudaStreamWaitEvent(stream, P.join[k], 0));
    }
    k++;
  }
  return PG_OK;
}

extern "C" int pg_end_plan_streams(pg_end_plan_t plan) {
  if (!plan) return fail(PG_ERR_ARG, "null plan");
  const end_plan& P = *reinterpret_cast<end_plan*>(plan);
  if (!P.concurrent) return 1;
  int n = 0;
  for (int dim = 0; dim < 4; dim++) n += !P.host[dim].empty();
  return n;
}

extern "C" int pg_end_plan_destroy(pg_end_plan_t plan) {
  if (!plan) return PG_OK;
  release_plan(reinterpret_cast<end_plan*>(plan));
  return PG_OK;
}

extern "C" int pg_selftest_end_lines_host(const pg_line_t* lines, int n) {
  const dev_tables_t T = host_tables_view();
  std::string err;
  unsigned errors = 0;
  for (int i = 0; i < n; i++) {
    line_dev_t d;
    if (!plan_line(to_in(lines[i]), d, err)) return fail(PG_ERR_ARG, err);
    record_set rs;
    const rec_loc at = rs.add(lines[i].section, lines[i].dimension);
    bind_line_records(d, rs.words.data(), at);
    switch (d.dim * 8 + d.g) {
#define PG_CASE(D, G) case D * 8 + G: errors |= host_line<D, G>(d, T); break;
      PG_FOR_DIM_G(PG_CASE)
#undef PG_CASE
    }
  }
  return errors ? fail(PG_ERR_BOUNDS, "bounds check failed") : PG_OK;
}

// Synchronize `stream` and report device-side bounds violations since the last check.
extern "C" int pg_end_check(void* stream) {
  PG_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  unsigned int e = 0, zero = 0;
  PG_CUDA(cudaMemcpyFromSymbol(&e, d_end_errors, sizeof e));
  PG_CUDA(cudaMemcpyToSymbol(d_end_errors, &zero, sizeof zero));
  return e ? fail(PG_ERR_BOUNDS, "device bounds check failed in the line kernel") : PG_OK;
}

extern "C" int pg_section_shape(uint64_t section, int32_t* shape4) {
  const section_t s = section_t::from_sig(section);
  if (!s.valid()) return fail(PG_ERR_ARG, "invalid section");
  int sh[4];
  s.shape(sh);
  for (int i = 0; i < 4; i++) shape4[i] = sh[i];
  return PG_OK;
}

extern "C" int pg_section_standardize(uint64_t section, uint64_t* standard, int32_t* transform) {
  const section_t s = section_t::from_sig(section);
  if (!s.valid()) return fail(PG_ERR_ARG, "invalid section");
  int g = 0;
  *standard = s.standardize(&g).sig();
  if (transform) *transform = g;
  return PG_OK;
}

// ---------------------------------------------------------------------------
// Unit-level superscore checks
// ---------------------------------------------------------------------------

namespace pg {
PG_HD void debug_super_one(int op, const uint64_t* in, const uint16_t* sym, uint64_t* out, int i, const uint32_t* wf) {
  super8 r;
  if (op == 3 || op == 4) {  // halfsupers: 3 = halfsuper_wins(side, parity = sym), 4 = rmax
    const half4 h = op == 3 ? s_split(s_super_wins(wf, in[i]), sym[i] & 1)
                            : h_rmax(h_from(reinterpret_cast<const uint4*>(in)[i]));
    reinterpret_cast<uint4*>(out)[i] = h_to(h);
    return;
  }
  if (op == 0) r = s_rmax(s_load(in + 4 * i));
  else if (op == 1) r = s_super_wins(wf, in[i]);
  else r = s_transform(s_load(in + 4 * i), sym[i] >> 8, sym[i] & 255);
  s_store(out + 4 * i, r);
}
__global__ void debug_super_kernel(int op, const uint64_t* in, const uint16_t* sym, uint64_t* out, int n,
                                   const uint32_t* wf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) debug_super_one(op, in, sym, out, i, wf);
}
}  // namespace pg

extern "C" int pg_selftest_super_host(int op, const uint64_t* in, const uint16_t* sym, uint64_t* out, int n) {
  if (op < 0 || op > 4 || n < 0) return fail(PG_ERR_ARG, "bad debug op");
  for (int i = 0; i < n; i++) debug_super_one(op, in, sym, out, i, &tables().win_factors[0][0][0]);
  return PG_OK;
}

extern "C" int pg_debug_super(int op, const uint64_t* in, const uint16_t* sym, uint64_t* out, int n, void* stream) {
  if (op < 0 || op > 4 || n < 0) return fail(PG_ERR_ARG, "bad debug op");
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  if (!n) return PG_OK;
  debug_super_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(op, in, sym, out, n, T->win_factors);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

// ===========================================================================
// Slice sweeps: every block line of every section of a slice, reading the
// child slice and writing the parent slice in place (the work of
// compute_lines + accumulate over a whole slice, mpi/flow.cc and
// end/block_store.cc:173-226, on one GPU).
//
// A slice is one tensor: its sections (standardized, sorted by sig) back to
// back, each section's blocks in row-major block order, each block row-major
// in its own shape.  Block offsets are arithmetic (blocks before b in row-major
// order hold sum_i prod_{j<i} s_j(b_j) * 8 b_i * prod_{j>i} S_j nodes, with S
// the section shape and s_j(k) = min(8, S_j - 8k)), so no offset tables exist.
//
// Lines of one (section, dimension) pair form a family that shares one
// prototype descriptor; a CTA fills in its line's block-dependent fields in
// shared memory and then runs the same microline code as pg_end_compute_lines.
// ===========================================================================

namespace pg {

struct alignas(16) family_t {
  line_dev_t proto;           // everything but the per-line fields
  int32_t pshape[4], cshape[4], bcount[4];
  int64_t parent_base, child_base;
  int32_t first_line, nlines;
  uint8_t xsym_full[4][kMaxLine];  // reflection local of every child rmin index (cross dims)
};

PG_HD int64_t block_offset(const int32_t* S, const int* b) {
  int64_t off = 0, before = 1;
  for (int i = 0; i < 4; i++) {
    int64_t after = 1;
    for (int j = i + 1; j < 4; j++) after *= S[j];
    off += before * 8 * b[i] * after;
    before *= std::min(8, S[i] - 8 * b[i]);
  }
  return off;
}

// Block coordinates of line t of a family (row-major over the other three
// block counts; 0 along the line); returns the line's microline count.
PG_HD int family_blocks(const family_t& F, int t, int* b) {
  const int dim = F.proto.dim;
  int od[3], k = 0;
  for (int i = 0; i < 4; i++) if (i != dim) od[k++] = i;
  b[od[2]] = t % F.bcount[od[2]];
  b[od[1]] = t / F.bcount[od[2]] % F.bcount[od[1]];
  b[od[0]] = t / (F.bcount[od[2]] * F.bcount[od[1]]);
  b[dim] = 0;
  int n = 1;
  for (int j = 0; j < 3; j++) n *= std::min(8, F.pshape[od[j]] - 8 * b[od[j]]);
  return n;
}

// Fill the per-line fields of a family member (line t of the family).
PG_HD void family_line(const family_t& F, int t, line_dev_t& L) {
  const int dim = F.proto.dim;
  int od[3], k = 0;
  for (int i = 0; i < 4; i++) if (i != dim) od[k++] = i;
  int b[4];
  family_blocks(F, t, b);
  for (int i = 0; i < 4; i++) {
    L.block0[i] = b[i];
    L.out_shape[i] = i == dim ? F.pshape[i] : std::min(8, F.pshape[i] - 8 * b[i]);
  }
  for (int j = 0; j < 3; j++) L.cross[j] = L.out_shape[od[j]];
  for (int i = 0; i < 4; i++) L.first_child_block[i] = b[L.perm[i]];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 8; j++) {
      const int idx = 8 * L.first_child_block[i] + j;
      L.xsym[i][j] = i == L.child_dim || idx >= kMaxLine ? 0 : F.xsym_full[i][idx];
    }
}

PG_HD void family_offsets(const family_t& F, line_dev_t& L, int start, int step) {
  int b[4];
  for (int k = start; k < L.length + L.input_blocks; k += step) {
    if (k < L.length) {
      for (int i = 0; i < 4; i++) b[i] = L.block0[i];
      b[L.dim] = k;
      L.out_off[k] = F.parent_base + block_offset(F.pshape, b);
    } else {
      const int kk = k - L.length;
      for (int i = 0; i < 4; i++) b[i] = L.first_child_block[i];
      b[L.child_dim] = kk;
      L.in_off[kk] = F.child_base + block_offset(F.cshape, b);
    }
  }
}

// One CTA computes MICRO microlines of one line of a family (a launch holds
// families whose lines take the same MICRO, line_micro).
template<int DIM, int G, int MICRO>
__global__ void __launch_bounds__(kLineThreads, kLineCtasPerSm)
sweep_kernel(const family_t* __restrict__ fams, int nfams, int line0, const dev_tables_t T) {
  __shared__ __align__(16) line_dev_t L;
  __shared__ cta_smem<MICRO> S;
  __shared__ int s_fam, s_nmicro;
  extern __shared__ uint4 dyn_smem[];
  const int tid = threadIdx.x, nt = blockDim.x;
  const int line = line0 + blockIdx.x;
  if (tid == 0) {
    int lo = 0, hi = nfams - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (fams[mid].first_line <= line) lo = mid; else hi = mid - 1;
    }
    s_fam = lo;
    int b[4];
    s_nmicro = family_blocks(fams[lo], line - fams[lo].first_line, b);
  }
  __syncthreads();
  // CTAs past a short line's last microline leave before any set-up
  if (int(blockIdx.y) * MICRO >= s_nmicro) return;
  const family_t& F = fams[s_fam];
  // copy the prototype (as 16-byte words) and fill in this line
  {
    const uint4* src = reinterpret_cast<const uint4*>(&F.proto);
    uint4* dst = reinterpret_cast<uint4*>(&L);
    for (int i = tid; i < int(sizeof(line_dev_t) / 16); i += nt) dst[i] = src[i];
  }
  __syncthreads();
  if (tid == 0) family_line(F, line - F.first_line, L);
  __syncthreads();
  family_offsets(F, L, tid, nt);
  __syncthreads();
  const int nmicro = L.cross[0] * L.cross[1] * L.cross[2];
  const int m0 = int(blockIdx.y) * MICRO;
  cta_microlines<DIM, G, MICRO>(L, S, dyn_smem, m0, min(MICRO, nmicro - m0), tid, nt);
}

static_assert(sizeof(line_dev_t) % 16 == 0 && alignof(line_dev_t) == 16, "line_dev_t copies as uint4");
static_assert(sizeof(family_t) % 16 == 0, "family_t array keeps proto 16-byte aligned");

template<int DIM, int G, int MICRO> static int sweep_smem_attr() {
  return cudaFuncSetAttribute(sweep_kernel<DIM, G, MICRO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kMaxLineSmem) == cudaSuccess ? 0 : PG_ERR_CUDA;
}
template<int DIM, int G, int MICRO> static int sweep_smem_limit() {
  return per_device_once((const void*)&sweep_smem_attr<DIM, G, MICRO>, sweep_smem_attr<DIM, G, MICRO>);
}
template<int DIM, int G, int MICRO>
static int launch_sweep(const family_t* fams, int nfams, int lines, int line0, size_t smem, cudaStream_t stream,
                        const dev_tables_t& T) {
  if (int rc = sweep_smem_limit<DIM, G, MICRO>()) return rc;
  sweep_kernel<DIM, G, MICRO><<<dim3(unsigned(lines), 512 / MICRO), kLineThreads, smem, stream>>>(fams, nfams, line0,
                                                                                                   T);
  return 0;
}

// Per-section (we-win, we-win-or-tie, total) counts over distinct positions
// (count_block_wins, end/block_store.cc:330-352, with popcounts_over_stabilizers,
// base/count.cc:235-261).  One CTA per block.
struct count_section_t {
  int32_t shape[4], bcount[4], rmin_off[4];
  int64_t base;        // node offset in the slice tensor
  int64_t first_block;  // prefix over sections
};

__global__ void __launch_bounds__(256)
count_kernel(const count_section_t* __restrict__ secs, int nsecs, const uint64_t* __restrict__ slice,
             unsigned long long* __restrict__ counts, const uint16_t* __restrict__ rmin_flat,
             const uint8_t* __restrict__ stab) {
  __shared__ int s_sec;
  __shared__ unsigned long long red[3][8];
  const int64_t blk = blockIdx.x;
  if (threadIdx.x == 0) {
    int lo = 0, hi = nsecs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (secs[mid].first_block <= blk) lo = mid; else hi = mid - 1;
    }
    s_sec = lo;
  }
  __syncthreads();
  const count_section_t& S = secs[s_sec];
  int64_t t = blk - S.first_block;
  int b[4], bs[4];
  for (int i = 3; i >= 0; i--) { b[i] = int(t % S.bcount[i]); t /= S.bcount[i]; }
  for (int i = 0; i < 4; i++) bs[i] = min(8, S.shape[i] - 8 * b[i]);
  const int nodes = bs[0] * bs[1] * bs[2] * bs[3];
  const uint64_t* data = slice + 8 * (S.base + block_offset(S.shape, b));
  unsigned long long c0 = 0, c1 = 0, c2 = 0;
  for (int n = threadIdx.x; n < nodes; n += blockDim.x) {
    int r = n, idx[4];
    for (int i = 3; i >= 0; i--) { idx[i] = r % bs[i]; r /= bs[i]; }
    int shift = 0;
    for (int q = 0; q < 4; q++) shift += stab[rmin_flat[S.rmin_off[q] + 8 * b[q] + idx[q]]];
    const uint4* p = reinterpret_cast<const uint4*>(data + 8 * int64_t(n));
    const uint4 w0 = p[0], w1 = p[1], n0 = p[2], n1 = p[3];
    const int pw = __popc(w0.x) + __popc(w0.y) + __popc(w0.z) + __popc(w0.w) + __popc(w1.x) + __popc(w1.y) +
                   __popc(w1.z) + __popc(w1.w);
    const int pn = __popc(n0.x) + __popc(n0.y) + __popc(n0.z) + __popc(n0.w) + __popc(n1.x) + __popc(n1.y) +
                   __popc(n1.z) + __popc(n1.w);
    c0 += pw >> shift;
    c1 += pn >> shift;
    c2 += 256 >> shift;
  }
  for (int o = 16; o; o >>= 1) {
    c0 += __shfl_xor_sync(0xffffffffu, c0, o);
    c1 += __shfl_xor_sync(0xffffffffu, c1, o);
    c2 += __shfl_xor_sync(0xffffffffu, c2, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[0][warp] = c0; red[1][warp] = c1; red[2][warp] = c2; }
  __syncthreads();
  if (threadIdx.x < 3) {
    unsigned long long s = 0;
    for (int w = 0; w < int(blockDim.x >> 5); w++) s += red[threadIdx.x][w];
    atomicAdd(counts + 3 * s_sec + threadIdx.x, s);
  }
}

static int64_t section_nodes(const section_t& s) {
  int sh[4];
  s.shape(sh);
  return int64_t(sh[0]) * sh[1] * sh[2] * sh[3];
}

// Build the family descriptor for (section, dim).
static bool make_family(const section_t& sec, int dim, int64_t parent_base, const uint64_t* child_sigs, int nchild_secs,
                        const int64_t* child_offsets, uint64_t* parent_slice, const uint64_t* child_slice, int flags,
                        family_t& F, std::string& err) {
  memset(&F, 0, sizeof F);
  line_in_t in;
  memset(&in, 0, sizeof in);
  in.section = sec.sig();
  in.dim = dim;
  int shape[4];
  sec.shape(shape);
  in.length = (shape[dim] + 7) / 8;
  in.flags = flags;
  in.output = parent_slice;
  in.input = child_slice;
  line_shapes_t s;
  if (!line_shapes(in, s, err)) return false;
  // child section base
  F.child_base = 0;
  if (sec.sum() < 35) {
    const uint64_t csig = s.child_std.sig();
    const uint64_t* it = std::lower_bound(child_sigs, child_sigs + nchild_secs, csig);
    if (it == child_sigs + nchild_secs || *it != csig) { err = "child section missing from the child slice"; return false; }
    F.child_base = child_offsets[it - child_sigs];
    s.child_std.shape(F.cshape);
  }
  // prototype: plan the line through block 0 and keep only family-wide fields
  if (!plan_line(in, F.proto, err)) return false;
  for (int i = 0; i < 4; i++) {
    F.pshape[i] = shape[i];
    F.bcount[i] = (shape[i] + 7) / 8;
  }
  F.parent_base = parent_base;
  F.nlines = 1;
  for (int i = 0; i < 4; i++) if (i != dim) F.nlines *= F.bcount[i];
  // reflection locals for every child rmin index of the cross dims
  if (s.st & 4) {
    const auto& T = tables();
    int perm[4];
    quadrant_permutation(invert_global(s.st), perm);
    for (int i = 0; i < 4; i++) {
      if (i == s.child_dim) continue;
      const int k = rmin_bucket(s.child_std.c[i][0], s.child_std.c[i][1]);
      const int n = T.rmin_off[k + 1] - T.rmin_off[k];
      for (int j = 0; j < n && j < kMaxLine; j++) {
        const uint16_t q = T.rmin_flat[T.rmin_off[k] + j];
        const int rq = T.pack[T.refl[T.unpack[q][0]]] + 2 * T.pack[T.refl[T.unpack[q][1]]];
        F.xsym_full[i][j] = uint8_t(sigma_apply(line_sigma(dim, F.proto.g), (T.rmin_inv[rq] & 3) << (2 * i)));
      }
    }
  }
  return true;
}

}  // namespace pg

extern "C" int pg_slice_layout(const uint64_t* sigs, int n, int64_t* offsets) {
  if (n < 0 || (n && (!sigs || !offsets))) return fail(PG_ERR_ARG, "bad slice layout arguments");
  int64_t off = 0;
  for (int i = 0; i < n; i++) {
    const section_t s = section_t::from_sig(sigs[i]);
    if (!s.valid()) return fail(PG_ERR_ARG, "invalid section");
    if (i && sigs[i] <= sigs[i - 1]) return fail(PG_ERR_ARG, "sections must be sorted by sig");
    offsets[i] = off;
    off += section_nodes(s);
  }
  offsets[n] = off;
  return PG_OK;
}

// The lines of a slice, or (one_child) only those that read child_sigs[0],
// every line then ORing into the parent slice.
// CTAs of the sweep kernel an SM holds at this dynamic shared memory (four at
// most, by registers): 228 KB per SM, each CTA also holding its static shared
// memory and 1 KB the hardware reserves.
static int sweep_ctas_per_sm(size_t dyn, int micro) {
  const size_t stat = micro == 8 ? sizeof(cta_smem<8>) : sizeof(cta_smem<4>);
  const size_t per = dyn + sizeof(line_dev_t) + stat + 64 + 1024;
  return int(std::max<size_t>(1, std::min<size_t>(kLineCtasPerSm, (size_t(228) << 10) / per)));
}

static int sweep_lines(const uint64_t* parent_sigs, int np, uint64_t* parent_slice, const uint64_t* child_sigs, int nc,
                       const uint64_t* child_slice, bool one_child, void* stream_) {
  if (np < 0 || nc < 0 || (np && (!parent_sigs || !parent_slice))) return fail(PG_ERR_ARG, "bad sweep arguments");
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  cudaStream_t stream = (cudaStream_t)stream_;
  std::vector<int64_t> poff(np + 1), coff(nc + 1);
  if (int rc = pg_slice_layout(parent_sigs, np, poff.data())) return rc;
  if (int rc = pg_slice_layout(child_sigs, nc, coff.data())) return rc;
  std::string err;
  for (int dim = 0; dim < 4; dim++) {
    std::vector<family_t> fams;
    record_set recs;
    std::vector<rec_loc> rec_off;
    for (int i = 0; i < np; i++) {
      const section_t sec = section_t::from_sig(parent_sigs[i]);
      if (sec.c[dim][0] + sec.c[dim][1] >= 9) continue;
      if (one_child && sec.child(dim).standardize(nullptr).sig() != child_sigs[0]) continue;
      int first = 0;
      while (sec.c[first][0] + sec.c[first][1] >= 9) first++;
      fams.emplace_back();
      family_t& F = fams.back();
      if (!make_family(sec, dim, poff[i], child_sigs, nc, coff.data(), parent_slice, child_slice,
                       dim == first && !one_child ? PG_LINE_STORE : PG_LINE_OR, F, err))
        return fail(PG_ERR_ARG, "section " + std::to_string(i) + ": " + err);
      rec_off.push_back(recs.add(sec.sig(), dim));
    }
    if (fams.empty()) continue;
    stream_scratch X(stream);
    const size_t rbytes = sizeof(uint4) * recs.words.size();
    uint4* recs_dev = nullptr;
    PG_CUDA(X.alloc(&recs_dev, rbytes));
    PG_CUDA(cudaMemcpyAsync(recs_dev, recs.words.data(), rbytes, cudaMemcpyHostToDevice, stream));
    for (size_t f = 0; f < fams.size(); f++) bind_line_records(fams[f].proto, recs_dev, rec_off[f]);
    // One launch per (microlines per CTA, occupancy class, child symmetry):
    // short lines go 8 microlines to a CTA (line_micro); a launch's shared
    // memory is sized for its largest line, so families whose lines fit more
    // CTAs on an SM do not run at the occupancy of the longest lines of the
    // dimension; and each kernel holds only its own children's transform.
    struct group_t { int micro, k, g; size_t first, count; int lines, maxchild, maxpat; };
    std::vector<size_t> order(fams.size());
    std::vector<int> klass(fams.size()), micro(fams.size());
    for (size_t f = 0; f < fams.size(); f++) {
      order[f] = f;
      const line_dev_t& D = fams[f].proto;
      const int pp = D.npat[0] + D.npat[1];
      micro[f] = line_micro(D.nparent, pp, D.nchild);
      klass[f] = kLineCtasPerSm - sweep_ctas_per_sm(line_smem_bytes(pp, D.nchild, micro[f]), micro[f]);
    }
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
      if (micro[a] != micro[b]) return micro[a] > micro[b];
      return klass[a] != klass[b] ? klass[a] < klass[b] : fams[a].proto.g < fams[b].proto.g;
    });
    std::vector<family_t> sorted;
    std::vector<group_t> groups;
    for (size_t f : order) {
      const family_t& F = fams[f];
      if (groups.empty() || groups.back().micro != micro[f] || groups.back().k != klass[f] ||
          groups.back().g != F.proto.g)
        groups.push_back(group_t{micro[f], klass[f], F.proto.g, sorted.size(), 0, 0, 0, 0});
      group_t& G = groups.back();
      sorted.push_back(F);
      sorted.back().first_line = G.lines;
      G.count++;
      G.lines += F.nlines;
      G.maxchild = std::max(G.maxchild, F.proto.nchild);
      G.maxpat = std::max(G.maxpat, F.proto.npat[0] + F.proto.npat[1]);
    }
    family_t* d = nullptr;
    PG_CUDA(X.alloc(&d, sizeof(family_t) * sorted.size()));
    PG_CUDA(cudaMemcpyAsync(d, sorted.data(), sizeof(family_t) * sorted.size(), cudaMemcpyHostToDevice, stream));
    for (const group_t& G : groups) {
      const size_t smem = line_smem_bytes(G.maxpat, G.maxchild, G.micro);
      for (int line0 = 0; line0 < G.lines; line0 += 1 << 30) {
        const int lines = std::min(G.lines - line0, 1 << 30);
        int rc = PG_ERR_ARG;
        switch (dim * 8 + G.g) {
#define PG_CASE(D, GG) case D * 8 + GG: \
          rc = G.micro == 8 ? launch_sweep<D, GG, 8>(d + G.first, int(G.count), lines, line0, smem, stream, *T) \
                            : launch_sweep<D, GG, 4>(d + G.first, int(G.count), lines, line0, smem, stream, *T); \
          break;
          PG_FOR_DIM_G(PG_CASE)
#undef PG_CASE
        }
        if (rc) return fail(rc, "cudaFuncSetAttribute failed");
        PG_CUDA(cudaGetLastError());
      }
    }
  }
  return PG_OK;
}

extern "C" int pg_end_sweep_slice(const uint64_t* parent_sigs, int np, uint64_t* parent_slice,
                                  const uint64_t* child_sigs, int nc, const uint64_t* child_slice, void* stream) {
  return sweep_lines(parent_sigs, np, parent_slice, child_sigs, nc, child_slice, false, stream);
}

extern "C" int pg_end_sweep_slice_child(const uint64_t* parent_sigs, int np, uint64_t* parent_slice,
                                        uint64_t child_section, const uint64_t* child_nodes, void* stream) {
  if (!child_nodes) return fail(PG_ERR_ARG, "null child section");
  const section_t c = section_t::from_sig(child_section);
  if (!c.valid() || c.standardize(nullptr).sig() != child_section) return fail(PG_ERR_ARG, "child section not standardized");
  return sweep_lines(parent_sigs, np, parent_slice, &child_section, 1, child_nodes, true, stream);
}

namespace pg {
static const uint8_t* stab_table() {
  static std::mutex m;
  static std::vector<uint8_t*> per_device;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lock(m);
  if (int(per_device.size()) <= dev) per_device.resize(dev + 1, nullptr);
  if (!per_device[dev]) {
    const auto& T = tables();
    std::vector<uint8_t> h(19683);
    for (int q = 0; q < 19683; q++) {  // log_count_local_stabilizers (base/count.cc:226-236)
      const uint16_t s0 = T.unpack[q][0], s1 = T.unpack[q][1];
      const uint16_t r0 = T.rot[s0][0], r1 = T.rot[s1][0];
      h[q] = (s0 == r0 && s1 == r1) ? 2 : (s0 == T.rot[r0][0] && s1 == T.rot[r1][0]) ? 1 : 0;
    }
    uint8_t* d = nullptr;
    if (cudaMalloc(&d, 19683) != cudaSuccess || cudaMemcpy(d, h.data(), 19683, cudaMemcpyHostToDevice) != cudaSuccess)
      return nullptr;
    per_device[dev] = d;
  }
  return per_device[dev];
}
}  // namespace pg

extern "C" int pg_section_counts(const uint64_t* sigs, int n, const uint64_t* slice, uint64_t* counts3, void* stream_) {
  if (n < 0 || (n && (!sigs || !slice || !counts3))) return fail(PG_ERR_ARG, "bad count arguments");
  const dev_tables_t* T = device_tables();
  const uint8_t* stab = stab_table();
  if (!T || !stab) return PG_ERR_CUDA;
  cudaStream_t stream = (cudaStream_t)stream_;
  std::vector<int64_t> off(n + 1);
  if (int rc = pg_slice_layout(sigs, n, off.data())) return rc;
  std::vector<count_section_t> secs(n);
  int64_t blocks = 0;
  for (int i = 0; i < n; i++) {
    const section_t s = section_t::from_sig(sigs[i]);
    count_section_t& c = secs[i];
    s.shape(c.shape);
    int64_t nb = 1;
    for (int q = 0; q < 4; q++) {
      c.bcount[q] = (c.shape[q] + 7) / 8;
      c.rmin_off[q] = tables().rmin_off[rmin_bucket(s.c[q][0], s.c[q][1])];
      nb *= c.bcount[q];
    }
    c.base = off[i];
    c.first_block = blocks;
    blocks += nb;
  }
  if (!n) return PG_OK;
  PG_CUDA(cudaMemsetAsync(counts3, 0, sizeof(uint64_t) * 3 * n, stream));
  stream_scratch X(stream);
  count_section_t* d = nullptr;
  PG_CUDA(X.alloc(&d, sizeof(count_section_t) * n));
  PG_CUDA(cudaMemcpyAsync(d, secs.data(), sizeof(count_section_t) * n, cudaMemcpyHostToDevice, stream));
  for (int64_t b0 = 0; b0 < blocks; b0 += int64_t(1) << 30) {
    // grid.x covers at most 2^30 blocks per launch; the kernel reads blockIdx.x only,
    // so sweeps with more blocks are split by section instead.
    if (blocks > (int64_t(1) << 30)) return fail(PG_ERR_ARG, "too many blocks in one count call");
    count_kernel<<<unsigned(blocks), 256, 0, stream>>>(d, n, slice, (unsigned long long*)counts3, T->rmin_flat, stab);
    PG_CUDA(cudaGetLastError());
  }
  return PG_OK;
}

// descendent_sections (end/sections.cc:18-49): the standardized sections that
// root depends on at `slice`, sorted by sig.  Returns the count (writes at
// most cap).
extern "C" int pg_descendent_sections(uint64_t root, int slice, uint64_t* sigs, int cap) {
  const section_t r = section_t::from_sig(root);
  if (!r.valid() || slice < r.sum() || slice > 35) return fail(PG_ERR_ARG, "bad root or slice");
  std::vector<uint64_t> seen, out, stack{root};
  while (!stack.empty()) {
    const section_t s = section_t::from_sig(stack.back()).standardize(nullptr);
    stack.pop_back();
    const uint64_t sig = s.sig();
    if (std::find(seen.begin(), seen.end(), sig) != seen.end()) continue;
    seen.push_back(sig);
    if (s.sum() == slice) out.push_back(sig);
    if (s.sum() < slice)
      for (int q = 0; q < 4; q++)
        if (s.c[q][0] + s.c[q][1] < 9) stack.push_back(s.child(q).sig());
  }
  std::sort(out.begin(), out.end());
  for (int i = 0; i < int(out.size()) && i < cap; i++) sigs[i] = out[i];
  return int(out.size());
}
