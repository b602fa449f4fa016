// The midsolve solve of one board, shared by the batch kernel (mid.cu) and
// the server kernel (serve.cu).  See mid.cu for the algorithm.
#pragma once
#include "superscore.cuh"
#include "tables.h"
#include "runtime.h"
#include "../../include/pentago_b200.h"
#include <cstring>
#include <string>

namespace pg {

// Tables the midsolve code reads: combinations[n][k] for n <= 18, k <= 10
// (mid/subsets.h:17-21), the 32 five-in-a-row masks, and the win factors.
struct mid_tables {
  const uint32_t (*choose)[11];
  const uint64_t* winpat;
  const uint32_t* wf;
};

PG_HD int choose_t(const uint32_t (*C)[11], int n, int k) {
  if (n < 0 || k < 0 || k > n) return 0;
  return int(C[n][k < n - k ? k : n - k]);
}

struct mid_grab { int ny, lo, size; };

struct mid_job_t {
  uint64_t side[2];
  uint32_t ply;
  int32_t spots;
  uint8_t empty[18];
  uint8_t pad[6];
  int32_t sets1p_off[20], wins1_off[20], cs1ps_off[20];
  mid_grab spaces[20];
  uint64_t* sets1p;       // global scratch
  uint4* wins1;           // 2 per entry: after, before
  uint16_t* cs1ps;
  uint4* workspace;       // global workspace, or null when it lives in shared memory
  pg_mid_values_t* out;
  int32_t ws_size;        // workspace entries, for bounds checks
  int32_t pad2;
};

static_assert(sizeof(mid_job_t) % 16 == 0, "mid_job_t is copied in 16-byte words");

struct set0_info {  // make_set0_info (mid/internal.h:174-259); 256 bytes
  uint4 wins0;
  uint16_t child_s0s[18];
  uint16_t offset0[90];
  uint8_t empty1[18];
  uint8_t pad[2];
};
static_assert(sizeof(set0_info) == 256, "set0_info layout");

// ---------------------------------------------------------------------------
// Subset ranking (mid/subsets.h:34-105)
// ---------------------------------------------------------------------------

// The index-th k-subset of [0,n) in large-entry-major order, 5 bits per entry.
PG_HD uint64_t unrank(const uint32_t (*C)[11], int n, int k, int index) {
  uint64_t set = 0;
  for (int i = k - 1; i >= 0; i--) {
    int j = i, base = 0;
    for (; j < n; j++) {
      const int next = base + choose_t(C, j, i);
      if (index < next) break;
      base = next;
    }
    set |= uint64_t(j) << (5 * i);
    index -= base;
  }
  return set;
}

PG_HD uint64_t set_side(const uint8_t* empty, int k, uint64_t set) {
  uint64_t s = 0;
  for (int i = 0; i < k; i++) s |= uint64_t(1) << empty[set >> (5 * i) & 0x1f];
  return s;
}

// ---------------------------------------------------------------------------
// Wins of one side: super_wins split by parity (halfsuper_wins, generated by
// pentago/base/precompute.cc:330-505; here computed from the full super).
// ---------------------------------------------------------------------------

PG_HD half4 h_wins(const uint32_t* wf, uint64_t side, int parity) {
  return s_split(s_super_wins(wf, side), parity);
}

PG_HD bool won(const uint64_t* pats, uint64_t side) {
  for (int i = 0; i < 32; i++)
    if ((side & pats[i]) == pats[i]) return true;
  return false;
}

// ---------------------------------------------------------------------------
// The per-board CTA kernel
// ---------------------------------------------------------------------------

constexpr int kMidThreads = 256;
constexpr int kSmemWorkspaceMax = 8400;  // bottleneck(10), in halfsupers

struct level_t {
  int n, k0, k1, spots, parity;
  uint64_t root0, root1;
  int nsets0, nsets1p;
};

PG_HD level_t make_level(const mid_job_t& J, const mid_tables& MT, int n) {
  level_t L;
  L.n = n;
  L.k0 = n >> 1;
  L.k1 = n - L.k0;
  L.spots = J.spots;
  L.parity = int((n + J.ply) & 1);
  L.root0 = J.side[(J.spots + n) & 1];
  L.root1 = J.side[(J.spots + n + 1) & 1];
  L.nsets0 = choose_t(MT.choose, J.spots, L.k0);
  L.nsets1p = choose_t(MT.choose, J.spots - L.k0, L.k1);
  return L;
}

// make_set0_info (mid/internal.h:174-259), in two parts that two threads
// may build side by side: part 1 the wins and child indices (and the free
// spots), part 2 the offsets (which recount the free spots for themselves);
// parts = 3 builds both.
PG_HD void build_set0(const mid_job_t& J, const mid_tables& MT, const level_t& L, int s0, set0_info& I0,
                      int parts = 3) {
  const uint64_t set0 = unrank(MT.choose, J.spots, L.k0, s0);
  const uint64_t side0 = L.root0 | set_side(J.empty, L.k0, set0);
  const uint64_t free_ = 0x01ff01ff01ff01ffull & ~side0;
  uint8_t empty1[18];
  int next = 0;
  for (int i = 0; i < J.spots; i++)
    if (free_ >> J.empty[i] & 1) empty1[next++] = uint8_t(i);
  if (parts & 1) {
    I0.wins0 = h_to(h_wins(MT.wf, side0, L.parity));
    for (int i = 0; i < next; i++) I0.empty1[i] = empty1[i];
    for (int i = 0; i < J.spots - L.k0; i++) {
      const int j = empty1[i] - i;
      int v = choose_t(MT.choose, empty1[i], j + 1);
      for (int a = 0; a < L.k0; a++) v += choose_t(MT.choose, int(set0 >> (5 * a) & 0x1f), a + (a >= j) + 1);
      I0.child_s0s[i] = uint16_t(v);
    }
  }
  if (parts & 2)
    for (int a = 0; a < L.k1; a++)
      for (int q = 0; q < J.spots - L.k0; q++) {
        int offset = a ? 0 : s0;
        for (int i = empty1[q] - q; i < L.k0; i++) {
          const int v = int(set0 >> (5 * i) & 0x1f);
          if (v > a) offset -= choose_t(MT.choose, v - a - 1, i);
        }
        I0.offset0[a * (J.spots - L.k0) + q] = uint16_t(offset);
      }
}

// inner (mid/internal.h:358-408)
// Returns false (and does nothing) if an index would leave the workspace.
PG_HD bool inner(const mid_job_t& J, const mid_tables& MT, const level_t& L, const set0_info& I0, int s1p,
                 int aggressive, const uint4* in, uint4* out, int in_ny, int out_ny, int in_size, int out_size,
                 uint4* results) {
  const int n = L.n, spots = L.spots, k0 = L.k0, k1 = L.k1;
  const uint64_t set1p = J.sets1p[J.sets1p_off[n] + s1p];
  const int turn_aggressive = aggressive ^ (n & 1);
  // Index arithmetic is mod 2^16 as in the reference: offset0 holds wrapped
  // negative offsets (mid/internal.h:372-381).
  uint32_t filled1p = 0;
  uint16_t s1 = 0, s0p = 0;
  for (int i = 0; i < k1; i++) {
    const int q = int(set1p >> (5 * i) & 0x1f);
    filled1p |= 1u << q;
    s1 = uint16_t(s1 + choose_t(MT.choose, I0.empty1[q], i + 1));
    s0p = uint16_t(s0p + I0.offset0[i * (spots - k0) + q]);
  }
  half4 us = (spots == n && !turn_aggressive) ? h_not(h_zero()) : h_zero();
  const uint16_t* cs = J.cs1ps + J.cs1ps_off[n] + s1p * (spots - k0);
  uint32_t unmoved = ~filled1p;
  for (int m = 0; m < spots - n; m++) {
    const int i = ctz32(unmoved);
    unmoved &= unmoved - 1;
    const int idx = int(I0.child_s0s[i]) * in_ny + cs[i];
    if (unsigned(idx) >= unsigned(in_size)) return false;
    us = h_or(us, h_from(in[idx]));
  }
  const uint4* w1 = J.wins1 + 2 * (J.wins1_off[n] + s1);
  const half4 after = h_from(w1[0]), before = h_from(w1[1]);
  const half4 wins0 = h_from(I0.wins0);
  const half4 inplay = h_not(h_or(wins0, after));
  const half4 mask = turn_aggressive ? h_not(after) : h_not(h_zero());
  us = h_or(h_and(inplay, us), h_and(wins0, mask));
  const int o = int(s1) * out_ny + s0p;
  if (unsigned(o) >= unsigned(out_size) || (n <= 1 && n + s1p >= 19)) return false;
  if (n <= 1) results[n + s1p] = h_to(us);
  out[o] = h_to(h_or(h_rmax(h_not(us)), before));
  return true;
}

// high_board_t helpers for the traversal (high/board.cc)
PG_HD uint64_t board_of(uint64_t s0, uint64_t s1) {
  uint64_t board = 0;
  for (int q = 0; q < 4; q++) {
    uint32_t quad = 0;
    for (int i = 8; i >= 0; i--) {
      const int j = 16 * q + i;
      quad = 3 * quad + uint32_t(s0 >> j & 1) + 2 * uint32_t(s1 >> j & 1);
    }
    board |= uint64_t(quad) << (16 * q);
  }
  return board;
}

PG_HD void rotate_sides(uint64_t* side, int q, int d) {
  for (int s = 0; s < 2; s++) {
    const uint32_t old = uint32_t(side[s] >> (16 * q)) & 0x1ff;
    uint32_t quad = 0;
    for (int i = 0; i < 9; i++)
      if (old >> i & 1) quad |= 1u << (4 - d * (3 * (i % 3) - i / 3 - 2));
    side[s] ^= uint64_t(old ^ quad) << (16 * q);
  }
}

// done_and_value (high/board.cc:20-29)
PG_HD bool done_value(const mid_tables& MT, const uint64_t* side, uint32_t ply, int* value) {
  const bool bw = won(MT.winpat, side[0]), ww = won(MT.winpat, side[1]);
  const int turn = int(ply >> 1 & 1);
  if (bw || ww) { *value = (bw && ww) ? 0 : (bw == !turn ? 1 : -1); return true; }
  if (ply == 72) { *value = 0; return true; }
  return false;
}

PG_HD int hbit(const uint4& h, int i) {
  const uint32_t w = i < 32 ? h.x : i < 64 ? h.y : i < 96 ? h.z : h.w;
  return int(w >> (i & 31) & 1);
}

PG_HD void append(pg_mid_values_t* out, uint64_t raw, int v) {
  const int k = out->size++;
  if (k < 163) { out->entries[k].raw = raw; out->entries[k].value = v; out->entries[k].pad = 0; }
}

// midsolve_traverse (midengine.cc:127-158), iteratively; supers[i] = (win, notlose)
PG_HD void traverse(const mid_job_t& J, const mid_tables& MT, const uint4* supers, pg_mid_values_t* out) {
  out->size = 0;
  out->pad = 0;
  uint64_t side[2] = {J.side[0], J.side[1]};
  const uint32_t ply = J.ply;
  auto middle_children = [&](const uint64_t* sd, uint32_t p, const uint4* r) {
    int best = -1;
    for (int s = 0; s < 8; s++) {
      const int q = s >> 1, d = (s & 1) ? -1 : 1;
      const int idx = ((d & 3) << (2 * q)) >> 1;
      const int v = hbit(r[0], idx) + hbit(r[1], idx) - 1;
      uint64_t rs[2] = {sd[0], sd[1]};
      rotate_sides(rs, q, d);
      append(out, board_of(rs[0], rs[1]) | uint64_t((p + 1) & 1) << 63, v);
      best = best > -v ? best : -v;
    }
    return best;
  };
  int value;
  if (done_value(MT, side, ply, &value)) {
  } else if (!(ply & 1)) {
    value = -1;
    const uint64_t empty = 0x01ff01ff01ff01ffull ^ side[0] ^ side[1];
    int s = 0;
    for (int bit = 0; bit < 64; bit++) {
      if (!(empty >> bit & 1)) continue;
      s++;
      uint64_t cs[2] = {side[0], side[1]};
      cs[(ply >> 1) & 1] |= uint64_t(1) << bit;
      const uint32_t cply = ply + 1;
      int cv;
      if (!done_value(MT, cs, cply, &cv)) cv = middle_children(cs, cply, supers + 2 * s);
      append(out, board_of(cs[0], cs[1]) | uint64_t(1) << 63, cv);
      value = value > cv ? value : cv;
    }
  } else {
    value = middle_children(side, ply, supers);
  }
  append(out, board_of(side[0], side[1]) | uint64_t(ply & 1) << 63, value);
}

#ifdef __CUDA_ARCH__
// traverse on one warp: the root's children (one per lane) at once, their
// records placed by a prefix sum over the lanes in the order traverse
// writes them.
__device__ void put_record(pg_mid_values_t* out, int k, uint64_t raw, int v) {
  if (k < 163) { out->entries[k].raw = raw; out->entries[k].value = v; out->entries[k].pad = 0; }
}
// The 8 rotation children of sd (8 records at out[at..]); returns their best value for the mover.
__device__ int middle_children_at(const uint64_t* sd, uint32_t p, const uint4* r, pg_mid_values_t* out, int at) {
  int best = -1;
  for (int s = 0; s < 8; s++) {
    const int q = s >> 1, d = (s & 1) ? -1 : 1;
    const int idx = ((d & 3) << (2 * q)) >> 1;
    const int v = hbit(r[0], idx) + hbit(r[1], idx) - 1;
    uint64_t rs[2] = {sd[0], sd[1]};
    rotate_sides(rs, q, d);
    put_record(out, at + s, board_of(rs[0], rs[1]) | uint64_t((p + 1) & 1) << 63, v);
    best = best > -v ? best : -v;
  }
  return best;
}
__device__ void traverse_warp(const mid_job_t& J, const mid_tables& MT, const uint4* supers, pg_mid_values_t* out,
                              int lane) {
  const unsigned full = 0xffffffffu;
  const uint64_t side[2] = {J.side[0], J.side[1]};
  const uint32_t ply = J.ply;
  int value = 0, total = 0;
  if (done_value(MT, side, ply, &value)) {
  } else if (!(ply & 1)) {
    // lane s: the s-th empty cell (at most 18)
    const uint64_t empty = 0x01ff01ff01ff01ffull ^ side[0] ^ side[1];
    const int nempty = __popcll(empty);
    int cnt = 0, cv = -1;
    uint64_t cs[2] = {side[0], side[1]};
    if (lane < nempty) {
      uint64_t e = empty;
      for (int i = 0; i < lane; i++) e &= e - 1;
      cs[(ply >> 1) & 1] |= e & (~e + 1);
      cnt = done_value(MT, cs, ply + 1, &cv) ? 1 : 9;
    }
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(full, incl, o);
      if (lane >= o) incl += v;
    }
    const int base = incl - cnt;
    total = __shfl_sync(full, incl, 31);
    if (lane < nempty) {
      if (cnt == 9) cv = middle_children_at(cs, ply + 1, supers + 2 * (lane + 1), out, base);
      put_record(out, base + cnt - 1, board_of(cs[0], cs[1]) | uint64_t(1) << 63, cv);
    }
    int v = cv;
    for (int o = 16; o; o >>= 1) {
      const int w = __shfl_xor_sync(full, v, o);
      v = v > w ? v : w;
    }
    value = v;
  } else {
    // lanes 0..7: the root's 8 rotation children
    int best = -1;
    if (lane < 8) {
      const int q = lane >> 1, d = (lane & 1) ? -1 : 1;
      const int idx = ((d & 3) << (2 * q)) >> 1;
      const int v = hbit(supers[0], idx) + hbit(supers[1], idx) - 1;
      uint64_t rs[2] = {side[0], side[1]};
      rotate_sides(rs, q, d);
      put_record(out, lane, board_of(rs[0], rs[1]) | uint64_t((ply + 1) & 1) << 63, v);
      best = -v;
    }
    for (int o = 16; o; o >>= 1) {
      const int w = __shfl_xor_sync(full, best, o);
      best = best > w ? best : w;
    }
    value = best;
    total = 8;
  }
  if (lane == 0) {
    put_record(out, total, board_of(side[0], side[1]) | uint64_t(ply & 1) << 63, value);
    out->size = total + 1;
    out->pad = 0;
  }
}
#endif

// The whole solve of one board by ncta groups of nt cooperating threads
// (thread tid of group cta).  `barrier` synchronizes one group, `gbarrier`
// all groups (with one group it is the same barrier).  Inside a level the
// (s0, s1p) items are split into one contiguous range per group, and each
// group builds the set0 rows of its own range; a level's output is read by
// the next level only after the all-group barrier.  Run with one group of one
// thread and no-op barriers it is the same computation done sequentially
// (used by the CPU self-test).  `raw` and `fault` are shared by the groups.
// Passes [pass0, pass1) are run (the two passes share nothing but the
// per-level tables); `finish` = false stops after them, leaving the records
// to a caller that gathers both passes' raw results.
template<class Barrier, class GridBarrier>
PG_HD void mid_board_body(const mid_job_t& J, const mid_tables& MT, set0_info* tiles, uint4* ws,
                          uint4 (*raw)[19], int* fault, int tid, int nt, int cta, int ncta, Barrier barrier,
                          GridBarrier gbarrier, uint4* dump = nullptr, int pass0 = 0, int pass1 = 2,
                          bool finish = true) {
  const int spots = J.spots;
  const int gtid = cta * nt + tid, gnt = ncta * nt;
  // Per-level tables, the same for both passes (midengine.cc:57-76, :101-107)
  for (int n = spots; n >= 0; n--) {
    const int k0 = n >> 1, k1 = n - k0;
    const int ns1p = choose_t(MT.choose, spots - k0, k1);
    for (int i = gtid; i < ns1p; i += gnt) J.sets1p[J.sets1p_off[n] + i] = unrank(MT.choose, spots - k0, k1, i);
    const int ns1 = choose_t(MT.choose, spots, k1);
    const int parity = int((n + J.ply) & 1);
    const uint64_t root1 = J.side[(spots + n + 1) & 1];
    for (int s = gtid; s < ns1; s += gnt) {
      const uint64_t side1 = root1 | set_side(J.empty, k1, unrank(MT.choose, spots, k1, s));
      const super8 w = s_super_wins(MT.wf, side1);
      J.wins1[2 * (J.wins1_off[n] + s)] = h_to(s_split(w, parity));
      J.wins1[2 * (J.wins1_off[n] + s) + 1] = h_to(s_split(w, !parity));
    }
  }
  gbarrier();
  for (int n = spots; n >= 0; n--) {  // make_cs1ps (mid/internal.h:135-150)
    const int k0 = n >> 1, k1 = n - k0;
    const int ns1p = choose_t(MT.choose, spots - k0, k1);
    const uint64_t* sp = J.sets1p + J.sets1p_off[n];
    for (int idx = gtid; idx < ns1p * (spots - k0); idx += gnt) {
      const int s1p = idx / (spots - k0), j = idx - s1p * (spots - k0);
      int c = s1p;
      for (int a = 0; a < k1; a++) {
        const int v = int(sp[s1p] >> (5 * a) & 0x1f);
        if (j < v) c -= choose_t(MT.choose, v - 1, a);
      }
      J.cs1ps[J.cs1ps_off[n] + idx] = uint16_t(c);
    }
  }
  gbarrier();

  for (int aggressive = pass0; aggressive < pass1; aggressive++) {
    for (int n = spots; n >= 0; n--) {
      const level_t L = make_level(J, MT, n);
      const mid_grab gi = J.spaces[n + 1], go = J.spaces[n];
      const uint4* in = ws + gi.lo;
      uint4* out = ws + go.lo;
      // This group's items [i0, i1) and the set0 rows they touch
      const int64_t total = int64_t(L.nsets0) * L.nsets1p;
      const int64_t i0 = total * cta / ncta, i1 = total * (cta + 1) / ncta;
      const int r0 = L.nsets1p ? int(i0 / L.nsets1p) : 0;
      const int r1 = L.nsets1p && i1 > i0 ? int((i1 - 1) / L.nsets1p) + 1 : r0;
      for (int base = r0; base < r1; base += kMidThreads) {
        const int rows = r1 - base < kMidThreads ? r1 - base : kMidThreads;
        if (nt >= 2 * rows) {  // spare threads: two per row, one part each
          if (tid < 2 * rows) build_set0(J, MT, L, base + (tid >> 1), tiles[tid >> 1], 1 + (tid & 1));
        } else {
          for (int r = tid; r < rows; r += nt) build_set0(J, MT, L, base + r, tiles[r]);
        }
        barrier();
        const int64_t a = i0 > int64_t(base) * L.nsets1p ? i0 : int64_t(base) * L.nsets1p;
        const int64_t b = i1 < int64_t(base + rows) * L.nsets1p ? i1 : int64_t(base + rows) * L.nsets1p;
        for (int64_t it = a + tid; it < b; it += nt) {
          const int row = int(it / L.nsets1p), s1p = int(it - int64_t(row) * L.nsets1p);
          if (!inner(J, MT, L, tiles[row - base], s1p, aggressive, in, out, gi.ny, go.ny, J.ws_size - gi.lo,
                     J.ws_size - go.lo, raw[aggressive]))
            *fault = 1;
        }
        barrier();
      }
      gbarrier();
    }
  }

  if (!finish) return;
  // Interleave (midengine.cc:119-124) and traverse; a failed bounds check
  // marks the record with size -1 instead.
  if (gtid == 0 && *fault) { J.out->size = -1; J.out->pad = 0; }
#ifdef __CUDA_ARCH__
  // the first warp traverses (nt >= 32 on the device)
  if (gtid < 32 && !*fault) {
    uint4 supers[2 * 19];
    for (int i = 0; i < 19; i++)
      for (int j = 0; j < 2; j++) supers[2 * i + j] = raw[j ^ (i == 0)][i];
    if (dump && gtid == 0)
      for (int i = 0; i < 38; i++) dump[i] = supers[i];
    traverse_warp(J, MT, supers, J.out, gtid);
  }
#else
  if (gtid == 0 && !*fault) {
    uint4 supers[2 * 19];
    for (int i = 0; i < 19; i++)
      for (int j = 0; j < 2; j++) supers[2 * i + j] = raw[j ^ (i == 0)][i];
    if (dump)
      for (int i = 0; i < 38; i++) dump[i] = supers[i];
    traverse(J, MT, supers, J.out);
  }
#endif
}


// Per translation unit: each .cu file that launches the body uploads these.
static __constant__ uint32_t c_choose[19][11];
static __constant__ uint64_t c_winpat[32];

struct sync_threads { __device__ void operator()() const { __syncthreads(); } };

// Barrier over the CTAs that solve one board together.  They are co-resident
// (a cooperative launch, or workers of the persistent server); the wait is bounded, and a timeout marks the board
// as failed and turns every later barrier of that board into a no-op, so the
// kernel always finishes.
constexpr unsigned kBarrierPolls = 1u << 28;  // about 20 s of 64 ns sleeps

struct board_barrier {
  unsigned* count;  // arrivals in the current generation
  unsigned* gen;    // generation number
  int ncta;
  int* fault;
  unsigned polls = kBarrierPolls;  // wait limit
  __device__ void operator()() const {
    __syncthreads();
    if (threadIdx.x == 0) {
      volatile unsigned* vg = gen;
      volatile int* vf = fault;
      const unsigned g = *vg;
      __threadfence();
      if (atomicAdd(count, 1u) == unsigned(ncta) - 1) {
        atomicExch(count, 0u);
        __threadfence();
        atomicAdd(gen, 1u);
      } else {
        for (unsigned i = 0; *vg == g && !*vf; i++) {
          if (i > polls) { atomicExch(fault, 1); break; }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
    __syncthreads();
  }
};


// ---------------------------------------------------------------------------
// Host helpers (mid.cu)
// ---------------------------------------------------------------------------

struct board_plan {
  mid_job_t job;
  size_t sets1p, wins1, cs1ps, workspace;  // element counts
};

int bottleneck(int spots);
int hchoose(int n, int k);
bool plan_board(uint64_t raw, board_plan& P, std::string& err);
// Device scratch the board needs, and pointing the job's tables into it.  The
// workspace is in global scratch when it does not fit shared memory, or
// always with global_ws.
size_t scratch_bytes_of(const board_plan& P, bool global_ws = false);
void carve_scratch(board_plan& P, char* base, bool global_ws = false);

// Upload this translation unit's constant tables (once per device).
static int mid_upload_constants() {
  uint32_t ch[19][11];
  for (int n = 0; n <= 18; n++)
    for (int k = 0; k <= 10; k++) ch[n][k] = uint32_t(hchoose(n, k));
  const tables_t& T = tables();
  if (cudaMemcpyToSymbol(c_choose, ch, sizeof ch) != cudaSuccess ||
      cudaMemcpyToSymbol(c_winpat, T.winpat, sizeof T.winpat) != cudaSuccess)
    return PG_ERR_CUDA;
  return PG_OK;
}
static int mid_prepare_device() { return per_device_once((const void*)&c_choose, mid_upload_constants); }

}  // namespace pg
