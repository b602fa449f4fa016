// Store coder: how the sweep keeps finished slices compressed in HBM.  No
// reference counterpart (the reference compresses blocks in memory with
// snappy, pentago/end/fast_compress.cc); this is an internal format that
// never leaves the device, so only its round trip is specified.
//
// A block of solved nodes is coded as the ternary symbols black wins + 2
// white wins of its 256 rotations per node (the on-disk convention), with
// static rANS (14-bit frequencies, byte renormalization at 2^23) whose
// frequencies depend on a context of five already-coded symbols: the same
// node one step back along each of the four rotation axes (3 where the
// coordinate is 0) and the same rotation of the previous node of the lane.
// One frequency table (1024 contexts x 3) serves a whole batch of blocks.
// A block's 32 lanes (one warp) each take a contiguous run of its nodes, so
// every context symbol is on the lane that codes the symbol and the lanes
// decode in parallel.  Stream layout: 32 lane lengths (u32), then the lanes'
// bytes; a block that some lane cannot code within its nodes' raw size is
// stored raw instead (first length ~0, then the 64-byte nodes), so a stream
// never needs more than its raw size plus 128 + 32 x 64 bytes.
#include "../../include/pentago_b200.h"
#include "runtime.h"
#include <cstdint>

namespace pg {
namespace {

constexpr int kCtx = 1024;
constexpr int kLanesS = 32;   // lanes per block: one warp
constexpr uint32_t kTotBits = 14, kTot = 1u << kTotBits, kLow = 1u << 23;
constexpr int kHead = 4 * kLanesS;
constexpr int kGroups = 4;   // streams per CTA of the coder kernels
constexpr int kThreads = kGroups * kLanesS;
// A batch's frequency table counts the contexts of at most this many of its
// blocks, spread evenly over it (about 2 G symbols for full blocks).
constexpr int kTableBlocks = 2048;

// Nodes per lane of a block of n nodes.
__host__ __device__ inline int lane_nodes(int n) { return (n + kLanesS - 1) / kLanesS; }
__host__ __device__ inline int64_t lane_cap(int n) { return int64_t(lane_nodes(n)) * 64 + 64; }
__host__ __device__ inline int64_t store_bound(int n) { return kHead + kLanesS * lane_cap(n); }

// Symbols of one node packed 2 bits each (16 per word, rotation r at bits
// 2 (r & 15) of word r >> 4): black bit + 2 white bit, for the side-to-move
// form [win, win or tie] of the sweep.
__device__ __forceinline__ uint32_t spread16(uint32_t x) {
  x &= 0xffffu;
  x = (x | x << 8) & 0x00ff00ffu;
  x = (x | x << 4) & 0x0f0f0f0fu;
  x = (x | x << 2) & 0x33333333u;
  return (x | x << 1) & 0x55555555u;
}
__device__ __forceinline__ uint32_t gather16(uint32_t x) {
  x &= 0x55555555u;
  x = (x | x >> 1) & 0x33333333u;
  x = (x | x >> 2) & 0x0f0f0f0fu;
  x = (x | x >> 4) & 0x00ff00ffu;
  return (x | x >> 8) & 0xffffu;
}
// A node's 16 symbol words live S words apart in shared memory: the coder
// threads keep theirs in columns (S = threads per CTA), so that a warp whose
// threads read the same word index reads 32 different banks.
template<int S>
__device__ __forceinline__ void pack_node(const uint64_t* node, int turn, uint32_t* sym) {
#pragma unroll
  for (int w = 0; w < 4; w++) {
    const uint64_t win = node[w], nl = node[4 + w];
    const uint64_t black = turn ? ~nl : win, white = turn ? win : ~nl;
#pragma unroll
    for (int h = 0; h < 4; h++)
      sym[S * (4 * w + h)] = spread16(uint32_t(black >> (16 * h))) | spread16(uint32_t(white >> (16 * h))) << 1;
  }
}
template<int S>
__device__ __forceinline__ int sym_at(const uint32_t* sym, int r) { return int(sym[S * (r >> 4)] >> (2 * (r & 15)) & 3); }

template<int S>
__device__ __forceinline__ int context(const uint32_t* cur, const uint32_t* prev, int r) {
  int c = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) c = 4 * c + ((r >> (2 * q) & 3) ? sym_at<S>(cur, r - (1 << (2 * q))) : 3);
  return 4 * c + (prev ? sym_at<S>(prev, r) : 3);
}

// The coder kernels take a node's symbols a word (16 rotations r = 16 w + i)
// at a time: the context fields of all 16 come from five words.  Axis 0's
// neighbour r - 1 and axis 1's r - 4 are symbols i - 1 and i - 4 of the same
// word (none where i % 4 == 0, resp. i < 4); axis 2's r - 16 and axis 3's
// r - 64 are words w - 1 and w - 4 (none where w % 4 == 0, resp. w < 4); the
// previous node's symbol is its word w.  A missing neighbour reads as 3.
constexpr uint32_t kNoAxis0 = 0x03030303u, kNoAxis1 = 0x000000ffu;
__device__ __forceinline__ int word_context(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t ap,
                                            int i) {
  return int((a0 >> (2 * i) & 3) << 8 | (a1 >> (2 * i) & 3) << 6 | (a2 >> (2 * i) & 3) << 4 |
             (a3 >> (2 * i) & 3) << 2 | (ap >> (2 * i) & 3));
}

// Frequencies of a context in one 8-byte shared-memory word: f0 | f1 << 16, f2.
__device__ __forceinline__ void load_freqs(const uint16_t* __restrict__ freq, uint2* F) {
  for (int c = threadIdx.x; c < kCtx; c += blockDim.x)
    F[c] = make_uint2(uint32_t(freq[3 * c]) | uint32_t(freq[3 * c + 1]) << 16, freq[3 * c + 2]);
}

// The encoder divides the state by a symbol's frequency f with a reciprocal
// multiply, as in F. Giesen's ryg_rans (after Alverson, "Integer division
// using reciprocals", 1991): with 2^(sh-1) < f <= 2^sh, rcp = ceil(2^(sh+31)
// / f) gives state / f = umulhi(state, rcp) >> (sh - 1) for every state below
// 2^31 (renormalization keeps it below 2^17 f <= 2^31).  f = 1 takes rcp =
// 2^32 - 1, shift 0 and a bias of 2^14 - 1, which yields the same new state.
// Per context: three reciprocals, and the three shifts in bits 16.. of F.y.
__device__ __forceinline__ void encoder_freqs(const uint16_t* __restrict__ freq, uint2* F, uint32_t* rcp) {
  for (int c = threadIdx.x; c < kCtx; c += blockDim.x) {
    uint32_t shifts = 0;
    for (int s = 0; s < 3; s++) {
      const uint32_t f = freq[3 * c + s];
      uint32_t sh = 0;
      while (f > (1u << sh)) sh++;
      rcp[3 * c + s] = f < 2 ? ~0u : uint32_t(((uint64_t(1) << (sh + 31)) + f - 1) / f);
      shifts |= (f < 2 ? 0u : sh - 1) << (4 * s);
    }
    F[c] = make_uint2(uint32_t(freq[3 * c]) | uint32_t(freq[3 * c + 1]) << 16, freq[3 * c + 2] | shifts << 16);
  }
}

// Context counts over every stride-th block of a batch: one CTA per block,
// thread r takes rotation r of every node in lane order.
__global__ void __launch_bounds__(256)
store_hist_kernel(const uint64_t* __restrict__ nodes, const int64_t* __restrict__ first,
                  const int32_t* __restrict__ count, int stride, int turn, unsigned* __restrict__ hist) {
  __shared__ unsigned h[kCtx * 3];
  __shared__ uint32_t cur[16], prev[16];
  for (int i = threadIdx.x; i < kCtx * 3; i += blockDim.x) h[i] = 0;
  const int b = blockIdx.x * stride, n = count[b], m = lane_nodes(n), r = threadIdx.x;
  const uint64_t* base = nodes + 8 * first[b];
  __syncthreads();
  for (int k = 0; k < n; k++) {
    if (r < 16) {
      const uint64_t* node = base + 8 * int64_t(k);
      const int w = r >> 2, hq = r & 3;
      const uint64_t win = node[w], nl = node[4 + w];
      const uint64_t black = turn ? ~nl : win, white = turn ? win : ~nl;
      cur[r] = spread16(uint32_t(black >> (16 * hq))) | spread16(uint32_t(white >> (16 * hq))) << 1;
    }
    __syncthreads();
    const int c = context<1>(cur, k % m ? prev : nullptr, r);
    atomicAdd(&h[3 * c + sym_at<1>(cur, r)], 1u);
    __syncthreads();
    if (r < 16) prev[r] = cur[r];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kCtx * 3; i += blockDim.x)
    if (h[i]) atomicAdd(hist + i, h[i]);
}

// Frequencies per context from its counts: proportional, at least 1, the
// rounding left on the largest (uniform when the context never occurs).
__global__ void store_table_kernel(const unsigned* __restrict__ hist, uint16_t* __restrict__ freq) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= kCtx) return;
  const uint64_t n[3] = {hist[3 * c], hist[3 * c + 1], hist[3 * c + 2]};
  const uint64_t sum = n[0] + n[1] + n[2];
  uint32_t f[3];
  if (!sum) {
    f[0] = kTot - 2 * (kTot / 3);
    f[1] = f[2] = kTot / 3;
  } else {
    for (int i = 0; i < 3; i++) {
      f[i] = uint32_t(n[i] * kTot / sum);
      if (!f[i]) f[i] = 1;
    }
    const int big = f[1] > f[0] ? (f[2] > f[1] ? 2 : 1) : (f[2] > f[0] ? 2 : 0);
    f[big] = uint32_t(int32_t(f[big]) + int32_t(kTot) - int32_t(f[0] + f[1] + f[2]));
  }
  for (int i = 0; i < 3; i++) freq[3 * c + i] = uint16_t(f[i]);
}

// Encode: one 8-lane group per block; lane l codes its run of nodes backward,
// each node's rotations from 255 to 0, into its own slot, then the lanes are
// packed behind the header.
__global__ void __launch_bounds__(kGroups * kLanesS)
store_encode_kernel(const uint64_t* __restrict__ nodes, const int64_t* __restrict__ first,
                    const int32_t* __restrict__ count, int nblocks, int turn, const uint16_t* __restrict__ freq,
                    uint8_t* __restrict__ out, const int64_t* __restrict__ out_offsets, int64_t* __restrict__ sizes) {
  __shared__ uint2 F[kCtx];
  __shared__ uint32_t RCP[kCtx * 3];
  __shared__ uint32_t buf[2 * 16][kThreads];
  encoder_freqs(freq, F, RCP);
  __syncthreads();
  const int g = threadIdx.x / kLanesS, lane = threadIdx.x % kLanesS;
  const int b = blockIdx.x * kGroups + g;
  if (b >= nblocks) return;
  constexpr unsigned gmask = 0xffffffffu;   // a block's lanes are one warp
  const int n = count[b], m = lane_nodes(n);
  const int k0 = lane * m, k1 = min(n, k0 + m);
  const uint64_t* base = nodes + 8 * first[b];
  uint8_t* sbase = out + out_offsets[b];
  const int64_t cap = lane_cap(n);
  uint8_t* slot_begin = sbase + kHead + lane * cap;
  uint8_t* slot_end = slot_begin + cap;
  uint8_t* p = slot_end;
  uint32_t state = kLow;
  int over = 0;
  uint32_t* cur = &buf[0][threadIdx.x];
  uint32_t* prev = &buf[16][threadIdx.x];
  if (k1 > k0) pack_node<kThreads>(base + 8 * int64_t(k1 - 1), turn, cur);
  for (int k = k1 - 1; k >= k0 && !over; k--) {
    const bool has_prev = k > k0;
    if (has_prev) pack_node<kThreads>(base + 8 * int64_t(k - 1), turn, prev);
    for (int w = 15; w >= 0 && !over; w--) {
      const uint32_t x = cur[kThreads * w];
      const uint32_t a0 = x << 2 | kNoAxis0, a1 = x << 8 | kNoAxis1;
      const uint32_t a2 = (w & 3) ? cur[kThreads * (w - 1)] : ~0u;
      const uint32_t a3 = w >= 4 ? cur[kThreads * (w - 4)] : ~0u;
      const uint32_t ap = has_prev ? prev[kThreads * w] : ~0u;
#pragma unroll
      for (int i = 15; i >= 0; i--) {
        const uint32_t sym = x >> (2 * i) & 3;
        const int c = word_context(a0, a1, a2, a3, ap, i);
        const uint2 fc = F[c];
        const uint32_t rcp = RCP[3 * c + sym];
        const uint32_t f0 = fc.x & 0xffffu, f1 = fc.x >> 16;
        const uint32_t f = sym == 0 ? f0 : sym == 1 ? f1 : fc.y & 0xffffu;
        const uint32_t cum = sym == 0 ? 0u : sym == 1 ? f0 : f0 + f1;
        const uint32_t xmax = ((kLow >> kTotBits) << 8) * f;
        while (state >= xmax) {
          if (p - slot_begin <= 4) { over = 1; break; }   // keep room for the final state
          *--p = uint8_t(state);
          state >>= 8;
        }
        if (over) break;
        const uint32_t q = __umulhi(state, rcp) >> (fc.y >> (16 + 4 * sym) & 15);
        state += cum + (f < 2 ? kTot - 1 : 0u) + q * (kTot - f);
      }
    }
    uint32_t* t = cur; cur = prev; prev = t;
  }
  if (__any_sync(gmask, over)) {
    // some lane would pass its nodes' raw size: store the block raw
    __syncwarp(gmask);
    const int64_t words = 8 * int64_t(n);
    for (int64_t i = lane; i < words; i += kLanesS)
      reinterpret_cast<uint64_t*>(sbase + kHead)[i] = base[i];
    if (lane == 0) {
      for (int j = 0; j < 4; j++) sbase[j] = 0xff;
      for (int j = 4; j < kHead; j++) sbase[j] = 0;
      sizes[b] = kHead + 8 * words;
    }
    return;
  }
  for (int j = 0; j < 4; j++) *--p = uint8_t(state >> (8 * j));
  const uint32_t len = uint32_t(slot_end - p);
  // Destination of this lane's bytes behind the header: the lengths of the
  // lanes before it (an exclusive warp scan), and the stream's total.
  uint32_t before = len;
#pragma unroll
  for (int o = 1; o < kLanesS; o <<= 1) {
    const uint32_t v = __shfl_up_sync(gmask, before, o);
    if (lane >= o) before += v;
  }
  const uint32_t total = __shfl_sync(gmask, before, kLanesS - 1);
  before -= len;
  // The lanes' bytes move left, one lane after another, the whole warp
  // copying 32 bytes a round; a round reads all its bytes before writing any.
  // A lane's destination never passes its own source (it moves left) nor a
  // later lane's source (each lane's bytes fit its slot).
  for (int l = 0; l < kLanesS; l++) {
    const uint32_t n_l = __shfl_sync(gmask, len, l);
    const int64_t dst_l = kHead + int64_t(__shfl_sync(gmask, before, l));
    const uint8_t* src_l = reinterpret_cast<const uint8_t*>(
        __shfl_sync(gmask, reinterpret_cast<unsigned long long>(p), l));
    for (uint32_t i0 = 0; i0 < n_l; i0 += kLanesS) {
      const uint32_t i = i0 + lane;
      const uint8_t v = i < n_l ? src_l[i] : 0;
      __syncwarp(gmask);
      if (i < n_l) sbase[dst_l + i] = v;
      __syncwarp(gmask);
    }
  }
  for (int j = 0; j < 4; j++) sbase[4 * lane + j] = uint8_t(len >> (8 * j));
  if (lane == 0) sizes[b] = kHead + int64_t(total);
}

// Decode: lane l decodes its nodes forward into shared memory, one node at a
// time, and writes each finished node (64 bytes) to its place.  status[b] =
// nodes decoded, or PG_ERR_FORMAT for a stream that does not end exactly
// where its lengths say with the initial state.
__global__ void __launch_bounds__(kGroups * kLanesS)
store_decode_kernel(const uint8_t* __restrict__ in, const int64_t* __restrict__ in_offsets,
                    const int64_t* __restrict__ in_sizes, const int32_t* __restrict__ count,
                    const int64_t* __restrict__ dst, int nblocks, int turn, const uint16_t* __restrict__ freq,
                    uint64_t* __restrict__ nodes, int64_t* __restrict__ status) {
  __shared__ uint2 F[kCtx];
  __shared__ uint32_t buf[2 * 16][kThreads];
  load_freqs(freq, F);
  __syncthreads();
  const int g = threadIdx.x / kLanesS, lane = threadIdx.x % kLanesS;
  const int b = blockIdx.x * kGroups + g;
  if (b >= nblocks) return;
  constexpr unsigned gmask = 0xffffffffu;   // a block's lanes are one warp
  const int n = count[b], m = lane_nodes(n);
  const int k0 = lane * m, k1 = min(n, k0 + m);
  const uint8_t* sbase = in + in_offsets[b];
  const int64_t size = in_sizes[b];
  int bad = size < kHead;
  uint64_t start = 0, total = 0;
  uint32_t mylen = 0;
  if (!bad && (sbase[0] & sbase[1] & sbase[2] & sbase[3]) == 0xff) {
    // a block stored raw
    const int64_t words = 8 * int64_t(n);
    const int ok = size == kHead + 8 * words;
    const uint8_t* src = sbase + kHead;
    uint64_t* o = nodes + 8 * dst[b];
    if (ok && !(reinterpret_cast<uintptr_t>(src) & 7)) {
      for (int64_t i = lane; i < words; i += kLanesS) o[i] = reinterpret_cast<const uint64_t*>(src)[i];
    } else if (ok) {
      for (int64_t i = lane; i < words; i += kLanesS) {
        uint64_t v = 0;
        for (int j = 0; j < 8; j++) v |= uint64_t(src[8 * i + j]) << (8 * j);
        o[i] = v;
      }
    }
    if (lane == 0) status[b] = ok ? n : PG_ERR_FORMAT;
    return;
  }
  {
    // this lane's length, the lengths before it (exclusive scan) and the sum
    uint32_t v = 0;
    if (!bad)
      for (int j = 0; j < 4; j++) v |= uint32_t(sbase[4 * lane + j]) << (8 * j);
    uint64_t incl = v;
#pragma unroll
    for (int o = 1; o < kLanesS; o <<= 1) {
      const uint64_t u = __shfl_up_sync(gmask, incl, o);
      if (lane >= o) incl += u;
    }
    mylen = v;
    start = incl - v;
    total = __shfl_sync(gmask, incl, kLanesS - 1);
    if (!bad) bad = total != uint64_t(size - kHead);
  }
  const uint8_t* p = sbase + kHead + start;
  const uint8_t* end = p + (bad ? 0 : mylen);
  uint32_t state = 0;
  for (int j = 0; j < 4 && p < end; j++) state = (state << 8) | *p++;
  uint32_t* cur = &buf[0][threadIdx.x];
  uint32_t* prev = &buf[16][threadIdx.x];
  uint64_t* outp = nodes + 8 * dst[b];
  for (int k = k0; k < k1 && !bad; k++) {
    const bool has_prev = k > k0;
    for (int w = 0; w < 16; w++) {
      const uint32_t a2 = (w & 3) ? cur[kThreads * (w - 1)] : ~0u;
      const uint32_t a3 = w >= 4 ? cur[kThreads * (w - 4)] : ~0u;
      const uint32_t ap = has_prev ? prev[kThreads * w] : ~0u;
      uint32_t x = 0;   // the word's symbols decoded so far
#pragma unroll
      for (int i = 0; i < 16; i++) {
        const uint32_t a0 = x << 2 | kNoAxis0, a1 = x << 8 | kNoAxis1;
        const uint2 fc = F[word_context(a0, a1, a2, a3, ap, i)];
        const uint32_t f0 = fc.x & 0xffffu, f1 = fc.x >> 16;
        const uint32_t slot = state & (kTot - 1);
        const uint32_t sym = slot < f0 ? 0 : slot < f0 + f1 ? 1 : 2;
        const uint32_t f = sym == 0 ? f0 : sym == 1 ? f1 : fc.y;
        const uint32_t cum = sym == 0 ? 0u : sym == 1 ? f0 : f0 + f1;
        state = f * (state >> kTotBits) + slot - cum;
        while (state < kLow && p < end) state = (state << 8) | *p++;
        x |= sym << (2 * i);
      }
      cur[kThreads * w] = x;
    }
    uint64_t* o = outp + 8 * int64_t(k);
    for (int w = 0; w < 4; w++) {
      uint64_t black = 0, white = 0;
      for (int h = 0; h < 4; h++) {
        const uint32_t x = cur[kThreads * (4 * w + h)];
        black |= uint64_t(gather16(x)) << (16 * h);
        white |= uint64_t(gather16(x >> 1)) << (16 * h);
      }
      o[w] = turn ? white : black;
      o[4 + w] = ~(turn ? black : white);
    }
    uint32_t* t = cur; cur = prev; prev = t;
  }
  if (!bad) bad = p != end || state != kLow;
  bad = __any_sync(gmask, bad);
  if (lane == 0) status[b] = bad ? PG_ERR_FORMAT : n;
}

int blocks_grid(int nblocks) { return (nblocks + kGroups - 1) / kGroups; }

}  // namespace
}  // namespace pg

using namespace pg;

extern "C" int64_t pg_store_bound(int64_t nodes) {
  if (nodes < 0 || nodes > 8 * 8 * 8 * 8 * 64) return fail(PG_ERR_ARG, "bad node count");
  return store_bound(int(nodes));
}

extern "C" int pg_store_table(const uint64_t* nodes, const int64_t* first, const int32_t* count, int nblocks, int turn,
                              uint16_t* table, void* stream_) {
  if (nblocks < 0 || !table || (nblocks && (!nodes || !first || !count))) return fail(PG_ERR_ARG, "bad store arguments");
  cudaStream_t stream = (cudaStream_t)stream_;
  stream_scratch scratch(stream);
  unsigned* hist = nullptr;
  PG_CUDA(scratch.alloc(&hist, sizeof(unsigned) * kCtx * 3));
  PG_CUDA(cudaMemsetAsync(hist, 0, sizeof(unsigned) * kCtx * 3, stream));
  if (nblocks) {
    const int stride = (nblocks + kTableBlocks - 1) / kTableBlocks;
    store_hist_kernel<<<(nblocks + stride - 1) / stride, 256, 0, stream>>>(nodes, first, count, stride, turn & 1,
                                                                            hist);
    PG_CUDA(cudaGetLastError());
  }
  store_table_kernel<<<kCtx / 256, 256, 0, stream>>>(hist, table);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

extern "C" int pg_store_encode(const uint64_t* nodes, const int64_t* first, const int32_t* count, int nblocks, int turn,
                               const uint16_t* table, uint8_t* out, const int64_t* out_offsets, int64_t* sizes,
                               void* stream) {
  if (nblocks < 0 || (nblocks && (!nodes || !first || !count || !table || !out || !out_offsets || !sizes)))
    return fail(PG_ERR_ARG, "bad store arguments");
  if (!nblocks) return PG_OK;
  store_encode_kernel<<<blocks_grid(nblocks), kGroups * kLanesS, 0, (cudaStream_t)stream>>>(
      nodes, first, count, nblocks, turn & 1, table, out, out_offsets, sizes);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

extern "C" int pg_store_decode(const uint8_t* in, const int64_t* in_offsets, const int64_t* in_sizes,
                               const int32_t* count, const int64_t* dst, int nblocks, int turn, const uint16_t* table,
                               uint64_t* nodes, int64_t* status, void* stream) {
  if (nblocks < 0 || (nblocks && (!in || !in_offsets || !in_sizes || !count || !dst || !table || !nodes || !status)))
    return fail(PG_ERR_ARG, "bad store arguments");
  if (!nblocks) return PG_OK;
  store_decode_kernel<<<blocks_grid(nblocks), kGroups * kLanesS, 0, (cudaStream_t)stream>>>(
      in, in_offsets, in_sizes, count, dst, nblocks, turn & 1, table, nodes, status);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}
