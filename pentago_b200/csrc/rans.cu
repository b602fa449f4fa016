// Static-table rANS over ternary win/tie/loss symbols, byte-identical to the
// reference's format version 2 (pentago/shard/arithmetic.cc:20-23, 48-77,
// 366-495): 8 interleaved 32-bit rANS lanes (symbol i on lane i % 8), 14-bit
// frequency total, byte renormalization at 2^23, each lane's bytes stored in
// decode order, header = version(4) | counts(3 x 8) | stream lengths(8 x 4).
//
// A stream has only 8 sequential chains, so the GPU encodes many streams at
// once: one 8-thread group per stream (four streams per warp).  A stream's
// lanes first count its symbols together (the frequency table comes from the
// counts, make_freq), then each lane encodes its symbols backward into its
// own slot of the output, and the lanes are finally packed behind the header.
#include "runtime.h"
#include "../../include/pentago_b200.h"
#include <cstdint>

namespace pg {

constexpr uint32_t kRansTotalBits = 14;
constexpr uint32_t kRansTotal = 1u << kRansTotalBits;
constexpr uint32_t kRansLower = 1u << 23;
constexpr int kLanes = 8;
constexpr int kHeader = 4 + 24 + 32;

struct rans_freq {
  uint32_t freq[3], cum[3], xmax[3];
};

// make_freq (arithmetic.cc:48-77), in the same integer arithmetic.
__host__ __device__ inline rans_freq make_freq(const uint64_t* counts) {
  rans_freq t;
  const uint64_t sum = counts[0] + counts[1] + counts[2];
  uint32_t f[3];
  if (sum) {
    for (int i = 0; i < 3; i++) f[i] = uint32_t(counts[i] * kRansTotal / sum);
    for (int i = 0; i < 3; i++) if (!f[i]) f[i] = 1;
    const int32_t adjust = int32_t(kRansTotal) - int32_t(f[0] + f[1] + f[2]);
    int largest = 0;
    if (f[1] > f[largest]) largest = 1;
    if (f[2] > f[largest]) largest = 2;
    f[largest] = uint32_t(int32_t(f[largest]) + adjust);
  } else {
    f[0] = f[1] = f[2] = kRansTotal / 3;
    f[0] += kRansTotal - 3 * (kRansTotal / 3);
  }
  const uint32_t xm = (kRansLower >> kRansTotalBits) << 8;
  for (int i = 0; i < 3; i++) { t.freq[i] = f[i]; t.xmax[i] = xm * f[i]; }
  t.cum[0] = 0;
  t.cum[1] = f[0];
  t.cum[2] = f[0] + f[1];
  return t;
}

// Worst-case lane slot (the reference's per-lane buffer, arithmetic.cc:377).
__host__ __device__ inline int64_t lane_capacity(int64_t n) { return n / kLanes * 2 + 64; }
__host__ __device__ inline int64_t stream_bound(int64_t n) { return kHeader + kLanes * lane_capacity(n); }

__device__ inline void put_u32(uint8_t* p, uint32_t v) { for (int i = 0; i < 4; i++) p[i] = uint8_t(v >> (8 * i)); }
__device__ inline void put_u64(uint8_t* p, uint64_t v) { for (int i = 0; i < 8; i++) p[i] = uint8_t(v >> (8 * i)); }
__device__ inline uint32_t get_u32(const uint8_t* p) {
  return uint32_t(p[0]) | uint32_t(p[1]) << 8 | uint32_t(p[2]) << 16 | uint32_t(p[3]) << 24;
}
__device__ inline uint64_t get_u64(const uint8_t* p) { return uint64_t(get_u32(p)) | uint64_t(get_u32(p + 4)) << 32; }

// Encoder constants of one symbol: state / freq by a reciprocal multiply
// (x < 2^31 after renormalization, where the reciprocal is exact), as in
// F. Giesen's ryg_rans (RansEncSymbolInit / RansEncPutSymbol, after
// Alverson, "Integer division using reciprocals", 1991).  The new state is
// x + bias + q * (total - freq) = (x / freq) * total + x % freq + cum.
struct rans_enc_sym {
  uint32_t xmax, rcp, shift, bias, cmpl;
};

__host__ __device__ inline rans_enc_sym enc_sym(const rans_freq& t, int s) {
  rans_enc_sym e;
  const uint32_t f = t.freq[s];
  e.xmax = t.xmax[s];
  e.cmpl = kRansTotal - f;
  if (f < 2) {
    e.rcp = ~0u;
    e.shift = 0;
    e.bias = t.cum[s] + kRansTotal - 1;
  } else {
    uint32_t sh = 0;
    while (f > (1u << sh)) sh++;
    e.rcp = uint32_t(((uint64_t(1) << (sh + 31)) + f - 1) / f);
    e.shift = sh - 1;
    e.bias = t.cum[s];
  }
  return e;
}

// One 8-thread group per stream.  out_offsets[s] has room for stream_bound(n_s).
// Long streams are latency bound (8 sequential chains per stream), so each
// lane loads its next 16 symbols while it codes the current 16.
__global__ void __launch_bounds__(256)
rans_encode_kernel(const uint8_t* __restrict__ symbols, const int64_t* __restrict__ offsets, int nstreams,
                   uint8_t* __restrict__ out, const int64_t* __restrict__ out_offsets, int64_t* __restrict__ sizes,
                   const int64_t* __restrict__ expect) {
  const int group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const int lane = threadIdx.x & 7;
  const unsigned gmask = 0xffu << (threadIdx.x & 24);
  if (group >= nstreams) return;
  const int64_t begin = offsets[group], n = offsets[group + 1] - begin;
  // With `expect`, a stream of another length has no room reserved: refuse it
  if (expect && n != expect[group]) {
    if (lane == 0) sizes[group] = PG_ERR_ARG;
    return;
  }
  const uint8_t* sym = symbols + begin;
  // Count symbols (ones and twos; zeros are the rest) and look for values
  // above 2: whole aligned words by all lanes, the ragged ends by lane 0
  uint64_t c1 = 0, c2 = 0;
  uint32_t badbits = 0;
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(sym), a1 = a0 + uintptr_t(n);
  uintptr_t w0 = (a0 + 3) & ~uintptr_t(3), w1 = a1 & ~uintptr_t(3);
  if (w1 < w0) w0 = w1 = a1;
  const uint32_t* W = reinterpret_cast<const uint32_t*>(w0);
  const int64_t nw = int64_t(w1 - w0) >> 2;
#pragma unroll 4
  for (int64_t k = lane; k < nw; k += kLanes) {
    const uint32_t w = W[k];
    c1 += __popc(w & 0x01010101u);
    c2 += __popc(w & 0x02020202u);
    badbits |= (w & 0xfcfcfcfcu) | (w & (w >> 1) & 0x01010101u);
  }
  if (lane == 0) {
    for (uintptr_t a = a0; a < a1; a++) {
      if (a == w0) a = w1;
      if (a >= a1) break;
      const uint32_t v = *reinterpret_cast<const uint8_t*>(a);
      c1 += v == 1;
      c2 += v == 2;
      badbits |= v > 2;
    }
  }
  for (int o = 4; o; o >>= 1) {
    c1 += __shfl_xor_sync(gmask, c1, o, 8);
    c2 += __shfl_xor_sync(gmask, c2, o, 8);
    badbits |= __shfl_xor_sync(gmask, badbits, o, 8);
  }
  if (badbits) {
    if (lane == 0) sizes[group] = PG_ERR_ARG;
    return;
  }
  const uint64_t c[3] = {uint64_t(n) - c1 - c2, c1, c2};
  const rans_freq t = make_freq(c);
  const rans_enc_sym e0 = enc_sym(t, 0), e1 = enc_sym(t, 1), e2 = enc_sym(t, 2);
  // Encode this lane's symbols (i = lane mod 8) backward into its slot
  uint8_t* base = out + out_offsets[group];
  const int64_t cap = lane_capacity(n);
  uint8_t* slot_end = base + kHeader + (lane + 1) * cap;
  uint8_t* cur = slot_end;
  uint32_t state = kRansLower;
  const int64_t cnt = n > lane ? (n - 1 - lane) / kLanes + 1 : 0;  // this lane's symbols
  const uint8_t* last = sym + lane + kLanes * (cnt - 1);          // its last symbol, coded first
  constexpr int kAhead = 16;
  uint8_t now[kAhead], next[kAhead];
#pragma unroll
  for (int k = 0; k < kAhead; k++) now[k] = k < cnt ? last[-kLanes * int64_t(k)] : 0;
  for (int64_t j0 = 0; j0 < cnt; j0 += kAhead) {
#pragma unroll
    for (int k = 0; k < kAhead; k++) {
      const int64_t j = j0 + kAhead + k;
      next[k] = j < cnt ? last[-kLanes * j] : 0;
    }
#pragma unroll
    for (int k = 0; k < kAhead; k++) {
      if (j0 + k >= cnt) break;
      const int s = now[k];
      const rans_enc_sym e = s == 0 ? e0 : s == 1 ? e1 : e2;
      while (state >= e.xmax) { *--cur = uint8_t(state & 0xff); state >>= 8; }
      const uint32_t q = __umulhi(state, e.rcp) >> e.shift;
      state += e.bias + q * e.cmpl;
    }
#pragma unroll
    for (int k = 0; k < kAhead; k++) now[k] = next[k];
  }
  for (int j = 0; j < 4; j++) *--cur = uint8_t(state >> (8 * j));
  const uint32_t len = uint32_t(slot_end - cur);
  // Lengths of all lanes, and this lane's destination behind the header
  uint32_t lens[kLanes];
  for (int l = 0; l < kLanes; l++) lens[l] = __shfl_sync(gmask, len, l, 8);
  int64_t dst = kHeader;
  for (int l = 0; l < lane; l++) dst += lens[l];
  // Pack lanes in order: lane l's bytes move left, never past a lane not yet moved
  for (int l = 0; l < kLanes; l++) {
    __syncwarp(gmask);
    if (l == lane) {
      uint8_t* d = base + dst;
      for (uint32_t k = 0; k < len; k++) d[k] = cur[k];
    }
  }
  __syncwarp(gmask);
  if (lane == 0) {
    put_u32(base, 2);
    for (int k = 0; k < 3; k++) put_u64(base + 4 + 8 * k, c[k]);
    int64_t total = kHeader;
    for (int l = 0; l < kLanes; l++) { put_u32(base + 28 + 4 * l, lens[l]); total += lens[l]; }
    sizes[group] = total;
  }
}

// status[s]: number of symbols decoded, or PG_ERR_FORMAT / PG_ERR_CAPACITY.
__global__ void __launch_bounds__(256)
rans_decode_kernel(const uint8_t* __restrict__ in, const int64_t* __restrict__ in_offsets,
                   const int64_t* __restrict__ in_sizes, int nstreams, uint8_t* __restrict__ symbols,
                   const int64_t* __restrict__ sym_offsets, const int64_t* __restrict__ sym_caps,
                   int64_t* __restrict__ status, int only_v2) {
  const int group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const int lane = threadIdx.x & 7;
  if (group >= nstreams) return;
  const uint8_t* base = in + in_offsets[group];
  const int64_t size = in_sizes[group];
  // Streams of another version are left to the learned decoder when asked
  if (only_v2 && size >= 4 && get_u32(base) != 2) return;
  // Header checks as arithmetic_deserialize / arithmetic_decode (arithmetic.cc:403-495)
  if (size < kHeader || get_u32(base) != 2) { if (lane == 0) status[group] = PG_ERR_FORMAT; return; }
  uint64_t c[3];
  for (int k = 0; k < 3; k++) c[k] = get_u64(base + 4 + 8 * k);
  const uint64_t n = c[0] + c[1] + c[2];
  if (c[0] > n || c[1] > n || c[2] > n || n > ~uint64_t(0) / 0x3fff) {
    if (lane == 0) status[group] = PG_ERR_FORMAT;
    return;
  }
  uint64_t total = 0, start = 0;
  uint32_t lens[kLanes];
  for (int l = 0; l < kLanes; l++) {
    lens[l] = get_u32(base + 28 + 4 * l);
    if (l < lane) start += lens[l];
    total += lens[l];
  }
  if (total != uint64_t(size - kHeader)) { if (lane == 0) status[group] = PG_ERR_FORMAT; return; }
  if (int64_t(n) > sym_caps[group]) { if (lane == 0) status[group] = PG_ERR_CAPACITY; return; }
  const rans_freq t = make_freq(c);
  const uint8_t* p = base + kHeader + start;
  const uint8_t* end = p + lens[lane];
  uint32_t state = 0;
  for (int j = 0; j < 4 && p < end; j++) state = (state << 8) | *p++;
  uint8_t* out = symbols + sym_offsets[group];
  for (uint64_t i = lane; i < n; i += kLanes) {
    const uint32_t slot = state & (kRansTotal - 1);
    const int s = slot < t.cum[1] ? 0 : slot < t.cum[2] ? 1 : 2;
    state = t.freq[s] * (state >> kRansTotalBits) + slot - t.cum[s];
    while (state < kRansLower && p < end) state = (state << 8) | *p++;
    out[i] = uint8_t(s);
  }
  if (lane == 0) status[group] = int64_t(n);
}

int64_t rans_stream_bound(int64_t n) { return stream_bound(n); }

int launch_rans_encode(const uint8_t* symbols, const int64_t* offsets, int nstreams, uint8_t* out,
                       const int64_t* out_offsets, int64_t* sizes, const int64_t* expect, cudaStream_t stream) {
  const int threads = 256, groups_per_block = threads / kLanes;
  rans_encode_kernel<<<(nstreams + groups_per_block - 1) / groups_per_block, threads, 0, stream>>>(
      symbols, offsets, nstreams, out, out_offsets, sizes, expect);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

int launch_rans_decode(const uint8_t* in, const int64_t* in_offsets, const int64_t* in_sizes, int nstreams,
                       uint8_t* symbols, const int64_t* sym_offsets, const int64_t* sym_caps, int64_t* status,
                       int only_v2, cudaStream_t stream) {
  const int threads = 256, groups_per_block = threads / kLanes;
  rans_decode_kernel<<<(nstreams + groups_per_block - 1) / groups_per_block, threads, 0, stream>>>(
      in, in_offsets, in_sizes, nstreams, symbols, sym_offsets, sym_caps, status, only_v2);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

// Ternary symbols of solved nodes in the on-disk convention
// (shard/shard.cc:448-449 after end/check.cc:154-156, 197-200): for rotation r
// of node k, symbol = black wins + 2 white wins.  Nodes are [we-win,
// we-win-or-tie] for the player to move; `turn` = 1 when white moves.
__global__ void node_symbols_kernel(const uint64_t* __restrict__ nodes, int64_t n, int turn,
                                    uint8_t* __restrict__ symbols) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;  // one thread per 64 symbols
  if (i >= n * 4) return;
  const int64_t k = i >> 2;
  const int w = int(i & 3);
  const uint64_t win = nodes[8 * k + w], notlost = nodes[8 * k + 4 + w];
  const uint64_t black = turn ? ~notlost : win, white = turn ? win : ~notlost;
  uint8_t* out = symbols + 64 * i;
  for (int b = 0; b < 64; b++) out[b] = uint8_t((black >> b & 1) + 2 * (white >> b & 1));
}

// The inverse: nodes of the side to move from their symbols (one thread per
// 64 symbols, read as four 16-byte words).
__global__ void symbols_nodes_kernel(const uint8_t* __restrict__ symbols, int64_t n, int turn,
                                     uint64_t* __restrict__ nodes) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n * 4) return;
  const int64_t k = i >> 2;
  const int w = int(i & 3);
  const uint4* in = reinterpret_cast<const uint4*>(symbols + 64 * i);
  uint64_t black = 0, white = 0;
#pragma unroll
  for (int v = 0; v < 4; v++) {
    const uint4 q = in[v];
    const uint32_t part[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int p = 0; p < 4; p++)
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const uint32_t sym = part[p] >> (8 * b) & 0xff;
        const int bit = 16 * v + 4 * p + b;
        black |= uint64_t(sym == 1) << bit;
        white |= uint64_t(sym == 2) << bit;
      }
  }
  nodes[8 * k + w] = turn ? white : black;
  nodes[8 * k + 4 + w] = ~(turn ? black : white);
}

// Copy stream s (in + in_offsets[s], sizes[s] bytes) to out + out_offsets[s]:
// one CTA per stream, 16-byte words where both ends allow it.
__global__ void pack_streams_kernel(const uint8_t* __restrict__ in, const int64_t* __restrict__ in_offsets,
                                    const int64_t* __restrict__ sizes, uint8_t* __restrict__ out,
                                    const int64_t* __restrict__ out_offsets) {
  const int s = blockIdx.x;
  const uint8_t* src = in + in_offsets[s];
  uint8_t* dst = out + out_offsets[s];
  const int64_t n = sizes[s];
  if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
    const int64_t w = n >> 4;
    for (int64_t i = threadIdx.x; i < w; i += blockDim.x)
      reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
    for (int64_t i = 16 * w + threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  } else {
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  }
}

}  // namespace pg

using namespace pg;

extern "C" int pg_symbols_nodes(const uint8_t* symbols, int64_t n, int turn, uint64_t* nodes, void* stream) {
  if (n < 0 || (n && (!symbols || !nodes))) return fail(PG_ERR_ARG, "bad node count");
  if (reinterpret_cast<uintptr_t>(symbols) & 15) return fail(PG_ERR_ARG, "symbols must be 16-byte aligned");
  if (!n) return PG_OK;
  const int64_t threads = 4 * n;
  symbols_nodes_kernel<<<unsigned((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(symbols, n, turn & 1, nodes);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

extern "C" int pg_pack_streams(const uint8_t* in, const int64_t* in_offsets, const int64_t* sizes, int n, uint8_t* out,
                               const int64_t* out_offsets, void* stream) {
  if (n < 0 || (n && (!in || !in_offsets || !sizes || !out || !out_offsets))) return fail(PG_ERR_ARG, "bad pack arguments");
  for (int s0 = 0; s0 < n; s0 += 65535) {
    const int k = n - s0 < 65535 ? n - s0 : 65535;
    pack_streams_kernel<<<k, 256, 0, (cudaStream_t)stream>>>(in, in_offsets + s0, sizes + s0, out, out_offsets + s0);
    PG_CUDA(cudaGetLastError());
  }
  return PG_OK;
}

extern "C" int64_t pg_rans_bound(int64_t n) { return n < 0 ? PG_ERR_ARG : stream_bound(n); }

extern "C" int pg_rans_encode_batch(const uint8_t* symbols, const int64_t* offsets, int nstreams, uint8_t* out,
                                    const int64_t* out_offsets, int64_t* sizes, void* stream) {
  if (nstreams < 0) return fail(PG_ERR_ARG, "bad stream count");
  if (!nstreams) return PG_OK;
  return launch_rans_encode(symbols, offsets, nstreams, out, out_offsets, sizes, nullptr, (cudaStream_t)stream);
}

extern "C" int pg_rans_decode_batch(const uint8_t* in, const int64_t* in_offsets, const int64_t* in_sizes,
                                    int nstreams, uint8_t* symbols, const int64_t* sym_offsets,
                                    const int64_t* sym_caps, int64_t* status, void* stream) {
  if (nstreams < 0) return fail(PG_ERR_ARG, "bad stream count");
  if (!nstreams) return PG_OK;
  return launch_rans_decode(in, in_offsets, in_sizes, nstreams, symbols, sym_offsets, sym_caps, status, 0,
                            (cudaStream_t)stream);
}

extern "C" int pg_node_symbols(const uint64_t* nodes, int64_t n, int turn, uint8_t* symbols, void* stream) {
  if (n < 0) return fail(PG_ERR_ARG, "bad node count");
  if (!n) return PG_OK;
  const int64_t threads = 4 * n;
  node_symbols_kernel<<<unsigned((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(nodes, n, turn & 1, symbols);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}
