// Shards of solved positions for training data (pentago/shard/shard.h,
// shard.cc, shard_permute.h): every (section, position, rotation) of a slice
// has a linear index offset[section] + 256 position + rotation (positions
// row-major over the section's shape, sections in signature order); a fixed
// bijection of [0, n) shuffles it; shard s of a power-of-two count holds the
// shuffled indices congruent to s, at position index >> log2(count).
//
// On the GPU: scatter_block for whole batches of blocks (one thread per 32
// rotations of a node; symbols are written as bytes, one per entry, ready for
// the format-2 coder), the permutation in both directions, and the board of
// a shuffled index.
#include "../../include/pentago_b200.h"
#include "lines.h"
#include "runtime.h"
#include "superscore.cuh"
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

namespace pg {
namespace {

// Shift amounts of the permutation per slice (pentago/shard/shard_permute.h:40-60,
// found there by search; part of the shard format).  The entry counts listed
// beside them there are the slices' totals, computed here from the sections.
constexpr uint8_t kPermShifts[19][8] = {
    {3, 2, 1, 5, 2, 2, 3, 6},         {6, 6, 4, 1, 3, 2, 6, 4},         {4, 6, 4, 8, 7, 6, 6, 3},
    {14, 6, 13, 12, 9, 7, 10, 3},     {6, 13, 8, 10, 6, 15, 4, 1},      {15, 17, 6, 16, 15, 13, 5, 18},
    {19, 21, 17, 16, 23, 16, 11, 20}, {15, 26, 10, 16, 13, 16, 9, 22},  {22, 23, 17, 24, 16, 19, 25, 21},
    {11, 24, 29, 23, 16, 21, 23, 1},  {24, 27, 3, 24, 7, 29, 25, 30},   {27, 30, 7, 27, 1, 28, 9, 31},
    {29, 33, 10, 34, 7, 29, 1, 31},   {18, 7, 4, 31, 34, 26, 18, 2},    {24, 29, 14, 35, 15, 22, 10, 18},
    {4, 9, 23, 41, 10, 37, 32, 35},   {8, 35, 33, 34, 14, 38, 7, 5},    {4, 42, 19, 41, 5, 39, 17, 37},
    {33, 40, 33, 39, 5, 42, 34, 37}};

// The permutation of one slice: windows L = [0, 2^k) and H = [n - 2^k, n),
// k = floor(log2 n); four pairs of steps on L, H, L, H, each x ^= x >> a
// then x += x << b (mod 2^k).  Both steps are bijections of the window.
struct perm_t {
  uint64_t n, pow2k, offset, mask;
  int k;
  int s[8];
};

PG_HD uint64_t perm_forward(const perm_t& P, uint64_t x) {
#pragma unroll
  for (int pair = 0; pair < 4; pair++) {
    const bool high = pair & 1;
    if (high ? x < P.offset : x >= P.pow2k) continue;
    uint64_t t = high ? x - P.offset : x;
    t ^= t >> P.s[2 * pair];
    t = (t + (t << P.s[2 * pair + 1])) & P.mask;
    x = high ? t + P.offset : t;
  }
  return x;
}

// Inverse: (1 + 2^b)^-1 = (1 - 2^b)(1 + 2^2b)(1 + 2^4b)... mod 2^k, and
// (I + R^a)^-1 = (I + R^a)(I + R^2a)(I + R^4a)... over GF(2).
PG_HD uint64_t perm_inverse(const perm_t& P, uint64_t x) {
#pragma unroll
  for (int pair = 3; pair >= 0; pair--) {
    const bool high = pair & 1;
    if (high ? x < P.offset : x >= P.pow2k) continue;
    uint64_t t = high ? x - P.offset : x;
    const int a = P.s[2 * pair], b = P.s[2 * pair + 1];
    t = (t - (t << b)) & P.mask;
    for (int c = 2 * b; c < P.k; c *= 2) t = (t + (t << c)) & P.mask;
    for (int c = a; c < P.k; c *= 2) t ^= t >> c;
    x = high ? t + P.offset : t;
  }
  return x;
}

// Sections of a slice in the mapping's order (all_boards_sections(slice, 8),
// pentago/base/all_boards.cc:160-203: standardized sections sorted by
// signature) with the prefix sums of 256 x their sizes.
struct slice_map {
  std::vector<uint64_t> sigs;
  std::vector<uint64_t> offsets;  // sigs.size() + 1
  perm_t perm;
};

bool section_standard(const section_t& s) { return s.standardize(nullptr).sig() == s.sig(); }

const slice_map& slice_mapping(int slice) {
  static std::mutex m;
  static std::map<int, slice_map> cache;
  std::lock_guard<std::mutex> g(m);
  auto it = cache.find(slice);
  if (it != cache.end()) return it->second;
  slice_map M;
  const int white = slice / 2, black = slice - white;
  // every split of the stones over the quadrants with at most 9 per quadrant
  for (int b3 = 0; b3 <= std::min(black, 9); b3++)
    for (int w3 = 0; w3 <= std::min(white, 9 - b3); w3++)
      for (int b2 = 0; b2 <= std::min(black - b3, 9); b2++)
        for (int w2 = 0; w2 <= std::min(white - w3, 9 - b2); w2++)
          for (int b1 = 0; b1 <= std::min(black - b3 - b2, 9); b1++)
            for (int w1 = 0; w1 <= std::min(white - w3 - w2, 9 - b1); w1++) {
              const int b0 = black - b3 - b2 - b1, w0 = white - w3 - w2 - w1;
              if (b0 > 9 || w0 > 9 || b0 + w0 > 9) continue;
              section_t s;
              const int c[4][2] = {{b0, w0}, {b1, w1}, {b2, w2}, {b3, w3}};
              for (int q = 0; q < 4; q++)
                for (int k = 0; k < 2; k++) s.c[q][k] = uint8_t(c[q][k]);
              if (section_standard(s)) M.sigs.push_back(s.sig());
            }
  std::sort(M.sigs.begin(), M.sigs.end());
  M.offsets.assign(1, 0);
  for (uint64_t sig : M.sigs) {
    int sh[4];
    section_t::from_sig(sig).shape(sh);
    M.offsets.push_back(M.offsets.back() + 256ull * uint64_t(sh[0]) * sh[1] * sh[2] * sh[3]);
  }
  perm_t& P = M.perm;
  P.n = M.offsets.back();
  P.k = 63 - __builtin_clzll(P.n);
  P.pow2k = uint64_t(1) << P.k;
  P.mask = P.pow2k - 1;
  P.offset = P.n - P.pow2k;
  for (int i = 0; i < 8; i++) P.s[i] = kPermShifts[slice][i];
  return cache.emplace(slice, std::move(M)).first->second;
}

// Per-section data the kernels read: linear offsets, shapes and the offsets
// of the four rotation-minimal quadrant lists.
struct shard_dev_t {
  perm_t perm;
  int nsec;
  const uint64_t* offsets;  // nsec + 1
  const int32_t* shape;     // 4 per section
  const int32_t* rmin;      // 4 per section: start in rmin_flat
};

// Section holding a linear index (binary search over the prefix sums).
PG_HD int find_section(const shard_dev_t& D, uint64_t linear) {
  int lo = 0, hi = D.nsec - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (ldg(D.offsets + mid) <= linear) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Quadrant side rotated left r times.
PG_HD uint32_t rotate_side(const dev_tables_t& T, uint32_t side, int r) {
  if (r == 3) return ldg(T.rot + 2 * side + 1);
  for (int i = 0; i < r; i++) side = ldg(T.rot + 2 * side);
  return side;
}

// board of a shuffled index (shard_mapping_t::board, shard.cc:137-168): the
// four rotation-minimal quadrants of the position, each rotated by its part
// of the rotation, packed 16 bits per quadrant.
PG_HD uint64_t shard_board(const shard_dev_t& D, const dev_tables_t& T, uint64_t shuffled) {
  const uint64_t linear = perm_inverse(D.perm, shuffled);
  const int si = find_section(D, linear);
  const uint64_t within = linear - ldg(D.offsets + si);
  uint64_t pos = within >> 8;
  const int rot = int(within & 255);
  int idx[4];
  for (int q = 3; q >= 0; q--) {
    const uint64_t d = uint64_t(ldg(D.shape + 4 * si + q));
    idx[q] = int(pos % d);
    pos /= d;
  }
  uint64_t board = 0;
  for (int q = 0; q < 4; q++) {
    const uint32_t v = ldg(T.rmin_flat + ldg(D.rmin + 4 * si + q) + idx[q]);
    const int r = rot >> (2 * q) & 3;
    const uint32_t s0 = rotate_side(T, ldg(T.unpack + 2 * v), r), s1 = rotate_side(T, ldg(T.unpack + 2 * v + 1), r);
    board |= uint64_t(ldg(T.pack + s0) + 2u * ldg(T.pack + s1)) << (16 * q);
  }
  return board;
}

__global__ void shard_permute_kernel(const perm_t P, const uint64_t* __restrict__ in, int64_t n, int inverse,
                                     uint64_t* __restrict__ out) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = inverse ? perm_inverse(P, in[i]) : perm_forward(P, in[i]);
}

__global__ void shard_board_kernel(const shard_dev_t D, const dev_tables_t T, const uint64_t* __restrict__ in,
                                   int64_t n, uint64_t* __restrict__ out) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t x = in[i];
    out[i] = x < D.perm.n ? shard_board(D, T, x) : ~uint64_t(0);
  }
}

struct block_dev_t {
  int32_t section;
  int32_t base[4];    // first position of the block (block coordinates x block size)
  int32_t shape[4];   // the block's shape
  int64_t node_offset;
};

// Where shard s's symbols start.  Packed (shard_off null): shards lo .. hi-1
// back to back, shard t holding q + (t < r) entries for n = q 2^shift + r,
// so the offset is arithmetic; otherwise the caller's table.
PG_HD int64_t shard_start(const int64_t* shard_off, uint64_t n, int shift, int lo, int s) {
  if (shard_off) return ldg(shard_off + (s - lo));
  const int64_t q = int64_t(n >> shift), r = int64_t(n & ((uint64_t(1) << shift) - 1));
  return (s - lo) * q + (std::min<int64_t>(s, r) - std::min<int64_t>(lo, r));
}

// scatter_block (shard.cc:405-464) for a batch of blocks: thread t of grid
// row b handles node t >> 3 of block b, rotations 32 (t & 7) .. + 31.
__global__ void __launch_bounds__(256)
shard_scatter_kernel(const shard_dev_t D, const block_dev_t* __restrict__ blocks, int block0,
                     const uint32_t* __restrict__ nodes, int turn, int shift, int lo, int hi,
                     const int64_t* __restrict__ shard_off, uint8_t* __restrict__ symbols) {
  const block_dev_t B = blocks[block0 + blockIdx.y];
  const int64_t nodes_in_block = int64_t(B.shape[0]) * B.shape[1] * B.shape[2] * B.shape[3];
  const int sshape[4] = {ldg(D.shape + 4 * B.section), ldg(D.shape + 4 * B.section + 1),
                         ldg(D.shape + 4 * B.section + 2), ldg(D.shape + 4 * B.section + 3)};
  const uint64_t sec_off = ldg(D.offsets + B.section);
  const uint64_t smask = (uint64_t(1) << shift) - 1;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < 8 * nodes_in_block;
       t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t node = t >> 3;
    const int w = int(t & 7);
    // position of the node: row-major over the section's shape
    int64_t r = node;
    int idx[4];
    for (int q = 3; q >= 0; q--) {
      idx[q] = B.base[q] + int(r % B.shape[q]);
      r /= B.shape[q];
    }
    const uint64_t pos = ((uint64_t(idx[0]) * sshape[1] + idx[1]) * sshape[2] + idx[2]) * sshape[3] + idx[3];
    const uint32_t* p = nodes + 16 * (B.node_offset + node);
    const uint32_t a = p[w], c = p[8 + w];
    uint32_t black, white;
    if (turn == 0) { black = a; white = ~c; }
    else if (turn == 1) { black = ~c; white = a; }
    else { black = a; white = c; }
    const uint64_t base = sec_off + 256 * pos + 32 * w;
    for (int bit = 0; bit < 32; bit++) {
      const uint64_t y = perm_forward(D.perm, base + bit);
      const int s = int(y & smask);
      if (s < lo || s >= hi) continue;
      symbols[shard_start(shard_off, D.perm.n, shift, lo, s) + int64_t(y >> shift)] =
          uint8_t((black >> bit & 1) + 2 * (white >> bit & 1));
    }
  }
}

// Device copies of a slice's per-section data (scratch of one call).
int upload_slice(const slice_map& M, stream_scratch& scratch, cudaStream_t stream, shard_dev_t& D) {
  const tables_t& T = tables();
  const int n = int(M.sigs.size());
  std::vector<int32_t> shape(4 * n), rmin(4 * n);
  for (int i = 0; i < n; i++) {
    const section_t s = section_t::from_sig(M.sigs[i]);
    s.shape(&shape[4 * i]);
    for (int q = 0; q < 4; q++) rmin[4 * i + q] = T.rmin_off[rmin_bucket(s.c[q][0], s.c[q][1])];
  }
  uint64_t* off = nullptr;
  int32_t *sh = nullptr, *rm = nullptr;
  PG_CUDA(scratch.alloc(&off, sizeof(uint64_t) * (n + 1)));
  PG_CUDA(scratch.alloc(&sh, sizeof(int32_t) * 4 * n));
  PG_CUDA(scratch.alloc(&rm, sizeof(int32_t) * 4 * n));
  PG_CUDA(cudaMemcpyAsync(off, M.offsets.data(), sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice, stream));
  PG_CUDA(cudaMemcpyAsync(sh, shape.data(), sizeof(int32_t) * 4 * n, cudaMemcpyHostToDevice, stream));
  PG_CUDA(cudaMemcpyAsync(rm, rmin.data(), sizeof(int32_t) * 4 * n, cudaMemcpyHostToDevice, stream));
  D.perm = M.perm;
  D.nsec = n;
  D.offsets = off;
  D.shape = sh;
  D.rmin = rm;
  return PG_OK;
}

bool slice_ok(int slice) { return 0 <= slice && slice <= 18; }

unsigned grid_for(int64_t n) { return unsigned(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32))); }

}  // namespace
}  // namespace pg

using namespace pg;

extern "C" int pg_shard_sections(int slice, uint64_t* sigs, int cap) {
  if (!slice_ok(slice) || cap < 0 || (cap && !sigs)) return fail(PG_ERR_ARG, "bad shard section arguments");
  const slice_map& M = slice_mapping(slice);
  for (int i = 0; i < int(M.sigs.size()) && i < cap; i++) sigs[i] = M.sigs[i];
  return int(M.sigs.size());
}

extern "C" int64_t pg_shard_total(int slice) {
  if (!slice_ok(slice)) return fail(PG_ERR_ARG, "slice must be 0..18");
  return int64_t(slice_mapping(slice).perm.n);
}

static bool shards_ok(int total_shards) { return total_shards > 0 && !(total_shards & (total_shards - 1)); }

extern "C" int64_t pg_shard_size(int slice, int total_shards, int shard) {
  if (!slice_ok(slice) || !shards_ok(total_shards) || shard < 0 || shard >= total_shards)
    return fail(PG_ERR_ARG, "bad shard size arguments (shard counts are powers of two)");
  const int shift = __builtin_ctz(unsigned(total_shards));
  return int64_t((slice_mapping(slice).perm.n + uint64_t(total_shards - 1) - uint64_t(shard)) >> shift);
}

extern "C" int pg_shard_permute(int slice, const uint64_t* in, int64_t n, int inverse, uint64_t* out, void* stream) {
  if (!slice_ok(slice) || n < 0 || (n && (!in || !out))) return fail(PG_ERR_ARG, "bad permute arguments");
  if (!n) return PG_OK;
  shard_permute_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(slice_mapping(slice).perm, in, n, inverse, out);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

extern "C" int pg_shard_boards(int slice, const uint64_t* shuffled, int64_t n, uint64_t* boards, void* stream_) {
  if (!slice_ok(slice) || n < 0 || (n && (!shuffled || !boards))) return fail(PG_ERR_ARG, "bad board arguments");
  if (!n) return PG_OK;
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  cudaStream_t stream = (cudaStream_t)stream_;
  stream_scratch scratch(stream);
  shard_dev_t D;
  if (int rc = upload_slice(slice_mapping(slice), scratch, stream, D)) return rc;
  shard_board_kernel<<<grid_for(n), 256, 0, stream>>>(D, *T, shuffled, n, boards);
  PG_CUDA(cudaGetLastError());
  return PG_OK;
}

extern "C" int pg_shard_scatter(int slice, int total_shards, int shard_lo, int shard_hi, const pg_shard_block_t* blocks,
                                int nblocks, const uint64_t* nodes, int turn, uint8_t* symbols,
                                const int64_t* shard_offsets, void* stream_) {
  if (!slice_ok(slice) || !shards_ok(total_shards) || shard_lo < 0 || shard_lo >= shard_hi ||
      shard_hi > total_shards || nblocks < 0 || turn < 0 || turn > PG_ST_RAW ||
      (nblocks && (!blocks || !nodes || !symbols)))
    return fail(PG_ERR_ARG, "bad scatter arguments");
  if (reinterpret_cast<uintptr_t>(nodes) & 15) return fail(PG_ERR_ARG, "nodes must be 16-byte aligned");
  if (!nblocks) return PG_OK;
  const slice_map& M = slice_mapping(slice);
  std::vector<block_dev_t> bd(nblocks);
  int64_t max_nodes = 0;
  for (int i = 0; i < nblocks; i++) {
    const pg_shard_block_t& b = blocks[i];
    if (b.section < 0 || b.section >= int(M.sigs.size()) || b.block_size < 2 || b.block_size > 26 ||
        (b.block_size & 1) || b.node_offset < 0)
      return fail(PG_ERR_ARG, "bad shard block");
    int sh[4];
    section_t::from_sig(M.sigs[b.section]).shape(sh);
    bd[i].section = b.section;
    bd[i].node_offset = b.node_offset;
    int64_t nn = 1;
    for (int q = 0; q < 4; q++) {
      const int base = b.block[q] * b.block_size;
      if (base >= sh[q]) return fail(PG_ERR_ARG, "block outside its section");
      bd[i].base[q] = base;
      bd[i].shape[q] = std::min(b.block_size, sh[q] - base);
      nn *= bd[i].shape[q];
    }
    max_nodes = std::max(max_nodes, nn);
  }
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  cudaStream_t stream = (cudaStream_t)stream_;
  stream_scratch scratch(stream);
  shard_dev_t D;
  if (int rc = upload_slice(M, scratch, stream, D)) return rc;
  block_dev_t* bdev = nullptr;
  int64_t* off = nullptr;
  PG_CUDA(scratch.alloc(&bdev, sizeof(block_dev_t) * nblocks));
  PG_CUDA(cudaMemcpyAsync(bdev, bd.data(), sizeof(block_dev_t) * nblocks, cudaMemcpyHostToDevice, stream));
  if (shard_offsets) {
    PG_CUDA(scratch.alloc(&off, sizeof(int64_t) * (shard_hi - shard_lo)));
    PG_CUDA(cudaMemcpyAsync(off, shard_offsets, sizeof(int64_t) * (shard_hi - shard_lo), cudaMemcpyHostToDevice,
                            stream));
  }
  const int shift = __builtin_ctz(unsigned(total_shards));
  const int64_t threads = 8 * max_nodes;
  for (int b0 = 0; b0 < nblocks; b0 += 65535) {
    const int nb = std::min(65535, nblocks - b0);
    const unsigned gx = unsigned(std::max<int64_t>(1, std::min<int64_t>((threads + 255) / 256, std::max(1, 148 * 16 / nb))));
    shard_scatter_kernel<<<dim3(gx, unsigned(nb)), 256, 0, stream>>>(D, bdev, b0, reinterpret_cast<const uint32_t*>(nodes),
                                                                    turn, shift, shard_lo, shard_hi, off, symbols);
    PG_CUDA(cudaGetLastError());
  }
  return PG_OK;
}

// The permutation (op 0 forward, 1 inverse) and boards (op 2) on the host,
// with the kernels' own functions.
extern "C" int pg_selftest_shard_host(int op, int slice, const uint64_t* in, int64_t n, uint64_t* out) {
  if (!slice_ok(slice) || op < 0 || op > 2 || n < 0 || (n && (!in || !out))) return fail(PG_ERR_ARG, "bad selftest arguments");
  const slice_map& M = slice_mapping(slice);
  if (op < 2) {
    for (int64_t i = 0; i < n; i++) out[i] = op ? perm_inverse(M.perm, in[i]) : perm_forward(M.perm, in[i]);
    return PG_OK;
  }
  const tables_t& H = tables();
  const int ns = int(M.sigs.size());
  std::vector<int32_t> shape(4 * ns), rmin(4 * ns);
  for (int i = 0; i < ns; i++) {
    const section_t s = section_t::from_sig(M.sigs[i]);
    s.shape(&shape[4 * i]);
    for (int q = 0; q < 4; q++) rmin[4 * i + q] = H.rmin_off[rmin_bucket(s.c[q][0], s.c[q][1])];
  }
  const shard_dev_t D = {M.perm, ns, M.offsets.data(), shape.data(), rmin.data()};
  const dev_tables_t T = host_tables_view();
  for (int64_t i = 0; i < n; i++) out[i] = in[i] < M.perm.n ? shard_board(D, T, in[i]) : ~uint64_t(0);
  return PG_OK;
}
