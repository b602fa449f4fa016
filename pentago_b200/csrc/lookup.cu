// Values of boards from solved slice files: block_cache_t::lookup and the
// high-level value() of a board (pentago/data/block_cache.cc:27-58,
// pentago/high/check.cc:21-37), batched on the GPU over a block cache in HBM.
//
// A call locates every board on the GPU (standardized section, block, index
// in the block, symmetry), the host brings the blocks not yet cached into
// free or least recently used cache slots (read and unfiltered by the slice
// reader), and a second kernel reads each board's node and applies the
// symmetry to both supers.
#include "../../include/pentago_b200.h"
#include "runtime.h"
#include "superscore.cuh"
#include <list>
#include <string>
#include <unordered_map>
#include <vector>

namespace pg {
namespace {

constexpr int kBlockNodes = 8 * 8 * 8 * 8;

struct lookup_loc_t {
  uint64_t section;   // standardized section of the board
  uint8_t block[4];
  uint16_t inblock;   // node index in the block (row-major in the block's shape)
  uint16_t sym;       // global << 8 | local: stored super -> the board's
  uint8_t turn;       // side to move (stone-count parity)
  uint8_t pad[7];
};
static_assert(sizeof(lookup_loc_t) == 24, "lookup_loc_t layout");

PG_HD int popc16(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __popc(x);
#else
  return __builtin_popcount(x);
#endif
}

// Quadrant sides rotated left r times.
PG_HD uint32_t rot_side(const dev_tables_t& T, uint32_t side, int r) {
  for (int i = 0; i < (r & 3); i++) side = ldg(T.rot + 2 * side);
  return side;
}

// transform_board(symmetry_t(g, 0), board) (pentago/base/symmetry.cc:46-78):
// rotate every quadrant by g, move the quadrants, reflect if g & 4.
PG_HD uint64_t board_global(const dev_tables_t& T, int g, uint64_t board) {
  const int src[4][4] = {{0, 1, 2, 3}, {1, 3, 0, 2}, {3, 2, 1, 0}, {2, 0, 3, 1}};
  uint32_t q[4][2], r[4][2];
  for (int i = 0; i < 4; i++) {
    const uint32_t v = uint32_t(board >> (16 * i) & 0xffff);
    q[i][0] = rot_side(T, ldg(T.unpack + 2 * v), g);
    q[i][1] = rot_side(T, ldg(T.unpack + 2 * v + 1), g);
  }
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 2; k++) r[i][k] = q[src[g & 3][i]][k];
  if (g & 4) {
    for (int k = 0; k < 2; k++) {
      const uint32_t t = r[0][k];
      r[0][k] = r[3][k];
      r[3][k] = t;
    }
    for (int i = 0; i < 4; i++)
      for (int k = 0; k < 2; k++) r[i][k] = ldg(T.refl + r[i][k]);
  }
  uint64_t out = 0;
  for (int i = 0; i < 4; i++) out |= uint64_t(ldg(T.pack + r[i][0]) + 2u * ldg(T.pack + r[i][1])) << (16 * i);
  return out;
}

// Counts of a section under global symmetry g (section_t::transform).
PG_HD uint64_t section_global(uint64_t sig, int g) {
  const int src[4][4] = {{0, 1, 2, 3}, {1, 3, 0, 2}, {3, 2, 1, 0}, {2, 0, 3, 1}};
  uint32_t c[4];
  for (int i = 0; i < 4; i++) c[i] = uint32_t(sig >> (16 * src[g & 3][i]) & 0xffff);
  if (g & 4) {
    const uint32_t t = c[0];
    c[0] = c[3];
    c[3] = t;
  }
  return uint64_t(c[0]) | uint64_t(c[1]) << 16 | uint64_t(c[2]) << 32 | uint64_t(c[3]) << 48;
}

// block_cache_t::lookup's location of an absolute board (block_cache.cc:27-58).
PG_HD lookup_loc_t lookup_locate(const dev_tables_t& T, uint64_t board, int* index_out = nullptr) {
  lookup_loc_t L = {};
  uint64_t sig = 0;
  int stones = 0;
  for (int q = 0; q < 4; q++) {
    const uint32_t v = uint32_t(board >> (16 * q) & 0xffff);
    const int b = popc16(ldg(T.unpack + 2 * v)), w = popc16(ldg(T.unpack + 2 * v + 1));
    sig |= uint64_t(b) << (16 * q) | uint64_t(w) << (16 * q + 8);
    stones += b + w;
  }
  // standardize<8>: the smallest signature over the global symmetries, the first on ties
  uint64_t best = sig;
  int g = 0;
  for (int t = 1; t < 8; t++) {
    const uint64_t s = section_global(sig, t);
    if (best > s) { best = s; g = t; }
  }
  const uint64_t b1 = board_global(T, g, board);
  int local = 0, idx[4];
  for (int q = 0; q < 4; q++) {
    const int ir = ldg(T.rmin_inv + uint32_t(b1 >> (16 * q) & 0xffff));
    idx[q] = ir >> 2;
    local |= (ir & 3) << (2 * q);
    if (index_out) index_out[q] = idx[q];
  }
  // shape of the standardized section, for the index inside the block
  int inblock = 0;
  for (int q = 0; q < 4; q++) {
    const int cb = int(best >> (16 * q) & 0xff), cw = int(best >> (16 * q + 8) & 0xff);
    const int k = cb * (21 - cb) / 2 + cw;
    const int shape = ldg(T.rmin_off + k + 1) - ldg(T.rmin_off + k);
    const int blk = idx[q] >> 3;
    L.block[q] = uint8_t(blk);
    const int extent = shape - 8 * blk < 8 ? shape - 8 * blk : 8;
    inblock = inblock * extent + (idx[q] & 7);
  }
  L.section = best;
  L.inblock = uint16_t(inblock);
  // symmetry1.inverse() * local_symmetry_t(local): the inverse of a global
  // symmetry is global, and a local factor on the right sets the local part
  L.sym = uint16_t(((g ^ ((~g >> 2 & (g & 1)) << 1)) << 8) | local);
  L.turn = uint8_t(stones & 1);
  return L;
}

__global__ void lookup_locate_kernel(const dev_tables_t T, const uint64_t* __restrict__ boards, int64_t n,
                                     lookup_loc_t* __restrict__ locs) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    locs[i] = lookup_locate(T, boards[i]);
}

// value(): win (1), tie (0) or loss (-1) for the side to move, from the
// node's [black wins, white wins] pair: extract (block_cache.cc:114-117) the
// mover's wins and win-or-tie, move them to the board's rotation, bit 0.
__global__ void lookup_value_kernel(const lookup_loc_t* __restrict__ locs, const int32_t* __restrict__ slots,
                                    int64_t n, const uint64_t* __restrict__ cache, int32_t* __restrict__ values) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const int32_t slot = slots[i];
    if (slot < 0) {
      values[i] = PG_LOOKUP_MISSING;
      continue;
    }
    const lookup_loc_t L = locs[i];
    const uint64_t* node = cache + 8 * (int64_t(slot) * kBlockNodes + L.inblock);
    const super8 black = s_load_ldg(node), white = s_load_ldg(node + 4);
    const super8 win = L.turn ? white : black;
    const super8 win_or_tie = s_not(L.turn ? black : white);
    const int g = L.sym >> 8, l = L.sym & 255;
    const int a = int(s_transform(win, g, l).w[0] & 1), b = int(s_transform(win_or_tie, g, l).w[0] & 1);
    values[i] = a + b - 1;
  }
}

struct block_key {
  uint64_t section;
  uint32_t block;
  bool operator==(const block_key& o) const { return section == o.section && block == o.block; }
};
struct block_key_hash {
  size_t operator()(const block_key& k) const { return std::hash<uint64_t>()(k.section * 0x9E3779B97F4A7C15ull ^ k.block); }
};

unsigned grid_for(int64_t n) { return unsigned(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32))); }

}  // namespace
}  // namespace pg

using namespace pg;

struct pg_lookup_s {
  std::vector<pg_supertensor_reader_t> readers;
  std::unordered_map<uint64_t, std::pair<int, int>> where;  // section -> (reader, section index)
  uint64_t* cache = nullptr;
  int slots = 0;
  // least recently used first
  std::list<block_key> lru;
  std::unordered_map<block_key, std::pair<int, std::list<block_key>::iterator>, block_key_hash> slot_of;
  std::vector<int> free_slots;
};

extern "C" int pg_lookup_open(const char* const* paths, int npaths, int64_t cache_bytes, pg_lookup_t* out) {
  if (!out || npaths < 0 || (npaths && !paths) || cache_bytes < 0) return fail(PG_ERR_ARG, "bad lookup arguments");
  *out = nullptr;
  const int64_t slot_bytes = int64_t(kBlockNodes) * 64;
  if (cache_bytes < slot_bytes) return fail(PG_ERR_ARG, "the block cache must hold at least one 256 KB block");
  if (!device_tables()) return PG_ERR_CUDA;
  auto* L = new pg_lookup_s;
  auto cleanup = [&](int rc) {
    pg_lookup_close(L);
    return rc;
  };
  for (int f = 0; f < npaths; f++) {
    pg_supertensor_reader_t r = nullptr;
    const int ns = pg_supertensor_open(paths[f], &r);
    if (ns < 0) return cleanup(ns);
    L->readers.push_back(r);
    for (int s = 0; s < ns; s++) {
      pg_supertensor_header_t h;
      pg_supertensor_header(r, s, &h);
      if (h.block_size != 8) return cleanup(fail(PG_ERR_FORMAT, "lookups need files of block size 8"));
      L->where.emplace(h.section, std::make_pair(f, s));
    }
  }
  L->slots = int(std::min<int64_t>(cache_bytes / slot_bytes, 1 << 30));
  if (cudaMalloc(&L->cache, size_t(L->slots) * slot_bytes) != cudaSuccess)
    return cleanup(fail(PG_ERR_CAPACITY, "cannot allocate the block cache"));
  for (int s = L->slots - 1; s >= 0; s--) L->free_slots.push_back(s);
  *out = L;
  return PG_OK;
}

extern "C" int pg_lookup_values(pg_lookup_t L, const uint64_t* boards, int64_t n, int32_t* values, void* stream_) {
  if (!L || n < 0 || (n && (!boards || !values))) return fail(PG_ERR_ARG, "bad lookup arguments");
  if (!n) return PG_OK;
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  cudaStream_t stream = (cudaStream_t)stream_;
  stream_scratch scratch(stream);
  uint64_t* b_dev = nullptr;
  lookup_loc_t* loc_dev = nullptr;
  int32_t *slot_dev = nullptr, *val_dev = nullptr;
  PG_CUDA(scratch.alloc(&b_dev, sizeof(uint64_t) * n));
  PG_CUDA(scratch.alloc(&loc_dev, sizeof(lookup_loc_t) * n));
  PG_CUDA(scratch.alloc(&slot_dev, sizeof(int32_t) * n));
  PG_CUDA(scratch.alloc(&val_dev, sizeof(int32_t) * n));
  PG_CUDA(cudaMemcpyAsync(b_dev, boards, sizeof(uint64_t) * n, cudaMemcpyHostToDevice, stream));
  lookup_locate_kernel<<<grid_for(n), 256, 0, stream>>>(*T, b_dev, n, loc_dev);
  PG_CUDA(cudaGetLastError());
  std::vector<lookup_loc_t> locs(n);
  PG_CUDA(cudaMemcpyAsync(locs.data(), loc_dev, sizeof(lookup_loc_t) * n, cudaMemcpyDeviceToHost, stream));
  PG_CUDA(cudaStreamSynchronize(stream));
  // The call's distinct blocks; refused before any change if they outnumber the slots
  std::vector<block_key> keys(n);
  std::vector<char> known(n, 0);
  std::unordered_map<block_key, int, block_key_hash> mine;  // block -> slot
  for (int64_t i = 0; i < n; i++) {
    if (!L->where.count(locs[i].section)) continue;
    keys[i] = {locs[i].section, uint32_t(locs[i].block[0]) | uint32_t(locs[i].block[1]) << 8 |
                                    uint32_t(locs[i].block[2]) << 16 | uint32_t(locs[i].block[3]) << 24};
    known[i] = 1;
    mine.emplace(keys[i], -1);
  }
  if (int64_t(mine.size()) > L->slots) return fail(PG_ERR_CAPACITY, "more distinct blocks than cache slots in one call");
  // Cached blocks move to the back of the LRU list, so that the missing ones,
  // which take free slots or evict from the front, never evict one of them
  for (auto& kv : mine) {
    const auto c = L->slot_of.find(kv.first);
    if (c == L->slot_of.end()) continue;
    kv.second = c->second.first;
    L->lru.erase(c->second.second);
    L->lru.push_back(kv.first);
    c->second.second = std::prev(L->lru.end());
  }
  std::vector<std::vector<std::pair<block_key, int>>> reads(L->readers.size());
  for (auto& kv : mine) {
    if (kv.second >= 0) continue;
    int slot;
    if (!L->free_slots.empty()) {
      slot = L->free_slots.back();
      L->free_slots.pop_back();
    } else {
      const block_key old = L->lru.front();
      L->lru.pop_front();
      slot = L->slot_of[old].first;
      L->slot_of.erase(old);
    }
    L->lru.push_back(kv.first);
    L->slot_of[kv.first] = std::make_pair(slot, std::prev(L->lru.end()));
    kv.second = slot;
    reads[L->where[kv.first.section].first].emplace_back(kv.first, slot);
  }
  std::vector<int32_t> slots(n, -1);
  for (int64_t i = 0; i < n; i++)
    if (known[i]) slots[i] = mine[keys[i]];
  for (size_t f = 0; f < reads.size(); f++) {
    if (reads[f].empty()) continue;
    std::vector<int32_t> secs;
    std::vector<uint8_t> blks;
    std::vector<int64_t> offs;
    for (const auto& kv : reads[f]) {
      secs.push_back(L->where[kv.first.section].second);
      for (int q = 0; q < 4; q++) blks.push_back(uint8_t(kv.first.block >> (8 * q)));
      offs.push_back(int64_t(kv.second) * kBlockNodes);
    }
    const int rc = pg_supertensor_read_blocks(L->readers[f], int(secs.size()), secs.data(), blks.data(), L->cache,
                                              offs.data(), PG_ST_RAW, 0, stream);
    if (rc) {
      // the slots of a failed read hold nothing valid
      for (const auto& kv : reads[f]) {
        L->lru.erase(L->slot_of[kv.first].second);
        L->slot_of.erase(kv.first);
        L->free_slots.push_back(kv.second);
      }
      return rc;
    }
  }
  PG_CUDA(cudaMemcpyAsync(slot_dev, slots.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream));
  lookup_value_kernel<<<grid_for(n), 256, 0, stream>>>(loc_dev, slot_dev, n, L->cache, val_dev);
  PG_CUDA(cudaGetLastError());
  PG_CUDA(cudaMemcpyAsync(values, val_dev, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, stream));
  PG_CUDA(cudaStreamSynchronize(stream));
  return PG_OK;
}

extern "C" int pg_lookup_close(pg_lookup_t L) {
  if (!L) return PG_OK;
  for (auto r : L->readers) pg_supertensor_close(r);
  if (L->cache) cudaFree(L->cache);
  delete L;
  return PG_OK;
}

extern "C" int pg_selftest_lookup_locate_host(const uint64_t* boards, int64_t n, uint64_t* sections, int32_t* index4,
                                              uint16_t* syms, int32_t* turns) {
  if (n < 0 || (n && (!boards || !sections || !index4 || !syms || !turns))) return fail(PG_ERR_ARG, "bad arguments");
  const dev_tables_t T = host_tables_view();
  for (int64_t i = 0; i < n; i++) {
    const lookup_loc_t L = lookup_locate(T, boards[i], index4 + 4 * i);
    sections[i] = L.section;
    syms[i] = L.sym;
    turns[i] = L.turn;
  }
  return PG_OK;
}
