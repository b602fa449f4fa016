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
#include <algorithm>
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

// Cache keys: the section's eight counts (4 bits each) and the block's four
// coordinates (6 bits each) in one word; ~0 marks an empty table entry.
PG_HD uint64_t block_key(const lookup_loc_t& L) {
  uint64_t k = 0;
  for (int i = 0; i < 8; i++) k |= (L.section >> (8 * i) & 15) << (4 * i);
  for (int q = 0; q < 4; q++) k |= uint64_t(L.block[q] & 63) << (32 + 6 * q);
  return k;
}
constexpr uint64_t kEmpty = ~uint64_t(0);

PG_HD uint64_t key_hash(uint64_t k) {
  k ^= k >> 29;
  k *= 0xBF58476D1CE4E5B9ull;
  k ^= k >> 32;
  return k;
}

// The open-addressed (linear probing) map block -> cache slot, mirrored on
// the device; the host edits it when blocks come and go.
struct slot_table {
  uint64_t* keys;   // mask + 1 entries
  int32_t* slots;
  uint64_t mask;
};

PG_HD int32_t table_find(const slot_table& H, uint64_t key) {
  for (uint64_t i = key_hash(key) & H.mask;; i = (i + 1) & H.mask) {
    const uint64_t k = ldg(H.keys + i);
    if (k == key) return ldg(H.slots + i);
    if (k == kEmpty) return -1;
  }
}

// Sections the open files hold (sorted), for telling missing boards apart.
PG_HD bool section_known(const uint64_t* secs, int n, uint64_t s) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ldg(secs + mid) < s) lo = mid + 1; else hi = mid;
  }
  return lo < n && ldg(secs + lo) == s;
}

// Locate every board and find its block in the cache: slot >= 0 (and the
// slot is marked used by this call), PG_LOOKUP_MISSING for boards of no
// open section, or -1 with the board queued for the host.
__global__ void lookup_probe_kernel(const dev_tables_t T, const uint64_t* __restrict__ boards, int64_t n,
                                    const uint64_t* __restrict__ secs, int nsecs, const slot_table H,
                                    lookup_loc_t* __restrict__ locs, int32_t* __restrict__ slot_of_board,
                                    uint32_t* __restrict__ used, uint32_t call, unsigned long long* __restrict__ nmiss,
                                    int64_t* __restrict__ misses) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const lookup_loc_t L = lookup_locate(T, boards[i]);
    locs[i] = L;
    int32_t slot = PG_LOOKUP_MISSING;
    if (section_known(secs, nsecs, L.section)) {
      slot = table_find(H, block_key(L));
      if (slot >= 0) used[slot] = call;
      else misses[atomicAdd(nmiss, 1ull)] = i;
    }
    slot_of_board[i] = slot;
  }
}

// The queued boards, once their blocks are in the cache.
__global__ void lookup_reprobe_kernel(const int64_t* __restrict__ misses, int64_t m, const lookup_loc_t* __restrict__ locs,
                                      const slot_table H, int32_t* __restrict__ slot_of_board) {
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < m; j += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = misses[j];
    slot_of_board[i] = table_find(H, block_key(locs[i]));
  }
}

unsigned grid_for(int64_t n) { return unsigned(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32))); }

}  // namespace
}  // namespace pg

using namespace pg;

struct pg_lookup_s {
  std::vector<pg_supertensor_reader_t> readers;
  std::unordered_map<uint64_t, std::pair<int, int>> where;  // section -> (reader, section index)
  uint64_t* secs_dev = nullptr;                             // the sections, sorted
  int nsecs = 0;
  uint64_t* cache = nullptr;
  int slots = 0;
  // block -> slot map: host copy and device copy
  std::vector<uint64_t> keys;
  std::vector<int32_t> table_slots;
  slot_table dev = {nullptr, nullptr, 0};
  std::vector<uint64_t> key_of_slot;  // kEmpty when free
  uint32_t* used_dev = nullptr;       // per slot: the last call that used it
  uint32_t call = 0;
  int hand = 0;                       // next slot the eviction looks at
  int64_t hits = 0, reads = 0;
};

namespace {

void table_insert(pg_lookup_s& L, uint64_t key, int32_t slot) {
  uint64_t i = key_hash(key) & L.dev.mask;
  while (L.keys[i] != kEmpty) i = (i + 1) & L.dev.mask;
  L.keys[i] = key;
  L.table_slots[i] = slot;
}

// Removal from a linear-probing table: later entries of the run move back
// into the hole when their home position allows it.
void table_erase(pg_lookup_s& L, uint64_t key) {
  const uint64_t m = L.dev.mask;
  uint64_t i = key_hash(key) & m;
  while (L.keys[i] != key) {
    if (L.keys[i] == kEmpty) return;
    i = (i + 1) & m;
  }
  for (uint64_t j = (i + 1) & m;; j = (j + 1) & m) {
    if (L.keys[j] == kEmpty) break;
    const uint64_t h = key_hash(L.keys[j]) & m;
    // entry j may fill hole i if its home h is not cyclically inside (i, j]
    if (((j - h) & m) >= ((j - i) & m)) {
      L.keys[i] = L.keys[j];
      L.table_slots[i] = L.table_slots[j];
      i = j;
    }
  }
  L.keys[i] = kEmpty;
  L.table_slots[i] = -1;
}

}  // namespace

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
  std::vector<uint64_t> secs;
  for (int f = 0; f < npaths; f++) {
    pg_supertensor_reader_t r = nullptr;
    const int ns = pg_supertensor_open(paths[f], &r);
    if (ns < 0) return cleanup(ns);
    L->readers.push_back(r);
    for (int s = 0; s < ns; s++) {
      pg_supertensor_header_t h;
      pg_supertensor_header(r, s, &h);
      if (h.block_size != 8) return cleanup(fail(PG_ERR_FORMAT, "lookups need files of block size 8"));
      if (L->where.emplace(h.section, std::make_pair(f, s)).second) secs.push_back(h.section);
    }
  }
  std::sort(secs.begin(), secs.end());
  L->nsecs = int(secs.size());
  L->slots = int(std::min<int64_t>(cache_bytes / slot_bytes, 1 << 28));
  uint64_t cap = 2;
  while (cap < 2 * uint64_t(L->slots)) cap <<= 1;
  L->keys.assign(cap, kEmpty);
  L->table_slots.assign(cap, -1);
  L->key_of_slot.assign(L->slots, kEmpty);
  L->dev.mask = cap - 1;
  if (cudaMalloc(&L->cache, size_t(L->slots) * slot_bytes) != cudaSuccess ||
      cudaMalloc(&L->dev.keys, sizeof(uint64_t) * cap) != cudaSuccess ||
      cudaMalloc(&L->dev.slots, sizeof(int32_t) * cap) != cudaSuccess ||
      cudaMalloc(&L->used_dev, sizeof(uint32_t) * L->slots) != cudaSuccess ||
      cudaMalloc(&L->secs_dev, sizeof(uint64_t) * std::max<size_t>(secs.size(), 1)) != cudaSuccess)
    return cleanup(fail(PG_ERR_CAPACITY, "cannot allocate the block cache"));
  if (cudaMemcpy(L->dev.keys, L->keys.data(), sizeof(uint64_t) * cap, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(L->dev.slots, L->table_slots.data(), sizeof(int32_t) * cap, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(L->used_dev, 0, sizeof(uint32_t) * L->slots) != cudaSuccess ||
      (secs.size() && cudaMemcpy(L->secs_dev, secs.data(), sizeof(uint64_t) * secs.size(), cudaMemcpyHostToDevice) != cudaSuccess))
    return cleanup(fail(PG_ERR_CUDA, "cannot initialize the block cache"));
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
  int64_t* miss_dev = nullptr;
  unsigned long long* nmiss_dev = nullptr;
  PG_CUDA(scratch.alloc(&b_dev, sizeof(uint64_t) * n));
  PG_CUDA(scratch.alloc(&loc_dev, sizeof(lookup_loc_t) * n));
  PG_CUDA(scratch.alloc(&slot_dev, sizeof(int32_t) * n));
  PG_CUDA(scratch.alloc(&val_dev, sizeof(int32_t) * n));
  PG_CUDA(scratch.alloc(&miss_dev, sizeof(int64_t) * n));
  PG_CUDA(scratch.alloc(&nmiss_dev, sizeof(unsigned long long)));
  const uint32_t call = ++L->call;
  PG_CUDA(cudaMemsetAsync(nmiss_dev, 0, sizeof(unsigned long long), stream));
  PG_CUDA(cudaMemcpyAsync(b_dev, boards, sizeof(uint64_t) * n, cudaMemcpyHostToDevice, stream));
  lookup_probe_kernel<<<grid_for(n), 256, 0, stream>>>(*T, b_dev, n, L->secs_dev, L->nsecs, L->dev, loc_dev, slot_dev,
                                                       L->used_dev, call, nmiss_dev, miss_dev);
  PG_CUDA(cudaGetLastError());
  unsigned long long m = 0;
  PG_CUDA(cudaMemcpyAsync(&m, nmiss_dev, sizeof m, cudaMemcpyDeviceToHost, stream));
  PG_CUDA(cudaStreamSynchronize(stream));
  L->hits += n - int64_t(m);
  if (m) {
    // Which blocks the queued boards need
    std::vector<int64_t> miss(m);
    std::vector<lookup_loc_t> locs(n);
    PG_CUDA(cudaMemcpyAsync(miss.data(), miss_dev, sizeof(int64_t) * m, cudaMemcpyDeviceToHost, stream));
    PG_CUDA(cudaMemcpyAsync(locs.data(), loc_dev, sizeof(lookup_loc_t) * n, cudaMemcpyDeviceToHost, stream));
    std::vector<uint32_t> used(L->slots);
    PG_CUDA(cudaMemcpyAsync(used.data(), L->used_dev, sizeof(uint32_t) * L->slots, cudaMemcpyDeviceToHost, stream));
    PG_CUDA(cudaStreamSynchronize(stream));
    std::unordered_map<uint64_t, const lookup_loc_t*> need;
    for (int64_t i : miss) need.emplace(block_key(locs[i]), &locs[i]);
    int64_t busy = 0;
    for (int s = 0; s < L->slots; s++) busy += used[s] == call;
    if (busy + int64_t(need.size()) > L->slots)
      return fail(PG_ERR_CAPACITY, "more distinct blocks than cache slots in one call");
    // Slots not used by this call, free ones first, then round the clock
    std::vector<std::vector<std::pair<const lookup_loc_t*, int>>> reads(L->readers.size());
    std::vector<int> taken;
    for (const auto& kv : need) {
      int slot = -1;
      for (int tries = 0; tries < L->slots && slot < 0; tries++) {
        const int s = L->hand;
        L->hand = (L->hand + 1) % L->slots;
        if (used[s] == call) continue;
        slot = s;
      }
      used[slot] = call;
      if (L->key_of_slot[slot] != kEmpty) table_erase(*L, L->key_of_slot[slot]);
      L->key_of_slot[slot] = kv.first;
      table_insert(*L, kv.first, slot);
      taken.push_back(slot);
      reads[L->where[kv.second->section].first].emplace_back(kv.second, slot);
    }
    int rc = PG_OK;
    for (size_t f = 0; f < reads.size() && rc == PG_OK; f++) {
      if (reads[f].empty()) continue;
      std::vector<int32_t> secs;
      std::vector<uint8_t> blks;
      std::vector<int64_t> offs;
      for (const auto& r : reads[f]) {
        secs.push_back(L->where[r.first->section].second);
        for (int q = 0; q < 4; q++) blks.push_back(r.first->block[q]);
        offs.push_back(int64_t(r.second) * kBlockNodes);
      }
      rc = pg_supertensor_read_blocks(L->readers[f], int(secs.size()), secs.data(), blks.data(), L->cache,
                                      offs.data(), PG_ST_RAW, 0, stream);
      L->reads += int64_t(secs.size());
    }
    if (rc != PG_OK) {
      // the slots of this call's reads hold nothing valid
      for (int s : taken) {
        table_erase(*L, L->key_of_slot[s]);
        L->key_of_slot[s] = kEmpty;
      }
    }
    const uint64_t cap = L->dev.mask + 1;
    PG_CUDA(cudaMemcpyAsync(L->dev.keys, L->keys.data(), sizeof(uint64_t) * cap, cudaMemcpyHostToDevice, stream));
    PG_CUDA(cudaMemcpyAsync(L->dev.slots, L->table_slots.data(), sizeof(int32_t) * cap, cudaMemcpyHostToDevice, stream));
    PG_CUDA(cudaMemcpyAsync(L->used_dev, used.data(), sizeof(uint32_t) * L->slots, cudaMemcpyHostToDevice, stream));
    // the host copies above are read before they change again
    PG_CUDA(cudaStreamSynchronize(stream));
    if (rc != PG_OK) return rc;
    lookup_reprobe_kernel<<<grid_for(int64_t(m)), 256, 0, stream>>>(miss_dev, int64_t(m), loc_dev, L->dev, slot_dev);
    PG_CUDA(cudaGetLastError());
  }
  lookup_value_kernel<<<grid_for(n), 256, 0, stream>>>(loc_dev, slot_dev, n, L->cache, val_dev);
  PG_CUDA(cudaGetLastError());
  PG_CUDA(cudaMemcpyAsync(values, val_dev, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, stream));
  PG_CUDA(cudaStreamSynchronize(stream));
  return PG_OK;
}

extern "C" int pg_lookup_close(pg_lookup_t L) {
  if (!L) return PG_OK;
  for (auto r : L->readers) pg_supertensor_close(r);
  for (void* p : {(void*)L->cache, (void*)L->dev.keys, (void*)L->dev.slots, (void*)L->used_dev, (void*)L->secs_dev})
    if (p) cudaFree(p);
  delete L;
  return PG_OK;
}

extern "C" int pg_lookup_stats(pg_lookup_t L, int64_t* stats3) {
  if (!L || !stats3) return fail(PG_ERR_ARG, "bad arguments");
  stats3[0] = L->hits;
  stats3[1] = L->reads;
  stats3[2] = L->slots;
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
