// C entry points into the reference's own CPU engine, for tests and the CPU
// baseline only.  This file is compiled together with the reference sources
// (read in place, never copied) into oracle/_ref/libpentago_ref.so by
// oracle/Makefile.  Nothing in the product links it: it is the checker.
//
// Every function mirrors one reference interface:
//   ref_rmax / ref_super_wins        base/superscore.h:264-306, base/superscore.cc:38-96
//   ref_transform_super               base/symmetry.cc:146-307
//   ref_section_shape / ref_line_sizes base/section.h:73, end/compute.cc:24-46 (line_data_t)
//   ref_compute_line                  end/compute.cc:55-123 (line_details_t) + :394-404
//   ref_count_block_wins              end/block_store.cc:330-352
//   ref_midsolve                      mid/midengine.cc:161-169 (+ midsolve_traverse :127-158)
//   ref_rans_encode / ref_rans_decode shard/arithmetic.cc:366-452 (+ serialize :456-495)
//   ref_random_supers                 base/superscore.cc:118-127
//   ref_st_interleave                 data/filter.cc (interleave / uninterleave)
//   ref_shard_*                       shard/shard.cc (shard_mapping_t, scatter_block), shard/shard_permute.h
//   ref_block_write_order             data/supertensor_test.cc:31-55 (iteration order of its block map)

#include "pentago/base/board.h"
#include "pentago/base/count.h"
#include "pentago/base/section.h"
#include "pentago/base/superscore.h"
#include "pentago/base/symmetry.h"
#include "pentago/end/block_store.h"
#include "pentago/end/blocks.h"
#include "pentago/end/compute.h"
#include "pentago/end/sections.h"
#include "pentago/data/filter.h"
#include "pentago/base/all_boards.h"
#include "pentago/shard/shard.h"
#include "pentago/high/board.h"
#include "pentago/mid/halfsuper.h"
#include "pentago/mid/midengine.h"
#include "pentago/shard/arithmetic.h"
#include "pentago/shard/ternary.h"
#include "pentago/utility/thread.h"
#include "pentago/utility/vector.h"
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <chrono>
#include <thread>
#include <unordered_map>

using namespace pentago;
using namespace pentago::end;

namespace {

section_t section_from_sig(uint64_t sig) {
  section_t s;
  for (int q = 0; q < 4; q++)
    for (int c = 0; c < 2; c++)
      s.counts[q][c] = uint8_t(sig >> (16 * q + 8 * c));
  return s;
}

super_t load_super(const uint64_t* p) { return super_t(p[0], p[1], p[2], p[3]); }

void store_super(uint64_t* p, const super_t s) {
  for (int i = 0; i < 4; i++) p[i] = 0;
  for (int r = 0; r < 256; r++)
    if (s(uint8_t(r))) p[r >> 6] |= uint64_t(1) << (r & 63);
}

// The reference's thread pool (init_threads) runs its idle workers in a busy
// wait, so it is started when a call needs it and released by the caller when
// it has finished timing, before anything else runs on the host.
std::mutex threads_mutex;
int pool_threads = 0;

void ensure_threads(int n) {
  std::lock_guard<std::mutex> lock(threads_mutex);
  if (!pool_threads) {
    pool_threads = n > 0 ? n : default_threads();
    init_threads(pool_threads, 0);
  }
}

}  // namespace

extern "C" {

int ref_threads(int n) {
  ensure_threads(n);
  return pool_threads;
}

// Stop the thread pool (its workers spin while idle); a later call that
// needs it starts it again.
int ref_release_threads(void) {
  std::lock_guard<std::mutex> lock(threads_mutex);
  if (pool_threads) {
    shutdown_threads();
    pool_threads = 0;
  }
  return 0;
}

const void* ref_table(const char* name, int* bytes) {
#define T(x) if (!strcmp(name, #x)) { *bytes = sizeof(x); return (const void*)&x; }
  T(pack_table) T(unpack_table) T(win_contributions) T(rotations) T(reflections)
  T(superwin_info) T(commute_global_local_symmetries) T(superstandardize_table)
  T(rotation_minimal_quadrants_offsets) T(rotation_minimal_quadrants_flat)
  T(rotation_minimal_quadrants_inverse) T(rotation_minimal_quadrants_reflect_moved)
#undef T
  *bytes = 0;
  return nullptr;
}

void ref_rmax(const uint64_t* in, uint64_t* out, int n) {
  for (int i = 0; i < n; i++) store_super(out + 4 * i, rmax(load_super(in + 4 * i)));
}

void ref_super_wins(const uint64_t* sides, uint64_t* out, int n) {
  for (int i = 0; i < n; i++) store_super(out + 4 * i, super_wins(sides[i]));
}

// syms[i] = global << 8 | local
void ref_transform_super(const uint16_t* syms, const uint64_t* in, uint64_t* out, int n) {
  for (int i = 0; i < n; i++)
    store_super(out + 4 * i, transform_super(symmetry_t(syms[i] >> 8, syms[i] & 255), load_super(in + 4 * i)));
}

// syms: pairs (a, b) as global<<8|local; out = a*b in the same encoding
void ref_symmetry_product(const uint16_t* a, const uint16_t* b, uint16_t* out, int n) {
  for (int i = 0; i < n; i++) {
    const auto p = symmetry_t(a[i] >> 8, a[i] & 255) * symmetry_t(b[i] >> 8, b[i] & 255);
    out[i] = uint16_t(p.global << 8 | p.local);
  }
}

void ref_halfsuper_wins(const uint64_t* sides, const uint8_t* parity, uint64_t* out, int n) {
  for (int i = 0; i < n; i++) {
    const halfsuper_t h = halfsuper_wins(sides[i], parity[i]);
    for (int j = 0; j < 2; j++) out[2 * i + j] = 0;
    for (int r = 0; r < 128; r++)
      if (h[uint8_t(r)]) out[2 * i + (r >> 6)] |= uint64_t(1) << (r & 63);
  }
}

void ref_halfsuper_rmax(const uint64_t* in, uint64_t* out, int n) {
  for (int i = 0; i < n; i++) {
    const halfsuper_t h = rmax(halfsuper_t(in[2 * i], in[2 * i + 1]));
    for (int j = 0; j < 2; j++) out[2 * i + j] = 0;
    for (int r = 0; r < 128; r++)
      if (h[uint8_t(r)]) out[2 * i + (r >> 6)] |= uint64_t(1) << (r & 63);
  }
}

// section_t::shape (base/section.h:73): rotation-minimal quadrant counts.
int ref_section_shape(uint64_t section_sig, int32_t* shape) {
  const auto s = section_from_sig(section_sig).shape();
  for (int i = 0; i < 4; i++) shape[i] = s[i];
  return 0;
}

// Shapes for a line: fills input_nodes/output_nodes (node counts of the packed
// input child line and the packed output line).  Returns 0 or -1 on bad input.
int ref_line_sizes(uint64_t section_sig, int dim, int length, const uint8_t* block_base,
                   int64_t* input_nodes, int64_t* output_nodes) {
  line_t line;
  line.section = section_from_sig(section_sig);
  line.dimension = dim;
  line.length = length;
  line.block_base = Vector<uint8_t,3>(block_base[0], block_base[1], block_base[2]);
  const line_data_t pre(line);
  *input_nodes = pre.input_shape.product();
  *output_nodes = pre.output_shape.product();
  return 0;
}

// Compute one block line with the reference's own line_details_t +
// schedule_compute_line on the reference thread pool.  `input` holds the child
// line's blocks packed back to back (each block row-major in its own block
// shape, no padding), `output` receives the parent line's blocks packed the
// same way.  Each node is 8 uint64 = [win(4), notlost(4)].
int ref_compute_line(uint64_t section_sig, int dim, int length, const uint8_t* block_base,
                     const uint64_t* input, uint64_t* output, int threads) {
  ensure_threads(threads);
  line_t line;
  line.section = section_from_sig(section_sig);
  line.dimension = dim;
  line.length = length;
  line.block_base = Vector<uint8_t,3>(block_base[0], block_base[1], block_base[2]);
  const line_data_t pre(line);
  std::mutex m;
  std::condition_variable cv;
  bool done = false;
  line_details_t details(pre, [&](line_details_t&, unit_t) {
    std::lock_guard<std::mutex> lock(m);
    done = true;
    cv.notify_all();
  });
  // Scatter packed input into the padded (block_stride + 1) layout
  const int nin = details.input_blocks;
  int64_t offset = 0;
  for (int k = 0; k < nin; k++) {
    const auto dst = details.input_block_data(k);
    // The reference reserves one extra slot per input block for compressed
    // receives; the real block is the first (nodes in block) entries.
    auto block = details.input_block(k);
    const auto child_shape = block_shape(details.standard_child_section.shape(), block);
    const int64_t nodes = Vector<int64_t,4>(child_shape).product();
    memcpy((void*)dst.data(), input + 8 * offset, 64 * nodes);
    offset += nodes;
  }
  if (pre.output_shape.product() == 0) return 0;
  schedule_compute_line(details);
  {
    std::unique_lock<std::mutex> lock(m);
    cv.wait(lock, [&] { return done; });
  }
  memcpy(output, details.output.data(), 64 * details.output.size());
  return 0;
}

// Per-block (win, win-or-tie, total) counts over distinct positions, in
// we-win/we-win-or-tie form.  Same loop as count_block_wins
// (end/block_store.cc:330-352), which lives in a file that also pulls in the
// compressed block store; the per-node work is the reference's own
// popcounts_over_stabilizers (base/count.cc:235-261).
void ref_count_block_wins(uint64_t section_sig, const uint8_t* block, const uint64_t* data,
                          uint64_t* counts3) {
  const auto section = section_from_sig(section_sig);
  const Vector<uint8_t,4> b(block[0], block[1], block[2], block[3]);
  const auto base = block_size * Vector<int,4>(b);
  const auto shape = block_shape(section.shape(), b);
  const auto r0 = safe_rmin_slice(section.counts[0], base[0] + range(shape[0])),
             r1 = safe_rmin_slice(section.counts[1], base[1] + range(shape[1])),
             r2 = safe_rmin_slice(section.counts[2], base[2] + range(shape[2])),
             r3 = safe_rmin_slice(section.counts[3], base[3] + range(shape[3]));
  const Vector<super_t,2>* nodes = (const Vector<super_t,2>*)data;
  Vector<uint64_t,3> c;
  int i = 0;
  for (int i0 = 0; i0 < shape[0]; i0++)
    for (int i1 = 0; i1 < shape[1]; i1++)
      for (int i2 = 0; i2 < shape[2]; i2++)
        for (int i3 = 0; i3 < shape[3]; i3++)
          c += Vector<uint64_t,3>(popcounts_over_stabilizers(quadrants(r0[i0], r1[i1], r2[i2], r3[i3]), nodes[i++]));
  for (int k = 0; k < 3; k++) counts3[k] = c[k];
}

// Standardized descendant sections of root at `slice` (sorted by sig).
// Returns the count; writes up to cap sigs.
int ref_descendent_sections(uint64_t root_sig, int slice, uint64_t* sigs, int cap) {
  const auto slices = descendent_sections(section_from_sig(root_sig), 35);
  const auto& s = slices.at(slice)->sections;
  for (int i = 0; i < s.size() && i < cap; i++) sigs[i] = s[i].sig();
  return s.size();
}

// Midsolve one board given as raw_t.  Writes up to 1+18+8*18 (raw, value)
// pairs in the reference's traversal order; returns the count.
int ref_midsolve(uint64_t raw, uint64_t* out_raws, int32_t* out_values) {
  const auto board = high_board_t::from_raw(raw);
  static thread_local Array<halfsuper_s> workspace;
  const int need = midsolve_workspace_size(board.count());
  if (workspace.size() < need) workspace = midsolve_workspace(board.count());
  const auto results = midsolve(board, workspace);
  int i = 0;
  for (const auto& [r, v] : results) {
    out_raws[i] = r;
    out_values[i] = v;
    i++;
  }
  return i;
}

// midsolve_internal's raw halfsupers: out holds (1+18) x (win, notlose) x 2 uint64
void ref_midsolve_internal(uint64_t raw, uint64_t* out) {
  const auto board = high_board_t::from_raw(raw);
  const auto workspace = midsolve_workspace(board.count());
  const auto r = midsolve_internal(board, workspace);
  memcpy(out, &r, sizeof(r));
}

int ref_midsolve_workspace_size(int stones) { return midsolve_workspace_size(stones); }

// Static rANS: symbols in {0,1,2}; writes the serialized v2 stream into out
// (capacity cap) and returns its size, or -1 if cap is too small.
int64_t ref_rans_encode(const uint8_t* symbols, int64_t n, uint8_t* out, int64_t cap) {
  ternaries_t t(n);
  for (int64_t i = 0; i < n; i++) t.set(i, symbols[i]);
  const auto enc = arithmetic_encode(t);
  const auto buf = arithmetic_serialize(enc);
  if (buf.size() > cap) return -1;
  memcpy(out, buf.data(), buf.size());
  return buf.size();
}

int64_t ref_rans_decode(const uint8_t* data, int64_t size, uint8_t* symbols, int64_t cap) {
  try {
    const auto enc = arithmetic_deserialize(RawArray<const uint8_t>(size, data));
    const auto t = arithmetic_decode(enc);
    if (int64_t(t.size) > cap) return -1;
    for (uint64_t i = 0; i < t.size; i++) symbols[i] = t[i];
    return t.size;
  } catch (...) {
    return -2;
  }
}

// random_supers(key, n) with key = hi << 64 | lo: n supers of 4 words each.
void ref_random_supers(uint64_t key_hi, uint64_t key_lo, int n, uint64_t* out) {
  const auto s = random_supers((uint128_t(key_hi) << 64) | key_lo, n);
  for (int i = 0; i < n; i++) store_super(out + 4 * i, s[i]);
}

// interleave (inverse = 0) or uninterleave (1) n on-disk pairs in place.
void ref_st_interleave(uint64_t* data, int64_t n, int inverse) {
  Array<Vector<super_t,2>> a(static_cast<int>(n));
  for (int64_t i = 0; i < n; i++)
    for (int k = 0; k < 2; k++) a[i][k] = load_super(data + 8 * i + 4 * k);
  if (inverse) uninterleave(a);
  else interleave(a);
  for (int64_t i = 0; i < n; i++)
    for (int k = 0; k < 2; k++) store_super(data + 8 * i + 4 * k, a[i][k]);
}

// Shards: sections of a slice in the mapping's order, the entry count, the
// permutation, boards of shuffled indices, and scatter_block of blocks of
// on-disk pairs (block b: section sigs[b], coordinates blocks[4b..], shape
// shapes[4b..], nodes at data + 8 * offsets[b]) into one shard's symbols.
int ref_shard_sections(int slice, uint64_t* sigs, int cap) {
  const auto s = all_boards_sections(slice, 8);
  for (int i = 0; i < s.size() && i < cap; i++) {
    uint64_t sig = 0;
    for (int q = 0; q < 4; q++)
      for (int c = 0; c < 2; c++) sig |= uint64_t(s[i].counts[q][c]) << (16 * q + 8 * c);
    sigs[i] = sig;
  }
  return s.size();
}

uint64_t ref_shard_total(int slice) { return shard_mapping_t(slice).total(); }

void ref_shard_permute(int slice, const uint64_t* in, int64_t n, int inverse, uint64_t* out) {
  const shard_permute_t p(slice);
  for (int64_t i = 0; i < n; i++) out[i] = inverse ? p.inverse(in[i]) : p.forward(in[i]);
}

void ref_shard_board(int slice, const uint64_t* in, int64_t n, uint64_t* out) {
  const shard_mapping_t m(slice);
  for (int64_t i = 0; i < n; i++) out[i] = m.board(in[i]);
}

void ref_shard_scatter(int slice, int total_shards, int shard, int nblocks, const uint64_t* sigs,
                       const uint8_t* blocks, const int* shapes, const int64_t* offsets, const uint64_t* data,
                       uint8_t* out) {
  const shard_mapping_t m(slice);
  const shard_locator_t loc(total_shards, range(shard, shard + 1));
  ternaries_t buf(loc.shard_size(m.total(), shard));
  for (int b = 0; b < nblocks; b++) {
    const Vector<int,4> shape(shapes[4 * b], shapes[4 * b + 1], shapes[4 * b + 2], shapes[4 * b + 3]);
    const auto* nodes = reinterpret_cast<const Vector<super_t,2>*>(data + 8 * offsets[b]);
    const RawArray<const Vector<super_t,2>,4> block_data(shape, nodes);
    scatter_block(m, total_shards, range(shard, shard + 1), RawArray<ternaries_t>(1, &buf),
                  section_from_sig(sigs[b]),
                  Vector<uint8_t,4>(blocks[4 * b], blocks[4 * b + 1], blocks[4 * b + 2], blocks[4 * b + 3]), block_data);
  }
  for (uint64_t i = 0; i < buf.size; i++) out[i] = uint8_t(buf[i]);
}

// Seconds the reference's scatter_block takes for the given blocks into every
// shard of total_shards (one buffer per shard), on `threads` host threads
// taking blocks in turn (as sharder.cc's parallel_for does).
double ref_shard_scatter_seconds(int slice, int total_shards, int nblocks, const uint64_t* sigs,
                                 const uint8_t* blocks, const int* shapes, const int64_t* offsets,
                                 const uint64_t* data, int threads) {
  const shard_mapping_t m(slice);
  const shard_locator_t loc(total_shards, range(0, total_shards));
  vector<ternaries_t> buffers;
  for (int s = 0; s < total_shards; s++) buffers.emplace_back(loc.shard_size(m.total(), s));
  std::atomic<int> next{0};
  const auto t0 = std::chrono::steady_clock::now();
  auto work = [&] {
    for (int b; (b = next.fetch_add(1)) < nblocks;) {
      const Vector<int,4> shape(shapes[4 * b], shapes[4 * b + 1], shapes[4 * b + 2], shapes[4 * b + 3]);
      const auto* nodes = reinterpret_cast<const Vector<super_t,2>*>(data + 8 * offsets[b]);
      scatter_block(m, total_shards, range(0, total_shards), asarray(buffers), section_from_sig(sigs[b]),
                    Vector<uint8_t,4>(blocks[4 * b], blocks[4 * b + 1], blocks[4 * b + 2], blocks[4 * b + 3]),
                    RawArray<const Vector<super_t,2>,4>(shape, nodes));
    }
  };
  vector<std::thread> pool;
  for (int t = 1; t < threads; t++) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// The order in which supertensor_test.cc writes its blocks: it inserts every
// block of a blocks[0] x .. x blocks[3] grid, in row-major order, into an
// unordered_map keyed by Vector<uint8_t,4> and writes them in the map's
// iteration order.  Returns the block count; out gets 4 bytes per block.
int ref_block_write_order(const int* blocks, uint8_t* out) {
  std::unordered_map<Vector<uint8_t,4>, int> data;
  for (int i = 0; i < blocks[0]; i++)
    for (int j = 0; j < blocks[1]; j++)
      for (int k = 0; k < blocks[2]; k++)
        for (int l = 0; l < blocks[3]; l++)
          data[vec(uint8_t(i), uint8_t(j), uint8_t(k), uint8_t(l))] = 0;
  int n = 0;
  for (const auto& e : data) {
    for (int a = 0; a < 4; a++) out[4 * n + a] = e.first[a];
    n++;
  }
  return n;
}

}  // extern "C"
