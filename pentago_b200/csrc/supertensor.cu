// Slice files in the reference's .pentago supertensor format
// (pentago/data/supertensor.h:1-232, pentago/data/supertensor.cc): packed
// headers, compressed block indices, blocks compressed one by one with zlib
// or xz (compress / decompress, pentago/data/compress.cc:34-95) on host
// threads, and the interleave filter with the node-form conversion of the
// slice writer and reader (pentago/mpi/io.cc:69-88, 468-481) as GPU kernels.
//
// Device reads and writes move blocks in batches through pinned host
// buffers: while the host threads (de)compress one batch, the GPU copies and
// (un)filters the other.
#include "../../include/pentago_b200.h"
#include "lines.h"
#include "runtime.h"
#include <zlib.h>
#include <dlfcn.h>
#include <errno.h>
#include <fcntl.h>
#include <unistd.h>
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "the file format is little endian, and so must the host be");

namespace pg {
namespace {

constexpr int kHeaderBytes = 85;
constexpr int kPreheaderBytes = 20 + 3 * 4;        // magic, version, sections, header size
const char kSingleMagic[21] = "pentago supertensor\n";
const char kMultipleMagic[21] = "pentago sections   \n";
constexpr uint32_t kMaxSections = 8239;            // open_supertensors' bound (supertensor.cc:428-429)
constexpr size_t kBatchBytes = size_t(128) << 20;  // on-disk bytes per device batch

struct blob_t {
  uint64_t uncompressed, compressed, offset;
};
static_assert(sizeof(blob_t) == 24, "an index entry is 3 little-endian uint64");

// --------------------------------------------------------------------------
// Filter kernels.  Thread t handles half h = t & 1 of node t >> 1: words 2h,
// 2h+1 of both supers of the pair, which are exactly the inputs of
// interleaved super h (interleave_super, pentago/data/filter.h:76-100).

struct seg_t {
  int64_t src, dst, n;  // node offsets into the source and destination, node count
};

// Bit interleave of two 16-bit halves: z = [x0 x1 y0 y1] (bytes, from a
// byte permute) becomes x's bits at the even and y's at the odd positions by
// three delta swaps (the outer perfect shuffle, Hacker's Delight 7-2, after
// its first stage, which the byte permute already did).  unshuffle32 undoes
// the three swaps in reverse order (each swap is its own inverse).
__device__ __forceinline__ uint32_t delta_swap(uint32_t z, uint32_t m, int k) {
  const uint32_t t = (z ^ (z >> k)) & m;
  return z ^ t ^ (t << k);
}
__device__ __forceinline__ uint32_t shuffle32(uint32_t z) {
  z = delta_swap(z, 0x00f000f0u, 4);
  z = delta_swap(z, 0x0c0c0c0cu, 2);
  return delta_swap(z, 0x22222222u, 1);
}
__device__ __forceinline__ uint32_t unshuffle32(uint32_t z) {
  z = delta_swap(z, 0x22222222u, 1);
  z = delta_swap(z, 0x0c0c0c0cu, 2);
  return delta_swap(z, 0x00f000f0u, 4);
}

// One interleaved 64-bit word from 32 bits of each super: bit i of a goes to
// bit 2i, bit i of b to bit 2i+1 (EXPAND(a) | EXPAND(b) << 1 of filter.h).
__device__ __forceinline__ uint2 interleave_word(uint32_t a, uint32_t b) {
  return make_uint2(shuffle32(__byte_perm(a, b, 0x5140)), shuffle32(__byte_perm(a, b, 0x7362)));
}
// Its inverse: the even bits of w to a, the odd bits to b.
__device__ __forceinline__ void deinterleave_word(uint2 w, uint32_t& a, uint32_t& b) {
  const uint32_t lo = unshuffle32(w.x), hi = unshuffle32(w.y);
  a = __byte_perm(lo, hi, 0x6420);
  b = __byte_perm(lo, hi, 0x7531);
}

__device__ __forceinline__ uint4 u4_not(uint4 a) { return make_uint4(~a.x, ~a.y, ~a.z, ~a.w); }
__device__ __forceinline__ uint4 u4_of(uint2 lo, uint2 hi) { return make_uint4(lo.x, lo.y, hi.x, hi.y); }

// Nodes -> on-disk bytes.  Node form [we win, we win or tie] becomes [black
// wins, white wins] (io.cc:79-86); PG_ST_RAW nodes already are that pair.
__global__ void __launch_bounds__(256, 8)
st_filter_kernel(const uint4* __restrict__ in, uint4* __restrict__ out, const seg_t* __restrict__ segs, int seg0,
                 int turn, int filter) {
  const seg_t s = segs[seg0 + blockIdx.y];
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < 2 * s.n; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t node = t >> 1;
    const int h = int(t & 1);
    const uint4* p = in + 4 * (s.src + node);
    uint4* q = out + 4 * (s.dst + node);
    const uint4 a = p[h], b = p[2 + h];  // words 2h, 2h+1 of the first and second super
    uint4 s0, s1;
    if (turn == 0) { s0 = a; s1 = u4_not(b); }
    else if (turn == 1) { s0 = u4_not(b); s1 = a; }
    else { s0 = a; s1 = b; }
    if (filter) {
      q[2 * h] = u4_of(interleave_word(s0.x, s1.x), interleave_word(s0.y, s1.y));
      q[2 * h + 1] = u4_of(interleave_word(s0.z, s1.z), interleave_word(s0.w, s1.w));
    } else {
      q[h] = s0;
      q[2 + h] = s1;
    }
  }
}

// On-disk bytes -> nodes (uninterleave_super, filter.h:102-127, then io.cc:476-481).
__global__ void __launch_bounds__(256, 8)
st_unfilter_kernel(const uint4* __restrict__ in, uint4* __restrict__ out, const seg_t* __restrict__ segs, int seg0,
                   int turn, int filter) {
  const seg_t s = segs[seg0 + blockIdx.y];
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < 2 * s.n; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t node = t >> 1;
    const int h = int(t & 1);
    const uint4* p = in + 4 * (s.src + node);
    uint4* q = out + 4 * (s.dst + node);
    uint4 s0, s1;
    if (filter) {
      const uint4 u = p[2 * h], v = p[2 * h + 1];  // interleaved super h
      deinterleave_word(make_uint2(u.x, u.y), s0.x, s1.x);
      deinterleave_word(make_uint2(u.z, u.w), s0.y, s1.y);
      deinterleave_word(make_uint2(v.x, v.y), s0.z, s1.z);
      deinterleave_word(make_uint2(v.z, v.w), s0.w, s1.w);
    } else {
      s0 = p[h];
      s1 = p[2 + h];
    }
    if (turn == 0) { q[h] = s0; q[2 + h] = u4_not(s1); }
    else if (turn == 1) { q[h] = s1; q[2 + h] = u4_not(s0); }
    else { q[h] = s0; q[2 + h] = s1; }
  }
}

// Launch over segments (device table) in chunks of at most 65535 per grid row.
int launch_segments(bool to_disk, const void* in, void* out, const seg_t* segs_dev, int nseg, int64_t max_nodes,
                    int turn, int filter, cudaStream_t stream) {
  if (!nseg || !max_nodes) return PG_OK;
  const int64_t want = (2 * max_nodes + 255) / 256;
  for (int s0 = 0; s0 < nseg; s0 += 65535) {
    const int ns = std::min(65535, nseg - s0);
    const unsigned gx = unsigned(std::max<int64_t>(1, std::min<int64_t>(want, std::max(1, 148 * 16 / ns))));
    const dim3 grid(gx, unsigned(ns));
    if (to_disk)
      st_filter_kernel<<<grid, 256, 0, stream>>>(static_cast<const uint4*>(in), static_cast<uint4*>(out), segs_dev,
                                                 s0, turn, filter);
    else
      st_unfilter_kernel<<<grid, 256, 0, stream>>>(static_cast<const uint4*>(in), static_cast<uint4*>(out), segs_dev,
                                                   s0, turn, filter);
    PG_CUDA(cudaGetLastError());
  }
  return PG_OK;
}

// --------------------------------------------------------------------------
// Compression (compress.cc:34-95): zlib below level 20, xz preset level - 20
// above.  liblzma is loaded on first use; the declarations below are the
// entry points of its public API that this file calls.

struct lzma_entry_points {
  size_t (*bound)(size_t);
  int (*encode)(uint32_t preset, int check, const void* allocator, const uint8_t* in, size_t in_size, uint8_t* out,
                size_t* out_pos, size_t out_size);
  int (*decode)(uint64_t* memlimit, uint32_t flags, const void* allocator, const uint8_t* in, size_t* in_pos,
                size_t in_size, uint8_t* out, size_t* out_pos, size_t out_size);
};
constexpr int kLzmaOk = 0;
constexpr int kLzmaCheckCrc64 = 4;
constexpr uint32_t kLzmaTellNoCheck = 1, kLzmaTellUnsupportedCheck = 2;

const lzma_entry_points* lzma(std::string& err) {
  static std::once_flag once;
  static lzma_entry_points L;
  static bool ok = false;
  std::call_once(once, [] {
    void* h = dlopen("liblzma.so.5", RTLD_NOW | RTLD_LOCAL);
    if (!h) return;
    L.bound = reinterpret_cast<size_t (*)(size_t)>(dlsym(h, "lzma_stream_buffer_bound"));
    L.encode = reinterpret_cast<decltype(L.encode)>(dlsym(h, "lzma_easy_buffer_encode"));
    L.decode = reinterpret_cast<decltype(L.decode)>(dlsym(h, "lzma_stream_buffer_decode"));
    ok = L.bound && L.encode && L.decode;
  });
  if (!ok) {
    err = "xz data needs liblzma.so.5, which could not be loaded";
    return nullptr;
  }
  return &L;
}

bool level_ok(int level) { return (1 <= level && level <= 9) || (20 <= level && level <= 29); }

bool compress_bytes(const uint8_t* in, size_t n, int level, std::vector<uint8_t>& out, std::string& err) {
  if (level < 20) {
    uLongf dest = compressBound(uLong(n));
    out.resize(dest);
    if (compress2(out.data(), &dest, in, uLong(n), level) != Z_OK) {
      err = "zlib compression failed";
      return false;
    }
    out.resize(dest);
    return true;
  }
  const lzma_entry_points* L = lzma(err);
  if (!L) return false;
  size_t cap = L->bound(n), pos = 0;
  out.resize(cap);
  if (L->encode(uint32_t(level - 20), kLzmaCheckCrc64, nullptr, in, n, out.data(), &pos, cap) != kLzmaOk) {
    err = "xz compression failed";
    return false;
  }
  out.resize(pos);
  return true;
}

bool is_xz(const uint8_t* p, size_t n) {
  static const uint8_t magic[6] = {0xfd, '7', 'z', 'X', 'Z', 0};
  return n >= 6 && !memcmp(p, magic, 6);
}

bool decompress_bytes(const uint8_t* in, size_t n, uint8_t* out, size_t expect, std::string& err) {
  if (!is_xz(in, n)) {
    uLongf dest = uLongf(expect);
    if (uncompress(out, &dest, in, uLong(n)) != Z_OK) {
      err = "zlib data is corrupt or does not fit its index size";
      return false;
    }
    if (dest != expect) {
      err = "decompressed size differs from the index";
      return false;
    }
    return true;
  }
  const lzma_entry_points* L = lzma(err);
  if (!L) return false;
  uint64_t memlimit = UINT64_MAX;
  size_t ip = 0, op = 0;
  if (L->decode(&memlimit, kLzmaTellNoCheck | kLzmaTellUnsupportedCheck, nullptr, in, &ip, n, out, &op, expect) !=
      kLzmaOk) {
    err = "xz data is corrupt or does not fit its index size";
    return false;
  }
  if (op != expect) {
    err = "decompressed size differs from the index";
    return false;
  }
  return true;
}

// --------------------------------------------------------------------------
// Host helpers.

// f(i) for i in [0, n) on up to `threads` threads (0: every core); the error
// of the lowest failing i is kept.
template<class F> bool parallel_for(int n, int threads, std::string& err, const F& f) {
  if (n <= 0) return true;
  int t = threads > 0 ? threads : int(std::thread::hardware_concurrency());
  t = std::max(1, std::min(t, n));
  std::atomic<int> next{0};
  std::mutex m;
  int bad = n;
  auto work = [&] {
    std::string e;
    for (int i; (i = next.fetch_add(1)) < n;) {
      if (!f(i, e)) {
        std::lock_guard<std::mutex> g(m);
        if (i < bad) { bad = i; err = e; }
      }
    }
  };
  std::vector<std::thread> pool;
  for (int k = 1; k < t; k++) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
  return bad == n;
}

bool pread_all(int fd, void* buf, size_t n, uint64_t off) {
  uint8_t* p = static_cast<uint8_t*>(buf);
  while (n) {
    const ssize_t r = pread(fd, p, n, off_t(off));
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) return false;
    p += r; n -= size_t(r); off += uint64_t(r);
  }
  return true;
}

bool pwrite_all(int fd, const void* buf, size_t n, uint64_t off) {
  const uint8_t* p = static_cast<const uint8_t*>(buf);
  while (n) {
    const ssize_t r = pwrite(fd, p, n, off_t(off));
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) return false;
    p += r; n -= size_t(r); off += uint64_t(r);
  }
  return true;
}

void pack_header(const pg_supertensor_header_t& h, uint8_t* out) {
  uint8_t* p = out;
  auto put = [&](const void* v, size_t n) { memcpy(p, v, n); p += n; };
  const uint8_t valid = h.valid ? 1 : 0;
  put(kSingleMagic, 20);
  put(&h.version, 4);
  put(&valid, 1);
  put(&h.stones, 4);
  put(&h.section, 8);
  put(h.shape, 8);
  put(&h.block_size, 4);
  put(h.blocks, 8);
  put(&h.filter, 4);
  put(h.index, 24);
}

bool unpack_header(const uint8_t* in, pg_supertensor_header_t& h) {
  memset(&h, 0, sizeof h);
  if (memcmp(in, kSingleMagic, 20)) return false;
  const uint8_t* p = in + 20;
  auto get = [&](void* v, size_t n) { memcpy(v, p, n); p += n; };
  uint8_t valid;
  get(&h.version, 4);
  get(&valid, 1);
  get(&h.stones, 4);
  get(&h.section, 8);
  get(h.shape, 8);
  get(&h.block_size, 4);
  get(h.blocks, 8);
  get(&h.filter, 4);
  get(h.index, 24);
  h.valid = valid;
  return true;
}

// Quadrant counts within the board (each color and their sum at most 9).
bool counts_ok(const section_t& s) {
  for (int q = 0; q < 4; q++)
    if (s.c[q][0] > 9 || s.c[q][1] > 9 || s.c[q][0] + s.c[q][1] > 9) return false;
  return true;
}

// The header a writer starts from (supertensor_header_t(section, block_size,
// filter), supertensor.cc:252-264).
pg_supertensor_header_t new_header(const section_t& s, int block_size, int filter) {
  pg_supertensor_header_t h;
  memset(&h, 0, sizeof h);
  h.version = 3;
  h.stones = uint32_t(s.sum());
  h.section = s.sig();
  int shape[4];
  s.shape(shape);
  h.block_size = uint32_t(block_size);
  for (int i = 0; i < 4; i++) {
    h.shape[i] = uint16_t(shape[i]);
    h.blocks[i] = uint16_t((shape[i] + block_size - 1) / block_size);
  }
  h.filter = uint32_t(filter);
  return h;
}

// The reader's consistency checks (supertensor.cc:156-172).
bool header_ok(const pg_supertensor_header_t& h, std::string& err) {
  if (h.version != 2 && h.version != 3) { err = "unknown supertensor version"; return false; }
  if (!h.valid) { err = "supertensor section is marked invalid"; return false; }
  const section_t s = section_t::from_sig(h.section);
  if (!counts_ok(s) || int(h.stones) != s.sum()) { err = "inconsistent section in supertensor header"; return false; }
  if (h.block_size < 1 || h.block_size > 27 || (h.block_size & 1)) { err = "bad supertensor block size"; return false; }
  if (h.filter > 1) { err = "unknown supertensor filter"; return false; }
  int shape[4];
  s.shape(shape);
  for (int i = 0; i < 4; i++) {
    if (h.shape[i] != shape[i]) { err = "supertensor shape does not match its section"; return false; }
    if (h.blocks[i] != (shape[i] + h.block_size - 1) / h.block_size) { err = "bad supertensor block counts"; return false; }
  }
  return true;
}

int64_t block_count(const pg_supertensor_header_t& h) {
  return int64_t(h.blocks[0]) * h.blocks[1] * h.blocks[2] * h.blocks[3];
}

// Row-major index of a block, or -1 if it lies outside the block grid.
int64_t block_flat(const pg_supertensor_header_t& h, const uint8_t* b) {
  int64_t f = 0;
  for (int i = 0; i < 4; i++) {
    if (b[i] >= h.blocks[i]) return -1;
    f = f * h.blocks[i] + b[i];
  }
  return f;
}

// supertensor_header_t::block_shape (supertensor.cc:25-32): nodes of a block.
int64_t block_nodes(const pg_supertensor_header_t& h, const uint8_t* b) {
  int64_t n = 1;
  for (int i = 0; i < 4; i++)
    n *= b[i] + 1 < h.blocks[i] ? int64_t(h.block_size) : int64_t(h.shape[i]) - int64_t(h.block_size) * (h.blocks[i] - 1);
  return n;
}

struct st_section {
  pg_supertensor_header_t h;
  std::vector<blob_t> index;
};

// Pinned host buffers reused across calls on one reader or writer.
struct pinned_pair {
  uint8_t* buf[2] = {nullptr, nullptr};
  seg_t* segs[2] = {nullptr, nullptr};
  size_t bytes = 0;
  int nseg = 0;
  cudaError_t reserve(size_t b, int s) {
    if (b <= bytes && s <= nseg) return cudaSuccess;
    release();
    for (int k = 0; k < 2; k++) {
      if (cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&buf[k]), b)) return e;
      if (cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&segs[k]), sizeof(seg_t) * s)) return e;
    }
    bytes = b;
    nseg = s;
    return cudaSuccess;
  }
  void release() {
    for (int k = 0; k < 2; k++) {
      if (buf[k]) cudaFreeHost(buf[k]);
      if (segs[k]) cudaFreeHost(segs[k]);
      buf[k] = nullptr;
      segs[k] = nullptr;
    }
    bytes = 0;
    nseg = 0;
  }
};

// A list of blocks split into consecutive batches of at most kBatchBytes
// on-disk bytes (a larger block is a batch of its own).
struct batch_plan {
  std::vector<int> start;      // batch b = items start[b] .. start[b+1]
  std::vector<int64_t> nodes;  // per item
  size_t max_bytes = 0;
  int max_items = 0;
  int64_t max_nodes = 0;
};

batch_plan plan_batches(const std::vector<int64_t>& nodes) {
  batch_plan P;
  P.nodes = nodes;
  size_t cur = 0;
  const int n = int(nodes.size());
  for (int i = 0; i < n; i++) {
    const size_t b = size_t(64) * size_t(nodes[i]);
    if (i == 0 || cur + b > kBatchBytes) {
      P.start.push_back(i);
      cur = 0;
    }
    cur += b;
    P.max_bytes = std::max(P.max_bytes, cur);
    P.max_nodes = std::max(P.max_nodes, nodes[i]);
  }
  P.start.push_back(n);
  for (size_t b = 0; b + 1 < P.start.size(); b++) P.max_items = std::max(P.max_items, P.start[b + 1] - P.start[b]);
  return P;
}

}  // namespace
}  // namespace pg

using namespace pg;

struct pg_supertensor_reader_s {
  int fd = -1;
  std::string path;
  std::vector<st_section> secs;
  pinned_pair pinned;
};

struct pg_supertensor_writer_s {
  int fd = -1;
  std::string path;
  bool multiple = false;
  int level = 6;
  std::vector<st_section> secs;
  std::vector<std::vector<uint8_t>> written;  // per section and block: 1 once written
  std::vector<bool> finalized;
  uint64_t next_offset = 0;
  std::mutex lock;
  pinned_pair pinned;
};

namespace {

bool ends_with_pentago(const char* path) {
  const size_t n = strlen(path);
  return n >= 8 && !strcmp(path + n - 8, ".pentago");
}

// Validate a block list against a set of sections: node counts per item.
int check_blocks(const std::vector<st_section>& secs, int n, const int32_t* sections, const uint8_t* blocks,
                 std::vector<int64_t>& nodes, std::vector<int64_t>* flat) {
  if (n < 0 || (n && (!sections || !blocks))) return fail(PG_ERR_ARG, "bad block list");
  nodes.resize(n);
  if (flat) flat->resize(n);
  for (int i = 0; i < n; i++) {
    if (sections[i] < 0 || sections[i] >= int(secs.size())) return fail(PG_ERR_ARG, "section index out of range");
    const auto& h = secs[sections[i]].h;
    const int64_t f = block_flat(h, blocks + 4 * i);
    if (f < 0) return fail(PG_ERR_ARG, "block outside the section's block grid");
    nodes[i] = block_nodes(h, blocks + 4 * i);
    if (flat) (*flat)[i] = f;
  }
  return PG_OK;
}

int read_section(pg_supertensor_reader_s& R, uint64_t header_offset) {
  uint8_t buf[kHeaderBytes];
  if (!pread_all(R.fd, buf, kHeaderBytes, header_offset)) return fail(PG_ERR_IO, "error reading supertensor header");
  st_section S;
  if (!unpack_header(buf, S.h)) return fail(PG_ERR_FORMAT, "invalid supertensor file: incorrect magic string");
  std::string err;
  if (!header_ok(S.h, err)) return fail(PG_ERR_FORMAT, err);
  const int64_t nb = block_count(S.h);
  const blob_t ib = {S.h.index[0], S.h.index[1], S.h.index[2]};
  if (ib.uncompressed != uint64_t(24 * nb) || ib.compressed >= (uint64_t(1) << 31) || !ib.offset)
    return fail(PG_ERR_FORMAT, "bad supertensor block index blob");
  std::vector<uint8_t> comp(ib.compressed);
  if (!pread_all(R.fd, comp.data(), comp.size(), ib.offset)) return fail(PG_ERR_IO, "error reading block index");
  S.index.resize(nb);
  if (!decompress_bytes(comp.data(), comp.size(), reinterpret_cast<uint8_t*>(S.index.data()), 24 * size_t(nb), err))
    return fail(PG_ERR_FORMAT, "block index: " + err);
  for (int64_t f = 0; f < nb; f++) {
    uint8_t b[4];
    int64_t r = f;
    for (int i = 3; i >= 0; i--) { b[i] = uint8_t(r % S.h.blocks[i]); r /= S.h.blocks[i]; }
    const blob_t& x = S.index[f];
    if (x.uncompressed != uint64_t(64 * block_nodes(S.h, b)) || x.compressed >= (uint64_t(1) << 31) || !x.offset)
      return fail(PG_ERR_FORMAT, "supertensor block index entry does not match the block's shape");
  }
  R.secs.push_back(std::move(S));
  return PG_OK;
}

// Decompress items [i0, i1) of a block list into dst + dst_off[i - i0].
bool read_items(pg_supertensor_reader_s& R, const int32_t* sections, const std::vector<int64_t>& flat, int i0, int i1,
                uint8_t* dst, const int64_t* dst_off, int threads, std::string& err) {
  return parallel_for(i1 - i0, threads, err, [&](int k, std::string& e) {
    const int i = i0 + k;
    const blob_t& b = R.secs[sections[i]].index[flat[i]];
    std::vector<uint8_t> comp(b.compressed);
    if (!pread_all(R.fd, comp.data(), comp.size(), b.offset)) { e = "error reading a supertensor block"; return false; }
    if (!decompress_bytes(comp.data(), comp.size(), dst + dst_off[k], b.uncompressed, e)) return false;
    return true;
  });
}

// Compress items [0, n) and place them at the end of the file in list order.
int write_items(pg_supertensor_writer_s& W, int n, const int32_t* sections, const std::vector<int64_t>& flat,
                const std::vector<int64_t>& nodes, const uint8_t* const* src, int threads) {
  std::vector<std::vector<uint8_t>> comp(n);
  std::string err;
  if (!parallel_for(n, threads, err, [&](int i, std::string& e) {
        return compress_bytes(src[i], size_t(64) * size_t(nodes[i]), W.level, comp[i], e);
      }))
    return fail(PG_ERR_IO, err);
  std::vector<uint64_t> off(n);
  {
    std::lock_guard<std::mutex> g(W.lock);
    for (int i = 0; i < n; i++) {
      off[i] = W.next_offset;
      W.next_offset += comp[i].size();
      W.secs[sections[i]].index[flat[i]] = {uint64_t(64 * nodes[i]), uint64_t(comp[i].size()), off[i]};
    }
  }
  if (!parallel_for(n, threads, err, [&](int i, std::string& e) {
        if (!pwrite_all(W.fd, comp[i].data(), comp[i].size(), off[i])) { e = "error writing a supertensor block"; return false; }
        return true;
      }))
    return fail(PG_ERR_IO, err);
  return PG_OK;
}

// Mark a block list as written, refusing blocks written before or twice in the list.
int claim_blocks(pg_supertensor_writer_s& W, int n, const int32_t* sections, const std::vector<int64_t>& flat) {
  std::lock_guard<std::mutex> g(W.lock);
  for (int i = 0; i < n; i++)
    if (W.finalized[sections[i]]) return fail(PG_ERR_ARG, "section already finalized");
  for (int i = 0; i < n; i++) {
    uint8_t& w = W.written[sections[i]][flat[i]];
    if (w) {
      for (int k = 0; k < i; k++) W.written[sections[k]][flat[k]] = 0;
      return fail(PG_ERR_ARG, "supertensor block written twice");
    }
    w = 1;
  }
  return PG_OK;
}

void unclaim_blocks(pg_supertensor_writer_s& W, int n, const int32_t* sections, const std::vector<int64_t>& flat) {
  std::lock_guard<std::mutex> g(W.lock);
  for (int i = 0; i < n; i++) W.written[sections[i]][flat[i]] = 0;
}

}  // namespace

extern "C" int pg_supertensor_header_pack(const pg_supertensor_header_t* h, uint8_t* out85) {
  if (!h || !out85) return fail(PG_ERR_ARG, "null argument");
  pack_header(*h, out85);
  return PG_OK;
}

extern "C" int pg_supertensor_header_unpack(const uint8_t* in85, pg_supertensor_header_t* h) {
  if (!in85 || !h) return fail(PG_ERR_ARG, "null argument");
  if (!unpack_header(in85, *h)) return fail(PG_ERR_FORMAT, "incorrect supertensor magic string");
  return PG_OK;
}

static int filter_call(bool to_disk, const void* in, void* out, int64_t n, int turn, int filter, void* stream_) {
  if (n < 0 || (n && (!in || !out)) || turn < 0 || turn > PG_ST_RAW || filter < 0 || filter > 1)
    return fail(PG_ERR_ARG, "bad filter arguments");
  if (!n) return PG_OK;
  if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15)
    return fail(PG_ERR_ARG, "node buffers must be 16-byte aligned");
  cudaStream_t stream = (cudaStream_t)stream_;
  stream_scratch scratch(stream);
  seg_t* segs = nullptr;
  PG_CUDA(scratch.alloc(&segs, sizeof(seg_t)));
  const seg_t s = {0, 0, n};
  PG_CUDA(cudaMemcpyAsync(segs, &s, sizeof s, cudaMemcpyHostToDevice, stream));
  // (cudaMemcpyAsync has taken the pageable record `s` before it returns)
  return launch_segments(to_disk, in, out, segs, 1, n, turn, filter, stream);
}

extern "C" int pg_supertensor_filter(const uint64_t* nodes, int64_t n, int turn, int filter, uint8_t* out,
                                     void* stream) {
  return filter_call(true, nodes, out, n, turn, filter, stream);
}

extern "C" int pg_supertensor_unfilter(const uint8_t* in, int64_t n, int turn, int filter, uint64_t* nodes,
                                       void* stream) {
  return filter_call(false, in, nodes, n, turn, filter, stream);
}

extern "C" int pg_supertensor_open(const char* path, pg_supertensor_reader_t* out) {
  if (!path || !out) return fail(PG_ERR_ARG, "null argument");
  *out = nullptr;
  if (!ends_with_pentago(path)) return fail(PG_ERR_ARG, "supertensor files end in .pentago");
  auto* R = new pg_supertensor_reader_s;
  R->path = path;
  R->fd = open(path, O_RDONLY | O_CLOEXEC);
  if (R->fd < 0) {
    delete R;
    return fail(PG_ERR_IO, std::string("cannot open ") + path + ": " + strerror(errno));
  }
  uint8_t magic[20];
  int rc = PG_OK;
  if (!pread_all(R->fd, magic, 20, 0)) rc = fail(PG_ERR_IO, "error reading supertensor magic string");
  else if (!memcmp(magic, kSingleMagic, 20)) rc = read_section(*R, 0);
  else if (!memcmp(magic, kMultipleMagic, 20)) {
    uint32_t pre[3];
    if (!pread_all(R->fd, pre, sizeof pre, 20)) rc = fail(PG_ERR_IO, "error reading supertensor sections header");
    else if (pre[0] != 3) rc = fail(PG_ERR_FORMAT, "multiple supertensor file has an unknown version");
    else if (pre[1] >= kMaxSections) rc = fail(PG_ERR_FORMAT, "multiple supertensor file has a weird section count");
    // headers follow the pre-header at its stated stride (supertensor.cc:430-432)
    for (uint32_t s = 0; rc == PG_OK && s < pre[1]; s++) rc = read_section(*R, kPreheaderBytes + uint64_t(pre[2]) * s);
  } else
    rc = fail(PG_ERR_FORMAT, "invalid supertensor file: bad magic string");
  if (rc != PG_OK) {
    close(R->fd);
    delete R;
    return rc;
  }
  *out = R;
  return int(R->secs.size());
}

extern "C" int pg_supertensor_header(pg_supertensor_reader_t R, int section, pg_supertensor_header_t* h) {
  if (!R || !h || section < 0 || section >= int(R->secs.size())) return fail(PG_ERR_ARG, "bad header arguments");
  *h = R->secs[section].h;
  return PG_OK;
}

extern "C" int pg_supertensor_block_blob(pg_supertensor_reader_t R, int section, const uint8_t* block4,
                                         uint64_t* blob3) {
  if (!R || !block4 || !blob3 || section < 0 || section >= int(R->secs.size()))
    return fail(PG_ERR_ARG, "bad blob arguments");
  const int64_t f = block_flat(R->secs[section].h, block4);
  if (f < 0) return fail(PG_ERR_ARG, "block outside the section's block grid");
  const blob_t& b = R->secs[section].index[f];
  blob3[0] = b.uncompressed;
  blob3[1] = b.compressed;
  blob3[2] = b.offset;
  return PG_OK;
}

extern "C" int pg_supertensor_read_blocks_host(pg_supertensor_reader_t R, int n, const int32_t* sections,
                                               const uint8_t* blocks, uint8_t* out, const int64_t* out_offsets,
                                               int threads) {
  if (!R) return fail(PG_ERR_ARG, "null reader");
  std::vector<int64_t> nodes, flat;
  if (int rc = check_blocks(R->secs, n, sections, blocks, nodes, &flat)) return rc;
  if (n && (!out || !out_offsets)) return fail(PG_ERR_ARG, "null output");
  std::string err;
  if (!read_items(*R, sections, flat, 0, n, out, out_offsets, threads, err)) return fail(PG_ERR_FORMAT, err);
  return PG_OK;
}

extern "C" int pg_supertensor_read_blocks(pg_supertensor_reader_t R, int n, const int32_t* sections,
                                          const uint8_t* blocks, uint64_t* nodes_dev, const int64_t* node_offsets,
                                          int turn, int threads, void* stream_) {
  if (!R) return fail(PG_ERR_ARG, "null reader");
  if (turn < 0 || turn > PG_ST_RAW) return fail(PG_ERR_ARG, "bad turn");
  std::vector<int64_t> nodes, flat;
  if (int rc = check_blocks(R->secs, n, sections, blocks, nodes, &flat)) return rc;
  if (!n) return PG_OK;
  if (!nodes_dev || !node_offsets || (reinterpret_cast<uintptr_t>(nodes_dev) & 15))
    return fail(PG_ERR_ARG, "bad node output");
  for (int i = 0; i < n; i++)
    if (R->secs[sections[i]].h.filter != R->secs[sections[0]].h.filter)
      return fail(PG_ERR_ARG, "blocks of one call must share a filter");
  const int filter = int(R->secs[sections[0]].h.filter);
  cudaStream_t stream = (cudaStream_t)stream_;
  const batch_plan P = plan_batches(nodes);
  const int nb = int(P.start.size()) - 1;
  PG_CUDA(R->pinned.reserve(P.max_bytes, P.max_items));
  stream_scratch scratch(stream);
  uint8_t* stage[2];
  seg_t* segs[2];
  for (int k = 0; k < 2; k++) {
    PG_CUDA(scratch.alloc(&stage[k], P.max_bytes));
    PG_CUDA(scratch.alloc(&segs[k], sizeof(seg_t) * P.max_items));
  }
  cudaEvent_t ev[2];
  PG_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
  if (cudaError_t e = cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming)) {
    cudaEventDestroy(ev[0]);
    return cuda_fail(e, "cudaEventCreateWithFlags");
  }
  int rc = PG_OK;
  bool pending[2] = {false, false};
  std::vector<int64_t> off;
  for (int b = 0; b < nb && rc == PG_OK; b++) {
    const int k = b & 1, i0 = P.start[b], i1 = P.start[b + 1];
    // the pinned buffer of batch b - 2 is free once its copy to the device ended
    if (pending[k] && cudaEventSynchronize(ev[k]) != cudaSuccess) { rc = fail(PG_ERR_CUDA, "batch copy failed"); break; }
    pending[k] = false;
    off.assign(i1 - i0, 0);
    int64_t at = 0;
    for (int i = i0; i < i1; i++) {
      off[i - i0] = 64 * at;
      R->pinned.segs[k][i - i0] = {at, node_offsets[i], nodes[i]};
      at += nodes[i];
    }
    std::string err;
    if (!read_items(*R, sections, flat, i0, i1, R->pinned.buf[k], off.data(), threads, err)) {
      rc = fail(PG_ERR_FORMAT, err);
      break;
    }
    if (cudaMemcpyAsync(stage[k], R->pinned.buf[k], size_t(64) * at, cudaMemcpyHostToDevice, stream) ||
        cudaMemcpyAsync(segs[k], R->pinned.segs[k], sizeof(seg_t) * (i1 - i0), cudaMemcpyHostToDevice, stream) ||
        cudaEventRecord(ev[k], stream)) {
      rc = fail(PG_ERR_CUDA, "batch copy to the device failed");
      break;
    }
    pending[k] = true;
    rc = launch_segments(false, stage[k], nodes_dev, segs[k], i1 - i0, P.max_nodes, turn, filter, stream);
  }
  // the pinned buffers must not be reused or freed while a copy still reads them
  for (int k = 0; k < 2; k++) {
    if (pending[k] && cudaEventSynchronize(ev[k]) != cudaSuccess && rc == PG_OK) rc = fail(PG_ERR_CUDA, "batch copy failed");
    cudaEventDestroy(ev[k]);
  }
  return rc;
}

extern "C" int pg_supertensor_close(pg_supertensor_reader_t R) {
  if (!R) return PG_OK;
  if (R->fd >= 0) close(R->fd);
  R->pinned.release();
  delete R;
  return PG_OK;
}

extern "C" int pg_supertensor_create(const char* path, const uint64_t* sections, int n, int multiple, int block_size,
                                     int filter, int level, pg_supertensor_writer_t* out) {
  if (!path || !out || !sections || n < 1) return fail(PG_ERR_ARG, "bad create arguments");
  *out = nullptr;
  if (!ends_with_pentago(path)) return fail(PG_ERR_ARG, "supertensor files end in .pentago");
  if (!multiple && n != 1) return fail(PG_ERR_ARG, "a single supertensor file holds one section");
  if (uint32_t(n) >= kMaxSections) return fail(PG_ERR_ARG, "too many sections");
  if (block_size < 2 || block_size > 26 || (block_size & 1))
    return fail(PG_ERR_ARG, "supertensor block size must be even, 2..26 (block-wise reflection)");
  if (filter < 0 || filter > 1) return fail(PG_ERR_ARG, "unknown supertensor filter");
  if (!level_ok(level)) return fail(PG_ERR_ARG, "compression level must be 1..9 (zlib) or 20..29 (xz)");
  auto* W = new pg_supertensor_writer_s;
  W->path = path;
  W->multiple = multiple != 0;
  W->level = level;
  for (int s = 0; s < n; s++) {
    const section_t sec = section_t::from_sig(sections[s]);
    if (!counts_ok(sec)) {
      delete W;
      return fail(PG_ERR_ARG, "invalid section");
    }
    st_section S;
    S.h = new_header(sec, block_size, filter);
    S.index.assign(block_count(S.h), blob_t{0, 0, 0});
    W->written.emplace_back(block_count(S.h), 0);
    W->secs.push_back(std::move(S));
  }
  W->finalized.assign(n, false);
  W->fd = open(path, O_WRONLY | O_CREAT | O_TRUNC | O_CLOEXEC, 0644);
  if (W->fd < 0) {
    delete W;
    return fail(PG_ERR_IO, std::string("cannot create ") + path + ": " + strerror(errno));
  }
  if (W->multiple) {
    // the pre-header of supertensor_writers (supertensor.cc:437-462); each
    // section's header follows at finalize
    uint8_t pre[kPreheaderBytes];
    memcpy(pre, kMultipleMagic, 20);
    const uint32_t v[3] = {3, uint32_t(n), uint32_t(kHeaderBytes)};
    memcpy(pre + 20, v, 12);
    if (!pwrite_all(W->fd, pre, kPreheaderBytes, 0)) {
      close(W->fd);
      unlink(path);
      delete W;
      return fail(PG_ERR_IO, "error writing the supertensor pre-header");
    }
    W->next_offset = kPreheaderBytes + uint64_t(kHeaderBytes) * n;
  } else
    W->next_offset = kHeaderBytes;
  *out = W;
  return PG_OK;
}

extern "C" int pg_supertensor_write_blocks_host(pg_supertensor_writer_t W, int n, const int32_t* sections,
                                                const uint8_t* blocks, const uint8_t* data,
                                                const int64_t* data_offsets, int threads) {
  if (!W) return fail(PG_ERR_ARG, "null writer");
  std::vector<int64_t> nodes, flat;
  if (int rc = check_blocks(W->secs, n, sections, blocks, nodes, &flat)) return rc;
  if (!n) return PG_OK;
  if (!data || !data_offsets) return fail(PG_ERR_ARG, "null data");
  if (int rc = claim_blocks(*W, n, sections, flat)) return rc;
  std::vector<const uint8_t*> src(n);
  for (int i = 0; i < n; i++) src[i] = data + data_offsets[i];
  const int rc = write_items(*W, n, sections, flat, nodes, src.data(), threads);
  if (rc != PG_OK) unclaim_blocks(*W, n, sections, flat);
  return rc;
}

extern "C" int pg_supertensor_write_blocks(pg_supertensor_writer_t W, int n, const int32_t* sections,
                                           const uint8_t* blocks, const uint64_t* nodes_dev,
                                           const int64_t* node_offsets, int turn, int threads, void* stream_) {
  if (!W) return fail(PG_ERR_ARG, "null writer");
  if (turn < 0 || turn > PG_ST_RAW) return fail(PG_ERR_ARG, "bad turn");
  std::vector<int64_t> nodes, flat;
  if (int rc = check_blocks(W->secs, n, sections, blocks, nodes, &flat)) return rc;
  if (!n) return PG_OK;
  if (!nodes_dev || !node_offsets || (reinterpret_cast<uintptr_t>(nodes_dev) & 15))
    return fail(PG_ERR_ARG, "bad node input");
  for (int i = 0; i < n; i++)
    if (W->secs[sections[i]].h.filter != W->secs[sections[0]].h.filter)
      return fail(PG_ERR_ARG, "blocks of one call must share a filter");
  const int filter = int(W->secs[sections[0]].h.filter);
  if (int rc = claim_blocks(*W, n, sections, flat)) return rc;
  cudaStream_t stream = (cudaStream_t)stream_;
  const batch_plan P = plan_batches(nodes);
  const int nb = int(P.start.size()) - 1;
  int rc = PG_OK;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool pending[2] = {false, false};
  {
    stream_scratch scratch(stream);
    uint8_t* stage[2] = {nullptr, nullptr};
    seg_t* segs[2] = {nullptr, nullptr};
    if (cudaError_t e = W->pinned.reserve(P.max_bytes, P.max_items)) rc = cuda_fail(e, "cudaMallocHost");
    for (int k = 0; k < 2 && rc == PG_OK; k++) {
      if (cudaError_t e = scratch.alloc(&stage[k], P.max_bytes)) rc = cuda_fail(e, "cudaMallocAsync");
      else if (cudaError_t e2 = scratch.alloc(&segs[k], sizeof(seg_t) * P.max_items)) rc = cuda_fail(e2, "cudaMallocAsync");
      else if (cudaError_t e3 = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming)) rc = cuda_fail(e3, "cudaEventCreate");
    }
    std::vector<const uint8_t*> src;
    // iteration b issues batch b on the GPU and compresses batch b - 1 on the host
    for (int b = 0; b <= nb && rc == PG_OK; b++) {
      if (b < nb) {
        const int k = b & 1, i0 = P.start[b], i1 = P.start[b + 1];
        int64_t at = 0;
        for (int i = i0; i < i1; i++) {
          W->pinned.segs[k][i - i0] = {node_offsets[i], at, nodes[i]};
          at += nodes[i];
        }
        if (cudaMemcpyAsync(segs[k], W->pinned.segs[k], sizeof(seg_t) * (i1 - i0), cudaMemcpyHostToDevice, stream)) {
          rc = fail(PG_ERR_CUDA, "segment copy failed");
          break;
        }
        if ((rc = launch_segments(true, nodes_dev, stage[k], segs[k], i1 - i0, P.max_nodes, turn, filter, stream))) break;
        if (cudaMemcpyAsync(W->pinned.buf[k], stage[k], size_t(64) * at, cudaMemcpyDeviceToHost, stream) ||
            cudaEventRecord(ev[k], stream)) {
          rc = fail(PG_ERR_CUDA, "batch copy to the host failed");
          break;
        }
        pending[k] = true;
      }
      if (b >= 1) {
        const int k = (b - 1) & 1, i0 = P.start[b - 1], i1 = P.start[b];
        if (cudaEventSynchronize(ev[k]) != cudaSuccess) { rc = fail(PG_ERR_CUDA, "batch copy failed"); break; }
        pending[k] = false;
        src.resize(i1 - i0);
        int64_t at = 0;
        for (int i = i0; i < i1; i++) {
          src[i - i0] = W->pinned.buf[k] + 64 * at;
          at += nodes[i];
        }
        std::vector<int64_t> fl(flat.begin() + i0, flat.begin() + i1), nd(nodes.begin() + i0, nodes.begin() + i1);
        rc = write_items(*W, i1 - i0, sections + i0, fl, nd, src.data(), threads);
      }
    }
    for (int k = 0; k < 2; k++) {
      if (pending[k]) cudaEventSynchronize(ev[k]);
      if (ev[k]) cudaEventDestroy(ev[k]);
    }
  }
  if (rc != PG_OK) unclaim_blocks(*W, n, sections, flat);
  return rc;
}

extern "C" int pg_supertensor_finalize(pg_supertensor_writer_t W, int section) {
  if (!W || section < -1 || section >= int(W->secs.size())) return fail(PG_ERR_ARG, "bad finalize arguments");
  const int s0 = section < 0 ? 0 : section, s1 = section < 0 ? int(W->secs.size()) : section + 1;
  for (int s = s0; s < s1; s++) {
    if (W->finalized[s]) continue;
    st_section& S = W->secs[s];
    for (uint8_t w : W->written[s])
      if (!w) return fail(PG_ERR_ARG, "can't finalize an incomplete supertensor file");
    // the block index, compressed, at the end of the file (supertensor.cc:315-339)
    std::vector<uint8_t> comp;
    std::string err;
    const size_t ib = sizeof(blob_t) * S.index.size();
    if (!compress_bytes(reinterpret_cast<const uint8_t*>(S.index.data()), ib, W->level, comp, err)) return fail(PG_ERR_IO, err);
    uint64_t off;
    {
      std::lock_guard<std::mutex> g(W->lock);
      off = W->next_offset;
      W->next_offset += comp.size();
    }
    if (!pwrite_all(W->fd, comp.data(), comp.size(), off)) return fail(PG_ERR_IO, "error writing a block index");
    pg_supertensor_header_t h = S.h;
    h.index[0] = ib;
    h.index[1] = comp.size();
    h.index[2] = off;
    h.valid = 1;
    uint8_t buf[kHeaderBytes];
    pack_header(h, buf);
    const uint64_t at = W->multiple ? kPreheaderBytes + uint64_t(kHeaderBytes) * s : 0;
    if (!pwrite_all(W->fd, buf, kHeaderBytes, at)) return fail(PG_ERR_IO, "error writing a supertensor header");
    S.h = h;
    W->finalized[s] = true;
  }
  return PG_OK;
}

extern "C" int pg_supertensor_writer_close(pg_supertensor_writer_t W) {
  if (!W) return PG_OK;
  bool done = true;
  for (bool f : W->finalized) done = done && f;
  if (W->fd >= 0) close(W->fd);
  if (!done) unlink(W->path.c_str());
  W->pinned.release();
  delete W;
  return PG_OK;
}
