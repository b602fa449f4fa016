// The drop-ins a reference maintainer would add for the end engine's lines and
// for midsolve, compiled against the
// reference's own headers and run beside the reference's functions on the
// same buffers.  Test infrastructure: built by `make -C oracle dropin` from
// this file, the reference objects oracle/Makefile already compiles, and the
// product library; run by tests/test_dropin_gpu.py on a GPU.
//
//   gpu_schedule_compute_line  replaces schedule_compute_line (pentago/end/compute.cc:394-404)
//                              for a line_details_t (end/compute.h:48-123) whose input and
//                              output buffers live on the device, in the reference's layout
//                              (input blocks at stride block_stride + PENTAGO_MPI_COMPRESS,
//                              end/compute.cc:84-94, 135-150)
//   gpu_midsolve               replaces midsolve(board, workspace) (pentago/mid/midengine.cc:161-178)
//
// Prints one line per case and "dropin: ok" when every output is bit-identical.

#include "pentago/end/compute.h"
#include "pentago/end/config.h"
#include "pentago/mid/midengine.h"
#include "pentago/high/board.h"
#include "pentago/utility/ceil_div.h"
#include "pentago/utility/thread.h"
#include "pentago_b200.h"
#include <cuda_runtime.h>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

using namespace pentago;
using namespace pentago::end;

// schedule_compute_line's drop-in: the line's own buffers, on the device.
static int gpu_schedule_compute_line(line_details_t& line, const void* input_dev, void* output_dev,
                                     cudaStream_t stream) {
  pg_line_t l;
  memset(&l, 0, sizeof l);
  l.section = line.pre.line.section.sig();
  l.dimension = line.pre.line.dimension;
  l.length = line.pre.line.length;
  for (int i = 0; i < 3; i++) l.block_base[i] = line.pre.line.block_base[i];
  l.flags = PG_LINE_STORE;
  l.input = static_cast<const uint64_t*>(input_dev);
  l.output = static_cast<uint64_t*>(output_dev);
  l.input_block_stride = line.block_stride + PENTAGO_MPI_COMPRESS;   // end/compute.cc:135-138
  l.output_block_stride = line.block_stride + PENTAGO_MPI_COMPRESS_OUTPUTS;
  return pg_end_compute_lines(&l, 1, stream);
}

// midsolve's drop-in: mid_values_t from the GPU midsolve.
static mid_values_t gpu_midsolve(const high_board_t board) {
  static pg_mid_values_t* out = nullptr;
  if (!out && cudaMallocManaged(&out, sizeof(pg_mid_values_t)) != cudaSuccess) throw std::runtime_error("alloc");
  const uint64_t raw = board.raw();
  if (pg_midsolve_batch(&raw, 1, out, nullptr, 0, nullptr) != PG_OK) throw std::runtime_error(pg_last_error());
  cudaDeviceSynchronize();
  mid_values_t results;
  for (int i = 0; i < out->size; i++) results.append(std::make_tuple(raw_t(out->entries[i].raw), int(out->entries[i].value)));
  return results;
}

static uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static section_t section_of(const int c[4][2]) {
  section_t s;
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 2; k++) s.counts[q][k] = uint8_t(c[q][k]);
  return s;
}

// One line through the reference engine and through the drop-in.
static bool check_line(const section_t section, int dim, Vector<uint8_t,3> block_base, uint64_t seed) {
  line_t line;
  line.section = section;
  line.dimension = dim;
  line.length = ceil_div(section.shape()[dim], block_size);
  line.block_base = block_base;
  const line_data_t pre(line);
  std::mutex m;
  std::condition_variable cv;
  bool done = false;
  line_details_t ref(pre, [&](line_details_t&, unit_t) {
    std::lock_guard<std::mutex> lock(m);
    done = true;
    cv.notify_all();
  });
  // Seeded children (win a subset of notlost), also in the padding slots
  uint64_t* in = (uint64_t*)ref.input.data();
  const size_t in_words = 8 * size_t(ref.input.size());
  for (size_t i = 0; i < in_words; i += 8) {
    for (int k = 0; k < 4; k++) {
      const uint64_t nl = splitmix(seed) & (splitmix(seed) | splitmix(seed));
      in[i + 4 + k] = nl;
      in[i + k] = nl & splitmix(seed);
    }
  }
  // The drop-in reads the same padded buffer, copied to the device
  void *d_in = nullptr, *d_out = nullptr;
  const size_t out_bytes = 64 * size_t(ref.output.size());
  if (cudaMalloc(&d_in, 64 * size_t(ref.input.size()) + 64) != cudaSuccess ||
      cudaMalloc(&d_out, out_bytes + 64) != cudaSuccess) {
    printf("cudaMalloc failed\n");
    return false;
  }
  cudaMemcpy(d_in, in, 64 * size_t(ref.input.size()), cudaMemcpyHostToDevice);
  cudaMemset(d_out, 0, out_bytes);
  const int rc = gpu_schedule_compute_line(ref, d_in, d_out, nullptr);
  if (pre.output_shape.product()) {
    schedule_compute_line(ref);
    std::unique_lock<std::mutex> lock(m);
    cv.wait(lock, [&] { return done; });
  }
  std::vector<uint64_t> got(out_bytes / 8);
  const cudaError_t e = cudaMemcpy(got.data(), d_out, out_bytes, cudaMemcpyDeviceToHost);
  cudaFree(d_in);
  cudaFree(d_out);
  const bool same = rc == PG_OK && e == cudaSuccess && !memcmp(got.data(), ref.output.data(), out_bytes);
  printf("line section %#llx dim %d block_base %d,%d,%d: %zu parent nodes %s%s\n",
         (unsigned long long)section.sig(), dim,
         block_base[0], block_base[1], block_base[2], size_t(ref.output.size()), same ? "identical" : "DIFFERENT",
         rc == PG_OK ? "" : pg_last_error());
  return same;
}

static bool check_midsolve(const board_t board) {
  const auto high = high_board_t::from_board(board, false);
  const auto workspace = midsolve_workspace(high.count());
  const auto want = midsolve(high, workspace);
  const auto got = gpu_midsolve(high);
  bool same = got.size() == want.size();
  for (int i = 0; same && i < int(want.size()); i++) same = got[i] == want[i];
  printf("midsolve board %llu (%d stones): %d values %s\n", (unsigned long long)board, high.count(),
         int(want.size()), same ? "identical" : "DIFFERENT");
  return same;
}

int main() {
  init_threads(default_threads(), 0);
  if (pg_init() != PG_OK) {
    printf("pg_init failed: %s\n", pg_last_error());
    return 2;
  }
  bool ok = true;
  // The 30-stone section's four lines through block (1,1,1,1): children in
  // standardized sections reached through reflections and rotations
  const int s30[4][2] = {{4, 4}, {4, 4}, {4, 3}, {3, 4}};
  for (int dim = 0; dim < 4; dim++) ok &= check_line(section_of(s30), dim, Vector<uint8_t,3>(1, 1, 1), 100 + dim);
  // A 34-stone line with a short last block and a 35-stone line (no children)
  const int s34[4][2] = {{5, 4}, {4, 5}, {4, 4}, {4, 4}};
  ok &= check_line(section_of(s34), 2, Vector<uint8_t,3>(0, 0, 1), 7);
  const int s35[4][2] = {{5, 4}, {4, 5}, {4, 4}, {5, 4}};
  ok &= check_line(section_of(s35), 2, Vector<uint8_t,3>(0, 1, 0), 8);
  // Midsolve: the reference benchmark's 18-stone board and two later ones
  for (const board_t b : {board_t(274440791932540184ull), board_t(2770041146411456919ull),
                          board_t(2770019925981538179ull)})
    ok &= check_midsolve(b);
  printf(ok ? "dropin: ok\n" : "dropin: FAILED\n");
  return ok ? 0 : 1;
}
