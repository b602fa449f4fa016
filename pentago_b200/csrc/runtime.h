// Per-device state of the library: uploaded tables and error reporting.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

namespace pg {

// Device copies of the lookup tables (global memory, read through __ldg).
struct dev_tables_t {
  const uint16_t* rmin_flat;   // 19683 entries
  const uint16_t* rmin_inv;    // 19683
  const uint16_t* unpack;      // 19683 x 2
  const uint32_t* win_factors; // 4 x 512 x 16
  const uint16_t* rmin_off;    // 56
  const uint8_t* commute;      // 8 x 256
  const uint32_t* win_union;   // 4 x 19683 x 16
  const uint16_t* pack;        // 512
  const uint16_t* pop_masks;   // 512, grouped by popcount
  const uint8_t* rank9;        // 512
  const uint8_t* term_pat;     // 4 x 17
  const uint8_t* term_other;   // 4 x 17 x 2
  const uint32_t* term_sub;    // 4 x 512 x 4
  const uint8_t* cov;          // 32 x 4 x 512
  const uint8_t* miss_pat;     // 4 x 15
  const uint8_t* miss_quad;    // 4 x 15 x 3
  const uint16_t* rot;         // 512 x 2: [left, right] rotation of a quadrant side
  const uint16_t* refl;        // 512: reflection of a quadrant side about x = y
  const uint16_t* cls_masks;   // 512: rotation-class representatives, grouped by stone count
};

// Tables on the current device (uploaded on first use).  Returns nullptr and
// sets the error on failure.
const dev_tables_t* device_tables();

// The same tables as host pointers, for the host self-tests that run kernel
// arithmetic on the CPU.
dev_tables_t host_tables_view();

// Run f() once per (current device, key) and return its result from then on
// (thread safe).  For per-device set-up such as kernel attributes and
// constant-memory uploads.
int per_device_once(const void* key, int (*f)());

// Device scratch of one call: allocated with cudaMallocAsync on the call's
// stream and released with cudaFreeAsync on it when the guard goes out of
// scope, on every return path.
struct stream_scratch {
  cudaStream_t stream;
  void* ptrs[8] = {};
  int n = 0;
  explicit stream_scratch(cudaStream_t s) : stream(s) {}
  stream_scratch(const stream_scratch&) = delete;
  stream_scratch& operator=(const stream_scratch&) = delete;
  template<class T> cudaError_t alloc(T** p, size_t bytes) {
    *p = nullptr;
    if (n == 8) return cudaErrorMemoryAllocation;
    const cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(p), bytes ? bytes : 16, stream);
    if (e == cudaSuccess) ptrs[n++] = *p;
    return e;
  }
  ~stream_scratch() {
    for (int i = 0; i < n; i++) cudaFreeAsync(ptrs[i], stream);
  }
};

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define PG_CUDA(call) do { const cudaError_t _e = (call); if (_e != cudaSuccess) return ::pg::cuda_fail(_e, #call); } while (0)

}  // namespace pg
