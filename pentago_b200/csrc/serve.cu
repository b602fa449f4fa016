// Continuous-batching midsolve server.
//
// A persistent kernel keeps three worker CTAs per SM.  Requests live in a ring in
// host-mapped memory: the host writes a planned board (mid_job_t with its
// scratch carved out of a device arena) and then publishes it by raising the
// ring's tail.  Workers claim ring entries with an atomic on a device counter,
// solve the board with the midsolve body (mid.cu), write the result records
// straight into host-mapped memory and raise the entry's done flag.  New
// requests are admitted by the host whenever the ring has a free entry and the
// arena has room for the board's scratch (its HBM budget), so work that
// arrives while others are on the GPU joins them as soon as resources free up.
//
// Idle workers poll a mirror of the ring's tail in device memory; one idle
// worker at a time (a device lock) refreshes the mirror from host memory, so
// at most one read crosses the bus while the pool waits.  (With every idle
// worker reading the host's tail itself, hundreds of reads in flight over
// the bus slowed every memory fence and host-memory load on the device by
// two orders of magnitude: a gang barrier took about 0.6 ms.)
//
// Every wait is bounded: an idle worker polls with nanosleep back-off and
// leaves after 2 s without work, by the GPU's global timer and a cap on polls
// (status kIdleExit), so a host that stops talking cannot hold the GPU; the
// host relaunches workers on the next submit.
#include "mid_body.cuh"
#include "runtime.h"
#include "../../include/pentago_b200.h"
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <vector>

namespace pg {

constexpr int kRing = 1024;
// An idle worker leaves after 2 s without work (GPU global timer), or after a
// hard cap of polls whatever the timer says; its sleep between polls grows to
// 20 us, so hundreds of idle workers do not flood the bus with mapped reads.
constexpr unsigned long long kIdleNs = 2000000000ull;
constexpr unsigned long long kIdlePollsMax = 1000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
enum : int { kRunning = 1, kIdleExit = 2, kClosed = 3, kFault = 4 };

struct serve_entry {          // host-mapped
  mid_job_t job;              // planned board; job.out points into the result area
  volatile int32_t done;      // 0 pending, 1 solved, -1 bounds failure (first entry of a request only)
  int32_t gang;               // workers solving this request together (consecutive entries)
  int32_t rank;               // this entry's worker within the gang
  int32_t first;              // ring slot of the request's first entry
};

// Device state of a request solved by a gang of workers, per ring slot of
// its first entry: barrier words, the n <= 1 results of both passes, the
// fault flag.  Zero when idle; the gang leaves it zero again.
struct gang_aux {
  unsigned count, gen;
  int fault, pad;
  uint4 raw[2][19];
};

// Workers per request.  The floor is the share a request gets under
// overload: boards with many empty spots are split over several workers so
// that they finish in tens of milliseconds instead of seconds (18 empty spots
// get 3/8 of the pool, each spot fewer halves that, down to one worker).
// When workers are idle at admission a request takes up to half of them, so
// that at moderate load a board finishes in a fraction of the time, but no
// more than keeps every member busy: a pass has about 17,300 (s0, s1p) items
// at 10 empty spots and 2.9x as many per spot more, and a member gets at
// least half of that.  Any gang of at most half the pool makes progress: the
// gang's entries are consecutive in the ring and claimed in order, so a
// member only waits for workers that are finishing earlier requests.
static int gang_size(int spots, int workers, int idle) {
  int g = spots < 12 ? 1 : int((int64_t(workers) * 3 / 8) >> (18 - std::min(spots, 18)));
  double items = 17303;
  for (int s = 10; s < spots; s++) items *= 2.87;
  for (int s = 10; s > spots; s--) items /= 2.87;
  const int useful = std::max(1, int(items / (17303 / 2)));
  g = std::max(g, std::min(useful, idle / 2));
  return std::max(1, std::min(g, workers / 2));
}

struct serve_ctl {            // host-mapped
  volatile unsigned long long tail;   // entries published by the host
  volatile int32_t close;             // host asks workers to leave
  volatile int32_t status;            // kRunning / kIdleExit / kClosed
};

struct serve_dev {            // device memory
  unsigned long long head;    // entries claimed by workers
  unsigned long long tail;    // mirror of serve_ctl::tail (never ahead of it)
  int close;                  // mirror of serve_ctl::close; zeroed at each launch
  int lock;                   // held by the idle worker refreshing the mirror
};

// Three workers per SM (80 registers, 65 KB of shared memory each): with two,
// a worker's gathers from its global workspace were less covered, and the
// server's capacity fell below one-request-at-a-time solving (496 against
// 511 boards/s on the serving benchmark; three give 602).
__global__ void __launch_bounds__(kMidThreads, 3)
serve_kernel(serve_entry* ring, serve_ctl* ctl, serve_dev* dev, gang_aux* aux,
             const uint32_t* __restrict__ wf) {
  extern __shared__ uint4 smem[];
  set0_info* tiles = reinterpret_cast<set0_info*>(smem);
  __shared__ uint4 raw[2][19];
  __shared__ int fault;
  __shared__ long long claimed;
  __shared__ mid_job_t job;
  __shared__ int gang_s, rank_s, first_s;
  const mid_tables MT = {c_choose, c_winpat, wf};
  for (;;) {
    if (threadIdx.x == 0) {
      claimed = -1;
      unsigned long long polls = 0;
      const unsigned long long idle_since = global_ns();
      unsigned sleep_ns = 256;
      for (;;) {
        const unsigned long long h = atomicAdd(&dev->head, 0ull);
        const unsigned long long t = atomicAdd(&dev->tail, 0ull);
        if (h < t) {
          if (atomicCAS(&dev->head, h, h + 1) == h) { claimed = (long long)h; __threadfence_system(); break; }
          continue;
        }
        if (atomicAdd(&dev->close, 0)) { ctl->status = kClosed; break; }
        if (atomicCAS(&dev->lock, 0, 1) == 0) {
          const unsigned long long ht = ctl->tail;
          const int hc = ctl->close;
          atomicMax(&dev->tail, ht);
          if (hc) atomicExch(&dev->close, 1);
          atomicExch(&dev->lock, 0);
          if (ht > t || hc) continue;
        }
        if (++polls > kIdlePollsMax || global_ns() - idle_since > kIdleNs) { ctl->status = kIdleExit; break; }
        __nanosleep(sleep_ns);
        if (sleep_ns < 20000) sleep_ns *= 2;
      }
      fault = 0;
    }
    __syncthreads();
    if (claimed < 0) return;
    serve_entry& E = ring[claimed % kRing];
    __threadfence_system();
    // The entry is in host memory: its descriptor crosses the bus once, into
    // shared memory, and every thread reads it there (uncached loads, since
    // ring entries are reused).
    {
      const uint4* src = reinterpret_cast<const uint4*>(&E.job);
      uint4* dst = reinterpret_cast<uint4*>(&job);
      for (int i = int(threadIdx.x); i < int(sizeof(mid_job_t) / 16); i += int(blockDim.x)) dst[i] = __ldcv(src + i);
      if (threadIdx.x == 0) { gang_s = __ldcv(&E.gang); rank_s = __ldcv(&E.rank); first_s = __ldcv(&E.first); }
    }
    __syncthreads();
    const mid_job_t& J = job;
    const int gang = gang_s, rank = rank_s, first = first_s;
    if (gang <= 1) {
      mid_board_body(J, MT, tiles, J.workspace, raw, &fault, int(threadIdx.x), int(blockDim.x), 0, 1,
                     sync_threads(), sync_threads());
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence_system();
        E.done = fault ? -1 : 1;
      }
    } else {
      // One share of a request split over `gang` workers; the entries of the
      // gang are consecutive, so earlier requests never wait on later ones.
      gang_aux& X = aux[first];
      const board_barrier gb{&X.count, &X.gen, gang, &X.fault};
      mid_board_body(J, MT, tiles, J.workspace, X.raw, &X.fault, int(threadIdx.x), int(blockDim.x), rank, gang,
                     sync_threads(), gb);
      __syncthreads();
      if (rank == 0 && threadIdx.x == 0) {
        const int f = atomicExch(&X.fault, 0);
        __threadfence_system();
        ring[first].done = f ? -1 : 1;
      }
    }
    __syncthreads();
  }
}

// Host side: first-fit arena over one device allocation
struct arena {
  char* base = nullptr;
  size_t size = 0;
  std::map<size_t, size_t> free_;  // offset -> length
  void init(char* b, size_t n) { base = b; size = n; free_.clear(); free_[0] = n; }
  bool alloc(size_t n, size_t& off) {
    n = (n + 255) & ~size_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= n) {
        off = it->first;
        const size_t rest = it->second - n;
        free_.erase(it);
        if (rest) free_[off + n] = rest;
        return true;
      }
    return false;
  }
  void release(size_t off, size_t n) {
    n = (n + 255) & ~size_t(255);
    auto it = free_.emplace(off, n).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) { it->second += next->second; free_.erase(next); }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) { prev->second += it->second; free_.erase(it); }
    }
  }
};

struct server {
  std::mutex m;
  int device = 0;
  cudaStream_t stream = nullptr;
  serve_entry* ring = nullptr;        // mapped
  serve_ctl* ctl = nullptr;           // mapped
  pg_mid_values_t* results = nullptr; // mapped, one per ring entry
  serve_dev* dev = nullptr;           // device claim counter and tail mirror
  gang_aux* aux = nullptr;            // device, one per ring slot
  arena A;
  unsigned long long next = 0;        // next ticket (ring entry)
  int busy = 0;                       // workers in the gangs of unpolled requests
  struct inflight { size_t off, bytes; int gang; bool live; };
  std::vector<inflight> slots;        // per ring entry
  bool launched = false;
  int workers = 0;
};

static int launch_workers(server& S) {
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  S.ctl->close = 0;
  S.ctl->status = kRunning;
  const size_t smem = kMidThreads * sizeof(set0_info);
  PG_CUDA(cudaMemsetAsync(&S.dev->close, 0, sizeof(int), S.stream));
  serve_kernel<<<S.workers, kMidThreads, smem, S.stream>>>(S.ring, S.ctl, S.dev, S.aux, T->win_factors);
  PG_CUDA(cudaGetLastError());
  S.launched = true;
  return PG_OK;
}

}  // namespace pg

using namespace pg;

extern "C" int pg_serve_open(int64_t budget_bytes, pg_server_t* out) {
  if (!out || budget_bytes <= 0) return fail(PG_ERR_ARG, "bad server arguments");
  if (int rc = mid_prepare_device()) return rc;
  auto* S = new server;
  PG_CUDA(cudaGetDevice(&S->device));
  // Every worker's workspace is in the arena, so a worker needs only its set0
  // tiles in shared memory and several workers share an SM.
  int sms = 0, per_sm = 0;
  PG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->device));
  PG_CUDA(cudaFuncSetAttribute(serve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kMidThreads * sizeof(set0_info))));
  PG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_kernel, kMidThreads,
                                                        kMidThreads * sizeof(set0_info)));
  S->workers = sms * std::max(1, per_sm);
  PG_CUDA(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
  PG_CUDA(cudaHostAlloc((void**)&S->ring, sizeof(serve_entry) * kRing, cudaHostAllocMapped));
  PG_CUDA(cudaHostAlloc((void**)&S->ctl, sizeof(serve_ctl), cudaHostAllocMapped));
  PG_CUDA(cudaHostAlloc((void**)&S->results, sizeof(pg_mid_values_t) * kRing, cudaHostAllocMapped));
  memset((void*)S->ring, 0, sizeof(serve_entry) * kRing);
  memset((void*)S->ctl, 0, sizeof(serve_ctl));
  char* base = nullptr;
  PG_CUDA(cudaMalloc(&base, size_t(budget_bytes)));
  S->A.init(base, size_t(budget_bytes));
  S->slots.assign(kRing, server::inflight{0, 0, 1, false});
  PG_CUDA(cudaMalloc(&S->dev, sizeof(serve_dev)));
  PG_CUDA(cudaMemset(S->dev, 0, sizeof(serve_dev)));
  PG_CUDA(cudaMalloc(&S->aux, sizeof(gang_aux) * kRing));
  PG_CUDA(cudaMemset(S->aux, 0, sizeof(gang_aux) * kRing));
  *out = reinterpret_cast<pg_server_t>(S);
  return PG_OK;
}

// Returns a ticket >= 0, or PG_ERR_CAPACITY when the ring or the budget is full
// right now (the caller retries after polling).
extern "C" int64_t pg_serve_submit(pg_server_t h, uint64_t raw) {
  if (!h) return fail(PG_ERR_ARG, "null server");
  server& S = *reinterpret_cast<server*>(h);
  std::lock_guard<std::mutex> lock(S.m);
  std::string err;
  board_plan P;
  if (!plan_board(raw, P, err)) return fail(PG_ERR_ARG, err);
  const unsigned long long ticket = S.next;
  const int slot = int(ticket % kRing);
  const int gang = gang_size(P.job.spots, S.workers, std::max(0, S.workers - S.busy));
  for (int g = 0; g < gang; g++)
    if (S.slots[(slot + g) % kRing].live) return fail(PG_ERR_CAPACITY, "request ring full");
  const size_t bytes = scratch_bytes_of(P, true);
  size_t off = 0;
  if (!S.A.alloc(bytes, off)) return fail(PG_ERR_CAPACITY, "scratch budget exhausted");
  carve_scratch(P, S.A.base + off, true);
  P.job.out = S.results + slot;
  for (int g = 0; g < gang; g++) {
    serve_entry& E = S.ring[(slot + g) % kRing];
    E.done = 0;
    E.job = P.job;
    E.gang = gang;
    E.rank = g;
    E.first = slot;
    S.slots[(slot + g) % kRing] = server::inflight{off, bytes, gang, true};
  }
  S.busy += gang;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  S.next = ticket + gang;
  S.ctl->tail = ticket + gang;
  if (!S.launched || S.ctl->status != kRunning) {
    if (S.launched) cudaStreamSynchronize(S.stream);  // workers left after idling
    if (int rc = launch_workers(S)) return rc;
  }
  return int64_t(ticket);
}

// 1 and the result when ticket is solved, 0 while pending, < 0 on failure.
extern "C" int pg_serve_poll(pg_server_t h, int64_t ticket, pg_mid_values_t* result) {
  if (!h || ticket < 0) return fail(PG_ERR_ARG, "bad poll arguments");
  server& S = *reinterpret_cast<server*>(h);
  std::lock_guard<std::mutex> lock(S.m);
  const int slot = int(ticket % kRing);
  if (!S.slots[slot].live || (unsigned long long)ticket >= S.next) return fail(PG_ERR_ARG, "unknown ticket");
  const int done = S.ring[slot].done;
  if (!done) return 0;
  std::atomic_thread_fence(std::memory_order_acquire);
  if (result) memcpy(result, (const void*)(S.results + slot), sizeof(pg_mid_values_t));
  S.A.release(S.slots[slot].off, S.slots[slot].bytes);
  const int gang = S.slots[slot].gang;
  for (int g = 0; g < gang; g++) S.slots[(slot + g) % kRing].live = false;
  S.busy -= gang;
  return done > 0 ? 1 : fail(PG_ERR_BOUNDS, "midsolve bounds check failed");
}

extern "C" int pg_serve_state(pg_server_t h) {
  if (!h) return fail(PG_ERR_ARG, "null server");
  server& S = *reinterpret_cast<server*>(h);
  std::lock_guard<std::mutex> lock(S.m);
  return S.launched ? int(S.ctl->status) : 0;
}

extern "C" int pg_serve_close(pg_server_t h) {
  if (!h) return PG_OK;
  server* S = reinterpret_cast<server*>(h);
  S->ctl->close = 1;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  cudaError_t e = cudaStreamSynchronize(S->stream);
  cudaFree(S->A.base);
  cudaFree(S->dev);
  cudaFree(S->aux);
  cudaFreeHost((void*)S->ring);
  cudaFreeHost((void*)S->ctl);
  cudaFreeHost(S->results);
  cudaStreamDestroy(S->stream);
  delete S;
  return e == cudaSuccess ? PG_OK : cuda_fail(e, "pg_serve_close");
}
