// Midsolve on the GPU: the replacement for midsolve / midsolve_internal
// (pentago/mid/midengine.cc:93-178).
//
// The reference solves every position downstream of a root with >= 18 stones
// by retrograde analysis over subset-ranked stone placements: two passes
// ("aggressive" = who wins ties), each sweeping the number of placed stones n
// from `spots` down to 0, where level n reads level n+1 from a workspace that
// ping-pongs between the two ends of one buffer (mid/internal.h:29-69,
// :358-408).
//
// Here a CTA runs whole passes of one board.  It precomputes the per-level
// tables (midengine.cc:57-76), then runs its passes with a CTA barrier
// between levels.  Inside a level the (s0, s1p) items are split over the
// CTA's threads in tiles of s0 rows whose per-row data (make_set0_info,
// internal.h:174-259) is built cooperatively in shared memory.  Boards with
// up to 10 empty spots (26 or more stones) keep their whole workspace in
// shared memory (bottleneck(10) = 8400 halfsupers = 134 KB): in a batch, one
// CTA per pass (mid_pass_kernel); larger boards use a global-memory
// workspace.  The last step, midsolve_traverse (midengine.cc:127-158), also
// runs on the device and writes the reference's mid_values_t records.
#include "mid_body.cuh"
#include "runtime.h"
#include <atomic>
#include <algorithm>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

namespace pg {

// Threads of a CTA that solves one board alone (its tiles stay kMidThreads
// set0 rows: the extra warps share the rows' items).
constexpr int kMidBoardThreads = 512;

__global__ void __launch_bounds__(kMidBoardThreads)
mid_board_kernel(const mid_job_t* __restrict__ jobs, const uint32_t* __restrict__ wf, int smem_workspace) {
  const mid_job_t& J = jobs[blockIdx.x];
  extern __shared__ uint4 smem[];
  set0_info* tiles = reinterpret_cast<set0_info*>(smem);  // kMidThreads entries
  uint4* ws = smem_workspace ? smem + kMidThreads * sizeof(set0_info) / sizeof(uint4) : J.workspace;
  __shared__ uint4 raw[2][19];
  __shared__ int fault;
  if (threadIdx.x == 0) fault = 0;
  __syncthreads();
  const mid_tables MT = {c_choose, c_winpat, wf};
  mid_board_body(J, MT, tiles, ws, raw, &fault, threadIdx.x, blockDim.x, 0, 1, sync_threads(), sync_threads());
}

// Where the two pass CTAs of one board meet: each publishes the n <= 1
// results of its pass (raw[pass][0..spots]) and its bounds-check fault, then
// counts itself done; zero at launch.
struct pass_meet {
  uint4 raw[2][19];
  unsigned done;
  int fault;
  int pad[2];
};

// The boards of pg_midsolve_batch whose workspace fits shared memory: two
// CTAs per board, CTA 2b + p running pass p (aggressive = p) of board b over
// its own copy of the per-level tables (jobs[2b + p]).  The passes share no
// workspace, so neither CTA waits for the other: the one that finishes second
// (an atomic count, no spinning) gathers both passes' results and runs the
// traversal.  A 64-board batch thus spreads over 128 SMs instead of 64.
__global__ void __launch_bounds__(kMidBoardThreads)
mid_pass_kernel(const mid_job_t* __restrict__ jobs, const uint32_t* __restrict__ wf, pass_meet* meet) {
  const int board = blockIdx.x >> 1, pass = blockIdx.x & 1;
  const mid_job_t& J = jobs[blockIdx.x];
  extern __shared__ uint4 smem[];
  set0_info* tiles = reinterpret_cast<set0_info*>(smem);  // kMidThreads entries
  uint4* ws = smem + kMidThreads * sizeof(set0_info) / sizeof(uint4);
  __shared__ uint4 raw[2][19];
  __shared__ int fault, last;
  if (threadIdx.x == 0) fault = 0;
  __syncthreads();
  const mid_tables MT = {c_choose, c_winpat, wf};
  mid_board_body(J, MT, tiles, ws, raw, &fault, threadIdx.x, blockDim.x, 0, 1, sync_threads(), sync_threads(),
                 nullptr, pass, pass + 1, false);
  pass_meet& M = meet[board];
  if (threadIdx.x < 19) M.raw[pass][threadIdx.x] = raw[pass][threadIdx.x];
  if (threadIdx.x == 0 && fault) atomicExch(&M.fault, 1);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&M.done, 1u) == 1u;
  __syncthreads();
  if (!last || threadIdx.x >= 32) return;
  __threadfence();
  if (atomicAdd(&M.fault, 0)) {
    if (threadIdx.x == 0) { J.out->size = -1; J.out->pad = 0; }
    return;
  }
  // Interleave (midengine.cc:119-124) and traverse on the first warp
  uint4 supers[2 * 19];
  for (int i = 0; i < 19; i++)
    for (int j = 0; j < 2; j++) supers[2 * i + j] = __ldcg(&M.raw[j ^ (i == 0)][i]);
#ifdef __CUDA_ARCH__
  traverse_warp(J, MT, supers, J.out, int(threadIdx.x));
#endif
}

// One CTA waiting twice at a barrier of two that the other never reaches:
// the first wait runs out after `polls` polls and marks the fault, the second
// returns at once (what a board whose CTAs stopped meeting gets).
__global__ void barrier_timeout_kernel(unsigned* words, int* fault, unsigned polls) {
  board_barrier gb{words, words + 1, 2, fault};
  gb.polls = polls;
  gb();
  gb();
}

// A few large boards: ncta CTAs per board (blockIdx.x / ncta), each taking a
// contiguous share of every level.  bar: 2 words per board; raw: 38 uint4 per
// board; faults: one per board; all zero at launch.
__global__ void __launch_bounds__(kMidThreads, 3)
mid_board_grid_kernel(const mid_job_t* __restrict__ jobs, const uint32_t* __restrict__ wf, int ncta, unsigned* bar,
                      uint4* rawg, int* faults) {
  const int board = blockIdx.x / ncta, cta = blockIdx.x % ncta;
  const mid_job_t& J = jobs[board];
  extern __shared__ uint4 smem[];
  set0_info* tiles = reinterpret_cast<set0_info*>(smem);
  const mid_tables MT = {c_choose, c_winpat, wf};
  const board_barrier gb{bar + 2 * board, bar + 2 * board + 1, ncta, faults + board};
  mid_board_body(J, MT, tiles, J.workspace, reinterpret_cast<uint4(*)[19]>(rawg + 38 * board), faults + board,
                 int(threadIdx.x), int(blockDim.x), cta, ncta, sync_threads(), gb);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

static uint32_t h_choose[19][11];

int hchoose(int n, int k) {
  if (n < 0 || k < 0 || k > n) return 0;
  long r = 1;
  for (int i = 0; i < k; i++) r = r * (n - i) / (i + 1);
  return int(r);
}

int bottleneck(int spots) {  // mid/internal.h:37-47
  int worst = 0, prev = 1;
  for (int n = 0; n <= spots; n++) {
    int next = hchoose(spots, n + 1);
    if (next) next *= hchoose(n + 1, (n + 1) / 2);
    worst = std::max(worst, prev + next);
    prev = next;
  }
  return worst;
}

static bool decode_board(uint64_t raw, mid_job_t& J, std::string& err) {
  // high_board_t::from_raw (high/board.h:77, board.cc:95-111)
  const uint64_t board = raw << 1 >> 1;
  const int middle = int(raw >> 63);
  uint64_t s0 = 0, s1 = 0;
  for (int q = 0; q < 4; q++) {
    uint32_t quad = uint32_t(board >> (16 * q)) & 0xffff;
    if (quad >= 19683) { err = "invalid board"; return false; }
    for (int i = 0; i < 9; i++) {
      const int s = quad % 3;
      quad /= 3;
      s0 |= uint64_t(s == 1) << (16 * q + i);
      s1 |= uint64_t(s == 2) << (16 * q + i);
    }
  }
  const int stones = __builtin_popcountll(s0 | s1);
  if (middle && stones == 0) { err = "invalid board"; return false; }
  J.side[0] = s0;
  J.side[1] = s1;
  J.ply = uint32_t(2 * stones - middle);
  J.spots = 36 - stones;
  if (J.spots > 18) { err = "midsolve needs at least 18 stones"; return false; }
  return true;
}

bool plan_board(uint64_t raw, board_plan& P, std::string& err) {
  mid_job_t& J = P.job;
  memset(&J, 0, sizeof J);
  if (!decode_board(raw, J, err)) return false;
  const uint64_t empty = 0x01ff01ff01ff01ffull ^ J.side[0] ^ J.side[1];
  int next = 0;
  for (int i = 0; i < 64; i++)
    if (empty >> i & 1) J.empty[next++] = uint8_t(i);
  const int spots = J.spots, ws = bottleneck(spots);
  for (int n = 0; n <= spots; n++) {  // make_info (mid/internal.h:49-69)
    const int k0 = n >> 1, k1 = n - k0;
    const int s1 = hchoose(spots, k1), s0p = hchoose(spots - k1, k0), s1p = hchoose(spots - k0, k1);
    J.sets1p_off[n + 1] = J.sets1p_off[n] + s1p;
    J.cs1ps_off[n + 1] = J.cs1ps_off[n] + s1p * (spots - k0);
    J.wins1_off[n + 1] = J.wins1_off[n] + s1;
    J.spaces[n].ny = s0p;
    J.spaces[n].lo = (n & 1) ? ws - s1 * s0p : 0;
    J.spaces[n].size = s1 * s0p;
  }
  J.spaces[spots + 1] = mid_grab{0, 0, 0};
  P.sets1p = J.sets1p_off[spots + 1];
  P.wins1 = 2 * size_t(J.wins1_off[spots + 1]);
  P.cs1ps = J.cs1ps_off[spots + 1];
  P.workspace = ws;
  J.ws_size = ws;
  return true;
}

static int mid_kernel_attrs() {
  const int smem_ws = int(kMidThreads * sizeof(set0_info) + kSmemWorkspaceMax * 16);
  return cudaFuncSetAttribute(mid_board_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_ws) ==
                     cudaSuccess &&
                 cudaFuncSetAttribute(mid_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_ws) ==
                     cudaSuccess &&
                 cudaFuncSetAttribute(mid_board_grid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(kMidThreads * sizeof(set0_info))) == cudaSuccess
             ? 0 : PG_ERR_CUDA;
}

static int upload_consts() {
  if (int rc = mid_prepare_device()) return rc;
  return per_device_once((const void*)&mid_kernel_attrs, mid_kernel_attrs);
}

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// CTAs per board for the grid kernel: the co-resident CTAs of the device
// shared evenly by the boards; 1 means one CTA per board (the batch kernel).
static int grid_ctas_per_board(int boards, size_t smem) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mid_board_grid_kernel, kMidThreads, smem) != cudaSuccess)
    return 1;
  return std::max(1, sms * per_sm / std::max(boards, 1));
}

// Per board of the grid kernel: barrier words, the n <= 1 results of both
// passes, a fault flag; all zero at launch.
static size_t grid_aux_bytes(int boards) {
  return align256(sizeof(unsigned) * 2 * size_t(boards)) + align256(sizeof(uint4) * 38 * size_t(boards)) +
         align256(sizeof(int) * size_t(boards));
}

// aux: device buffer of grid_aux_bytes(boards).
static int launch_grid_boards(const mid_job_t* jobs, int boards, int ncta, size_t smem, const uint32_t* wf,
                              char* aux, cudaStream_t stream) {
  PG_CUDA(cudaMemsetAsync(aux, 0, grid_aux_bytes(boards), stream));
  unsigned* bar = (unsigned*)aux;
  uint4* rawg = (uint4*)(aux + align256(sizeof(unsigned) * 2 * size_t(boards)));
  int* faults = (int*)(aux + align256(sizeof(unsigned) * 2 * size_t(boards)) +
                       align256(sizeof(uint4) * 38 * size_t(boards)));
  void* args[] = {(void*)&jobs, (void*)&wf, (void*)&ncta, (void*)&bar, (void*)&rawg, (void*)&faults};
  PG_CUDA(cudaLaunchCooperativeKernel((void*)mid_board_grid_kernel, dim3(unsigned(boards * ncta)), dim3(kMidThreads),
                                      args, smem, stream));
  return PG_OK;
}

size_t scratch_bytes_of(const board_plan& P, bool global_ws) {
  return align256(P.sets1p * 8) + align256(P.wins1 * 16) + align256(P.cs1ps * 2) +
         (global_ws || P.workspace > size_t(kSmemWorkspaceMax) ? align256(P.workspace * 16) : 0);
}

void carve_scratch(board_plan& P, char* base, bool global_ws) {
  mid_job_t& J = P.job;
  size_t off = 0;
  J.sets1p = (uint64_t*)(base + off); off += align256(P.sets1p * 8);
  J.wins1 = (uint4*)(base + off); off += align256(P.wins1 * 16);
  J.cs1ps = (uint16_t*)(base + off); off += align256(P.cs1ps * 2);
  J.workspace = global_ws || P.workspace > size_t(kSmemWorkspaceMax) ? (uint4*)(base + off) : nullptr;
}

// pg_midsolve_batch's scratch: the pass_meet records of the shared-memory
// boards, the job descriptors (two per shared-memory board, one per pass
// CTA, then one per larger board), the grid kernel's per-board words, then
// per board its tables (twice for a
// shared-memory board: one copy per pass CTA) and, for a larger board, its
// global workspace.  With the caller's scratch, nothing is allocated.
static bool smem_board(const board_plan& P) { return P.workspace <= size_t(kSmemWorkspaceMax); }
static size_t batch_bytes_of(const board_plan& P) { return (smem_board(P) ? 2 : 1) * scratch_bytes_of(P); }
static size_t meet_bytes(int nsmall) { return align256(sizeof(pass_meet) * size_t(nsmall)); }
static size_t small_jobs_bytes(int nsmall) { return align256(sizeof(mid_job_t) * 2 * size_t(nsmall)); }
static size_t jobs_bytes(int nsmall, int nlarge) {
  return small_jobs_bytes(nsmall) + align256(sizeof(mid_job_t) * size_t(nlarge));
}
// Everything before the boards' tables: pass_meet records, job descriptors
// and the grid kernel's per-board words.
static size_t head_bytes(int nsmall, int nlarge) {
  return meet_bytes(nsmall) + jobs_bytes(nsmall, nlarge) + (nlarge ? grid_aux_bytes(nlarge) : 0);
}

}  // namespace pg

using namespace pg;

extern "C" int pg_midsolve_workspace_size(int stones) {
  if (stones < 18 || stones > 36) return fail(PG_ERR_ARG, "stones out of range");
  return bottleneck(36 - stones);
}

extern "C" int pg_midsolve_scratch_bytes(const uint64_t* raws, int n, int64_t* bytes) {
  std::string err;
  size_t total = 0;
  int nsmall = 0;
  for (int i = 0; i < n; i++) {
    board_plan P;
    if (!plan_board(raws[i], P, err)) return fail(PG_ERR_ARG, err);
    total += batch_bytes_of(P);
    nsmall += smem_board(P);
  }
  *bytes = int64_t(total + head_bytes(nsmall, n - nsmall));
  return PG_OK;
}

// Solve a batch of boards given as raw_t (high/board.h:77).  out: device array
// of n pg_mid_values_t.  scratch: device buffer of pg_midsolve_scratch_bytes
// bytes, or null to let the library allocate it on the stream.
extern "C" int pg_midsolve_batch(const uint64_t* raws, int n, pg_mid_values_t* out, void* scratch,
                                 int64_t scratch_bytes, void* stream_) {
  if (n < 0 || (n && (!raws || !out))) return fail(PG_ERR_ARG, "bad midsolve arguments");
  if (!n) return PG_OK;
  cudaStream_t stream = (cudaStream_t)stream_;
  const dev_tables_t* T = device_tables();
  if (!T) return PG_ERR_CUDA;
  if (int rc = upload_consts()) return fail(rc, "midsolve constant upload failed");
  std::string err;
  std::vector<board_plan> plans(n);
  size_t total = 0;
  int nsmall = 0;
  for (int i = 0; i < n; i++) {
    if (!plan_board(raws[i], plans[i], err)) return fail(PG_ERR_ARG, "board " + std::to_string(i) + ": " + err);
    total += batch_bytes_of(plans[i]);
    nsmall += smem_board(plans[i]);
  }
  const int nlarge = n - nsmall;
  const size_t head = meet_bytes(nsmall), jbytes = jobs_bytes(nsmall, nlarge);
  total += head_bytes(nsmall, nlarge);
  stream_scratch X(stream);
  char* base = (char*)scratch;
  if (!base) {
    PG_CUDA(X.alloc(&base, std::max<size_t>(total, 256)));
  } else if (size_t(scratch_bytes) < total) {
    return fail(PG_ERR_CAPACITY, "midsolve scratch too small");
  }
  pass_meet* meets = reinterpret_cast<pass_meet*>(base);
  // The job descriptors in the layout they take on the device, copied in one
  // piece: small boards' pass jobs (board b at 2b, 2b + 1), then large boards.
  std::vector<char> host_jobs(jbytes);
  mid_job_t* small = reinterpret_cast<mid_job_t*>(host_jobs.data());
  mid_job_t* large = reinterpret_cast<mid_job_t*>(host_jobs.data() + small_jobs_bytes(nsmall));
  char* grid_aux = base + head + jbytes;
  size_t off = head_bytes(nsmall, nlarge);
  for (int i = 0, ns = 0, nl = 0; i < n; i++) {
    auto& P = plans[i];
    P.job.out = out + i;
    const size_t bytes = scratch_bytes_of(P);
    for (int copy = 0; copy < (smem_board(P) ? 2 : 1); copy++) {
      carve_scratch(P, base + off);
      off += bytes;
      if (smem_board(P)) small[ns++] = P.job;
      else large[nl++] = P.job;
    }
  }
  char* djobs = base + head;
  PG_CUDA(cudaMemcpyAsync(djobs, host_jobs.data(), jbytes, cudaMemcpyHostToDevice, stream));
  if (nsmall) {
    PG_CUDA(cudaMemsetAsync(meets, 0, sizeof(pass_meet) * size_t(nsmall), stream));
    const size_t smem = kMidThreads * sizeof(set0_info) + kSmemWorkspaceMax * 16;
    mid_pass_kernel<<<unsigned(2 * nsmall), kMidBoardThreads, smem, stream>>>(
        reinterpret_cast<const mid_job_t*>(djobs), T->win_factors, meets);
    PG_CUDA(cudaGetLastError());
  }
  if (nlarge) {
    const mid_job_t* d = reinterpret_cast<const mid_job_t*>(djobs + small_jobs_bytes(nsmall));
    const size_t smem = kMidThreads * sizeof(set0_info);
    const int ncta = grid_ctas_per_board(nlarge, smem);
    if (ncta <= 1) {
      mid_board_kernel<<<unsigned(nlarge), kMidBoardThreads, smem, stream>>>(d, T->win_factors, 0);
      PG_CUDA(cudaGetLastError());
    } else {
      if (int rc = launch_grid_boards(d, nlarge, ncta, smem, T->win_factors, grid_aux, stream)) return rc;
    }
  }
  return PG_OK;
}

extern "C" int pg_debug_barrier_timeout(unsigned polls, int* fault_out) {
  if (!fault_out) return fail(PG_ERR_ARG, "null argument");
  cudaStream_t st = nullptr;
  stream_scratch X(st);
  unsigned* words = nullptr;
  int* fault = nullptr;
  PG_CUDA(X.alloc(&words, 2 * sizeof(unsigned)));
  PG_CUDA(X.alloc(&fault, sizeof(int)));
  PG_CUDA(cudaMemsetAsync(words, 0, 2 * sizeof(unsigned), st));
  PG_CUDA(cudaMemsetAsync(fault, 0, sizeof(int), st));
  barrier_timeout_kernel<<<1, 32, 0, st>>>(words, fault, polls);
  PG_CUDA(cudaGetLastError());
  PG_CUDA(cudaMemcpyAsync(fault_out, fault, sizeof(int), cudaMemcpyDeviceToHost, st));
  PG_CUDA(cudaStreamSynchronize(st));
  return PG_OK;
}

// The kernel's own solve, run single-threaded on the host (CPU self-test of
// the midsolve arithmetic and indexing).  out: host array of n records.
extern "C" int pg_selftest_midsolve_host(const uint64_t* raws, int n, pg_mid_values_t* out, uint64_t* supers) {
  for (int k = 0; k <= 18; k++)
    for (int j = 0; j <= 10; j++) h_choose[k][j] = uint32_t(hchoose(k, j));
  const tables_t& T = tables();
  const mid_tables MT = {h_choose, T.winpat, &T.win_factors[0][0][0]};
  std::string err;
  std::vector<set0_info> tiles(kMidThreads);
  uint4 raw[2][19];
  for (int i = 0; i < n; i++) {
    board_plan P;
    if (!plan_board(raws[i], P, err)) return fail(PG_ERR_ARG, err);
    std::vector<uint64_t> sets1p(P.sets1p + 1);
    std::vector<uint4> wins1(P.wins1 + 1), ws(P.workspace + 1);
    std::vector<uint16_t> cs1ps(P.cs1ps + 1);
    mid_job_t J = P.job;
    J.sets1p = sets1p.data();
    J.wins1 = wins1.data();
    J.cs1ps = cs1ps.data();
    J.workspace = ws.data();
    J.out = out + i;
    memset(raw, 0, sizeof raw);
    int fault = 0;
    J.ws_size = int(P.workspace);
    mid_board_body(J, MT, tiles.data(), ws.data(), raw, &fault, 0, 1, 0, 1, [] {}, [] {},
                   supers ? reinterpret_cast<uint4*>(supers + 76 * size_t(i)) : nullptr);
  }
  return PG_OK;
}

namespace {
struct host_barrier {
  std::mutex m;
  std::condition_variable cv;
  int n, count = 0;
  unsigned gen = 0;
  explicit host_barrier(int n_) : n(n_) {}
  void wait() {
    std::unique_lock<std::mutex> lock(m);
    const unsigned g = gen;
    if (++count == n) {
      count = 0;
      gen++;
      cv.notify_all();
    } else {
      cv.wait(lock, [&] { return gen != g; });
    }
  }
};
}  // namespace

extern "C" int pg_selftest_midsolve_groups_host(const uint64_t* raws, int n, int groups, pg_mid_values_t* out) {
  if (n < 0 || groups < 1 || groups > 64) return fail(PG_ERR_ARG, "bad arguments");
  for (int k = 0; k <= 18; k++)
    for (int j = 0; j <= 10; j++) h_choose[k][j] = uint32_t(hchoose(k, j));
  const tables_t& T = tables();
  const mid_tables MT = {h_choose, T.winpat, &T.win_factors[0][0][0]};
  std::string err;
  for (int i = 0; i < n; i++) {
    board_plan P;
    if (!plan_board(raws[i], P, err)) return fail(PG_ERR_ARG, err);
    std::vector<uint64_t> sets1p(P.sets1p + 1);
    std::vector<uint4> wins1(P.wins1 + 1), ws(P.workspace + 1);
    std::vector<uint16_t> cs1ps(P.cs1ps + 1);
    mid_job_t J = P.job;
    J.sets1p = sets1p.data();
    J.wins1 = wins1.data();
    J.cs1ps = cs1ps.data();
    J.workspace = ws.data();
    J.out = out + i;
    J.ws_size = int(P.workspace);
    uint4 raw[2][19];
    memset(raw, 0, sizeof raw);
    int fault = 0;
    host_barrier hb(groups);
    std::vector<std::vector<set0_info>> tiles(groups, std::vector<set0_info>(kMidThreads));
    std::vector<std::thread> threads;
    for (int g = 0; g < groups; g++)
      threads.emplace_back([&, g] {
        mid_board_body(J, MT, tiles[g].data(), ws.data(), raw, &fault, 0, 1, g, groups, [] {}, [&] { hb.wait(); });
      });
    for (auto& t : threads) t.join();
  }
  return PG_OK;
}

// ===========================================================================
// Midsolve without allocation.
//
// Some callers cannot allocate device memory at the moment they want a
// solve: code inside a framework whose memory pool owns the whole device, or
// a real-time loop that must not pay for, or fail in, an allocation.
// pg_midsolve_batch_noalloc serves them with the one-CTA-per-board kernel
// (mid_board_kernel, both passes in one CTA), and every byte of device scratch it
// uses (the boards' job descriptors, their per-level tables and, for boards
// with more than 10 empty spots, their workspace) lives in one fixed array
// that is part of the library image, plus a fixed copy of the win-pattern
// table.
// ===========================================================================

namespace pg {

// Fixed scratch: 16 MiB per device, held by every GPU that loads the library
// until the process exits.  That fits, for example, 64 boards of 26 or more
// stones (about 70 KB each) or one board of 22 stones (about 15 MB).
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char noalloc_scratch[kNoAllocScratchBytes];
static __device__ __align__(256) uint32_t noalloc_win_factors[4 * 512 * 16];

struct noalloc_device {
  unsigned char* scratch = nullptr;   // device address of noalloc_scratch
  uint32_t* win_factors = nullptr;    // device address of noalloc_win_factors
  std::atomic<bool> ready{false};     // set last, once both are valid
};
static noalloc_device noalloc_state[64];  // per device ordinal
static std::mutex noalloc_mutex;

// Per-device set-up on the first call with that device current: resolve the
// device addresses of the two arrays (in host code their names are only
// host-side stand-ins) and fill the win-pattern table.  Nothing here
// allocates device memory.  Threads that race to make the first call wait on
// the lock; the ready flag is published after the addresses.
static int noalloc_setup(int dev) {
  noalloc_device& D = noalloc_state[dev];
  if (D.ready.load(std::memory_order_acquire)) return PG_OK;
  std::lock_guard<std::mutex> lock(noalloc_mutex);
  if (D.ready.load(std::memory_order_relaxed)) return PG_OK;
  void* s = nullptr;
  void* w = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&s, noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc_scratch)");
  e = cudaGetSymbolAddress(&w, noalloc_win_factors);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc_win_factors)");
  const tables_t& T = tables();
  e = cudaMemcpyToSymbol(noalloc_win_factors, &T.win_factors[0][0][0], sizeof(noalloc_win_factors));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyToSymbol(noalloc_win_factors)");
  if (int rc = upload_consts()) return fail(rc, "midsolve constant upload failed");
  D.win_factors = static_cast<uint32_t*>(w);
  D.scratch = static_cast<unsigned char*>(s);
  D.ready.store(true, std::memory_order_release);
  return PG_OK;
}

}  // namespace pg

// Same results as pg_midsolve_batch; see include/pentago_b200.h for the
// contract (fixed scratch, first-call set-up, calls that overlap race).
extern "C" int pg_midsolve_batch_noalloc(const uint64_t* raws, int n, pg_mid_values_t* out, void* stream_) {
  if (n < 0 || (n && (!raws || !out))) return fail(PG_ERR_ARG, "bad midsolve arguments");
  if (!n) return PG_OK;
  int dev = 0;
  PG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(PG_ERR_ARG, "device ordinal out of range");
  if (int rc = noalloc_setup(dev)) return rc;
  const noalloc_device& D = noalloc_state[dev];
  cudaStream_t stream = (cudaStream_t)stream_;
  std::string err;
  // Layout inside the fixed array: job descriptors of the shared-memory
  // boards, then of the global-workspace boards, then every board's tables.
  int nsmall = 0, nlarge = 0;
  size_t tables_bytes = 0;
  for (int i = 0; i < n; i++) {
    board_plan P;
    if (!plan_board(raws[i], P, err)) return fail(PG_ERR_ARG, "board " + std::to_string(i) + ": " + err);
    (P.workspace > size_t(kSmemWorkspaceMax) ? nlarge : nsmall)++;
    tables_bytes += scratch_bytes_of(P);
  }
  const size_t jobs_bytes = align256(sizeof(mid_job_t) * nsmall) + align256(sizeof(mid_job_t) * nlarge);
  if (jobs_bytes + tables_bytes > kNoAllocScratchBytes)
    return fail(PG_ERR_CAPACITY, "boards need " + std::to_string(jobs_bytes + tables_bytes) +
                                     " bytes of scratch; pg_midsolve_batch_noalloc has " +
                                     std::to_string(kNoAllocScratchBytes));
  unsigned char* small_dev = D.scratch;
  unsigned char* large_dev = D.scratch + align256(sizeof(mid_job_t) * nsmall);
  size_t off = jobs_bytes;
  std::vector<mid_job_t> small, large;
  for (int i = 0; i < n; i++) {
    board_plan P;
    plan_board(raws[i], P, err);
    carve_scratch(P, reinterpret_cast<char*>(D.scratch) + off);
    off += scratch_bytes_of(P);
    P.job.out = out + i;
    (P.workspace > size_t(kSmemWorkspaceMax) ? large : small).push_back(P.job);
  }
  for (int pass = 0; pass < 2; pass++) {
    const auto& jobs = pass ? large : small;
    if (jobs.empty()) continue;
    mid_job_t* d = reinterpret_cast<mid_job_t*>(pass ? large_dev : small_dev);
    PG_CUDA(cudaMemcpyAsync(d, jobs.data(), sizeof(mid_job_t) * jobs.size(), cudaMemcpyHostToDevice, stream));
    const int smem_ws = pass == 0;
    const size_t smem = kMidThreads * sizeof(set0_info) + (smem_ws ? kSmemWorkspaceMax * 16 : 0);
    mid_board_kernel<<<unsigned(jobs.size()), kMidBoardThreads, smem, stream>>>(d, D.win_factors, smem_ws);
    PG_CUDA(cudaGetLastError());
  }
  return PG_OK;
}
