// Per-device table upload and error reporting.
#include "runtime.h"
#include "tables.h"
#include "../../include/pentago_b200.h"
#include <map>
#include <mutex>
#include <vector>

namespace pg {

static thread_local std::string last_error;

void set_error(const std::string& msg) { last_error = msg; }
int fail(int code, const std::string& msg) { last_error = msg; return code; }
int cuda_fail(cudaError_t e, const char* what) {
  last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return PG_ERR_CUDA;
}

static std::mutex once_mutex;
static std::map<std::pair<int, const void*>, int> once_done;

int per_device_once(const void* key, int (*f)()) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(PG_ERR_CUDA, "no CUDA device");
  std::lock_guard<std::mutex> lock(once_mutex);
  auto it = once_done.find({dev, key});
  if (it != once_done.end()) return it->second;
  const int rc = f();
  once_done[{dev, key}] = rc;
  return rc;
}

static std::mutex dev_mutex;
static std::vector<dev_tables_t*> per_device;

template<class T> static T* upload(const T* host, size_t count) {
  T* d = nullptr;
  if (cudaMalloc(&d, sizeof(T) * count) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, host, sizeof(T) * count, cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
  return d;
}

const dev_tables_t* device_tables() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { set_error("no CUDA device"); return nullptr; }
  std::lock_guard<std::mutex> lock(dev_mutex);
  if (int(per_device.size()) <= dev) per_device.resize(dev + 1, nullptr);
  if (per_device[dev]) return per_device[dev];
  const tables_t& T = tables();
  auto* t = new dev_tables_t;
  t->rmin_flat = upload(T.rmin_flat, 19683);
  t->rmin_inv = upload(T.rmin_inv, 19683);
  t->unpack = upload(&T.unpack[0][0], 2 * 19683);
  t->win_factors = upload(&T.win_factors[0][0][0], 4 * 512 * 16);
  t->rmin_off = upload(T.rmin_off, 56);
  t->commute = upload(&T.commute[0][0], 8 * 256);
  t->win_union = upload(T.win_union.data(), T.win_union.size());
  t->pack = upload(T.pack, 512);
  t->pop_masks = upload(T.pop_masks, 512);
  t->rank9 = upload(T.rank9, 512);
  t->term_pat = upload(&T.term_pat[0][0], 4 * 17);
  t->term_other = upload(&T.term_other[0][0][0], 4 * 17 * 2);
  t->term_sub = upload(&T.term_sub[0][0][0], 4 * 512 * 4);
  t->cov = upload(&T.cov[0][0][0], 32 * 4 * 512);
  t->miss_pat = upload(&T.miss_pat[0][0], 4 * 15);
  t->miss_quad = upload(&T.miss_quad[0][0][0], 4 * 15 * 3);
  t->rot = upload(&T.rot[0][0], 512 * 2);
  t->refl = upload(T.refl, 512);
  t->cls_masks = upload(T.cls_masks, 512);
  if (!t->rmin_flat || !t->rmin_inv || !t->unpack || !t->win_factors || !t->rmin_off || !t->commute ||
      !t->win_union || !t->pack || !t->pop_masks || !t->rank9 || !t->term_pat || !t->term_other || !t->term_sub ||
      !t->cov || !t->miss_pat || !t->miss_quad || !t->rot || !t->refl || !t->cls_masks) {
    set_error("table upload failed");
    delete t;
    return nullptr;
  }
  // The entry points take their small per-call scratch (line records,
  // descriptors) from the device's default stream-ordered pool.  By default
  // that pool returns freed memory to the device at every synchronization,
  // so a caller that synchronizes between calls (a sweep, slice by slice)
  // paid to map it again on each call; the pool now keeps up to 256 MB for
  // reuse.  This is an attribute of this process's pool, gone at exit.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = uint64_t(256) << 20;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  per_device[dev] = t;
  return t;
}

dev_tables_t host_tables_view() {
  const tables_t& H = tables();
  return dev_tables_t{H.rmin_flat, H.rmin_inv, &H.unpack[0][0], &H.win_factors[0][0][0], H.rmin_off,
                      &H.commute[0][0], H.win_union.data(), H.pack, H.pop_masks, H.rank9,
                      &H.term_pat[0][0], &H.term_other[0][0][0], &H.term_sub[0][0][0], &H.cov[0][0][0],
                      &H.miss_pat[0][0], &H.miss_quad[0][0][0], &H.rot[0][0], H.refl, H.cls_masks};
}

}  // namespace pg

extern "C" const char* pg_last_error(void) { return pg::last_error.c_str(); }

extern "C" int pg_init(void) {
  pg::tables();
  return pg::device_tables() ? PG_OK : PG_ERR_CUDA;
}

// Host copy of a named lookup table, for tests that pin the tables against
// the SHA-1 hashes of the reference's generator.
extern "C" const void* pg_selftest_table(const char* name, int* bytes) {
  const pg::tables_t& T = pg::tables();
  const std::string n(name);
#define PG_T(str, x) if (n == str) { *bytes = int(sizeof(x)); return &x; }
  PG_T("pack_table", T.pack) PG_T("unpack_table", T.unpack) PG_T("rotations", T.rot)
  PG_T("reflections", T.refl) PG_T("commute_global_local_symmetries", T.commute)
  PG_T("rotation_minimal_quadrants_offsets", T.rmin_off) PG_T("rotation_minimal_quadrants_inverse", T.rmin_inv)
  PG_T("rotation_minimal_quadrants_reflect_moved", T.rmin_moved)
#undef PG_T
  if (n == "rotation_minimal_quadrants_flat") { *bytes = 2 * T.rmin_count; return T.rmin_flat; }
  *bytes = 0;
  return nullptr;
}
