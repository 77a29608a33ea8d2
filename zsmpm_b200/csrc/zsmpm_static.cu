// zsmpm_activate_blocks_noalloc: block activation (ComputeSparsity + EnlargeSparsity +
// ascending block order) that allocates nothing.
//
// Some callers cannot call cudaMalloc when they need this step: hosts whose own pool has
// already reserved the GPU's memory, and plug-in or real-time loops that forbid allocation
// after start-up.  For them the scratch of this entry point (hash table, dense
// bitmap, scan partials, counters) lives in a fixed file-scope device array instead of
// scene-owned buffers; the caller passes the inputs and the outputs.
//
// Limits: at most kNoAllocMaxParticles particles, at most kNoAllocTableSlots - 20 active
// blocks (every call uses the whole kNoAllocTableSlots-slot table: the sorted keys do not
// depend on the table size, so a sparse input of few particles may still activate up to that
// many blocks), and an active-block bounding box of at most kNoAllocBitmapWords * 32
// positions.  The array occupies kNoAllocScratchBytes (about 3 MB) on every GPU that loads the
// library, until the process exits.
//
// Every call shares the one array and overwrites what the previous call left there; each
// call clears the parts that must start at zero (table, counters, bitmap, status) itself.
// Calls whose work overlaps on a GPU (on different streams, or from different host threads
// without ordering) race on the array and give undefined results.
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda.h>
#include <cuda_runtime.h>

#include "zsmpm.h"
#include "zsmpm_internal.h"

namespace zsmpm {
namespace {

constexpr int64_t kNoAllocTableSlots = 32768;
constexpr int64_t kNoAllocMaxParticles = (kNoAllocTableSlots / 16) * 512;  // 1,048,576
constexpr int64_t kNoAllocBitmapWords = 65536;
constexpr int64_t kNoAllocScanParts = 2 * kScanCtas + 1;

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// byte offsets of the regions inside the scratch array
constexpr size_t kOffPk = 0;
constexpr size_t kOffKeys = kOffPk + align256(8 * kNoAllocTableSlots);
constexpr size_t kOffIdx = kOffKeys + align256(12 * kNoAllocTableSlots);
constexpr size_t kOffStatus = kOffIdx + align256(4 * kNoAllocTableSlots);
constexpr size_t kOffActive = kOffStatus + align256(4 * kNoAllocTableSlots);
constexpr size_t kOffInsPk = kOffActive + align256(12 * kNoAllocTableSlots);
constexpr size_t kOffInsSlot = kOffInsPk + align256(8 * kNoAllocTableSlots);
constexpr size_t kOffBlkPk = kOffInsSlot + align256(4 * kNoAllocTableSlots);
constexpr size_t kOffBitmap = kOffBlkPk + align256(8 * kNoAllocTableSlots);
constexpr size_t kOffPrefix = kOffBitmap + align256(4 * kNoAllocBitmapWords);
constexpr size_t kOffCtr = kOffPrefix + align256(4 * (kNoAllocBitmapWords + 1));
constexpr size_t kOffCnt = kOffCtr + align256(4 * kCtrCount);
constexpr size_t kOffScan = kOffCnt + align256(4);
constexpr size_t kNoAllocScratchBytes = kOffScan + align256(4 * kNoAllocScanParts);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Host code must not pass &g_noalloc_scratch to a kernel: on the host that name is a
// stand-in, not a device address.  The device address belongs to a CUDA context (the module
// holding the array is loaded per context), so it is looked up with cudaGetSymbolAddress once
// per context, with that context's device current, and cached under the context's
// process-unique id (cuCtxGetId).  A context that the caller destroys and recreates (for
// example after cudaDeviceReset), or a context the host made itself, has a new id and gets a
// fresh lookup, so a cached address is never used outside the context it came from.  The two
// driver calls are reached through cudaGetDriverEntryPoint, so the library needs no libcuda
// link.
using ctx_get_current_fn = CUresult (*)(CUcontext *);
using ctx_get_id_fn = CUresult (*)(CUcontext, unsigned long long *);
constexpr int kMaxContexts = 64;
std::mutex g_mutex;
ctx_get_current_fn g_ctx_get_current = nullptr;
ctx_get_id_fn g_ctx_get_id = nullptr;
struct cached_address {
  unsigned long long ctx_id;
  unsigned char *ptr;
};
cached_address g_cache[kMaxContexts] = {};
int g_cached = 0;  // entries in use
int g_oldest = 0;  // entry replaced next once all are in use

int driver_calls() {
  if (g_ctx_get_current && g_ctx_get_id) return ZSMPM_OK;
  void *f0 = nullptr, *f1 = nullptr;
  cudaDriverEntryPointQueryResult q0{}, q1{};
  cudaError_t e0 = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0);
  cudaError_t e1 = cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1);
  if (e0 != cudaSuccess || e1 != cudaSuccess || !f0 || !f1 || q0 != cudaDriverEntryPointSuccess ||
      q1 != cudaDriverEntryPointSuccess)
    return record_error(ZSMPM_ERR_CUDA, "cuCtxGetCurrent / cuCtxGetId not available from the CUDA driver");
  g_ctx_get_current = reinterpret_cast<ctx_get_current_fn>(f0);
  g_ctx_get_id = reinterpret_cast<ctx_get_id_fn>(f1);
  return ZSMPM_OK;
}

int current_context_id(unsigned long long *id) {
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return 1;
  return g_ctx_get_id(ctx, id) == CUDA_SUCCESS ? 0 : 1;
}

int scratch_address(unsigned char **out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  int st = driver_calls();
  if (st != ZSMPM_OK) return st;
  unsigned long long id = 0;
  const bool have_ctx = current_context_id(&id) == 0;
  if (have_ctx)
    for (int k = 0; k < g_cached; ++k)
      if (g_cache[k].ctx_id == id) {
        *out = g_cache[k].ptr;
        return ZSMPM_OK;
      }
  // the lookup also makes the device's primary context current when none is
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    std::string msg = std::string("cudaGetSymbolAddress of the no-alloc scratch: ") + cudaGetErrorString(e);
    return record_error(ZSMPM_ERR_CUDA, msg.c_str());
  }
  if (current_context_id(&id) == 0) {
    // once every entry is in use (a process that recreates contexts often), the oldest goes
    int k = g_cached;
    if (g_cached < kMaxContexts) {
      ++g_cached;
    } else {
      k = g_oldest;
      g_oldest = (g_oldest + 1) % kMaxContexts;
    }
    g_cache[k] = cached_address{id, static_cast<unsigned char *>(p)};
  }
  *out = static_cast<unsigned char *>(p);
  return ZSMPM_OK;
}

}  // namespace
}  // namespace zsmpm

using namespace zsmpm;

extern "C" ZSMPM_API zsmpm_status zsmpm_activate_blocks_noalloc(const float *x, int64_t n, float dx,
                                                                int32_t *keys_out, int32_t cap_blocks,
                                                                int32_t *count_out, void *stream) {
  if (!x || !keys_out || !count_out)
    return (zsmpm_status)record_error(ZSMPM_ERR_INVALID_ARG, "x, keys_out and count_out are required");
  if (!(dx > 0.f)) return (zsmpm_status)record_error(ZSMPM_ERR_INVALID_ARG, "dx must be > 0");
  if (cap_blocks < 1) return (zsmpm_status)record_error(ZSMPM_ERR_INVALID_ARG, "cap_blocks must be >= 1");
  if (n < 1 || n > kNoAllocMaxParticles)
    return (zsmpm_status)record_error(
        ZSMPM_ERR_CAPACITY,
        "zsmpm_activate_blocks_noalloc takes 1 to 1048576 particles (its fixed scratch holds a "
        "32768-slot table); use a scene (zsmpm_scene_create) for more");
  unsigned char *base = nullptr;
  int st = scratch_address(&base);
  if (st != ZSMPM_OK) return (zsmpm_status)st;

  // the whole table on every call: the sorted keys are the same for any table that holds them
  const int64_t T = kNoAllocTableSlots;
  scene_device s{};
  s.prm.n = (int)n;
  s.prm.dx = dx;
  s.prm.inv_dx = 1.f / dx;
  s.prm.table_size = (int)T;
  s.prm.nb_cap = (int)(T - 20);
  s.prm.bitmap_cap = (int)kNoAllocBitmapWords;
  s.pk = reinterpret_cast<uint64_t *>(base + kOffPk);
  s.tkeys = reinterpret_cast<int *>(base + kOffKeys);
  s.tidx = reinterpret_cast<int *>(base + kOffIdx);
  s.tstatus = reinterpret_cast<int *>(base + kOffStatus);
  s.active_keys = reinterpret_cast<int *>(base + kOffActive);
  s.ins_pk = reinterpret_cast<uint64_t *>(base + kOffInsPk);
  s.ins_slot = reinterpret_cast<int *>(base + kOffInsSlot);
  s.blk_pk = reinterpret_cast<uint64_t *>(base + kOffBlkPk);
  s.bitmap = reinterpret_cast<uint32_t *>(base + kOffBitmap);
  s.word_prefix = reinterpret_cast<int *>(base + kOffPrefix);
  s.ctr = reinterpret_cast<int *>(base + kOffCtr);
  s.view_cnt = reinterpret_cast<int *>(base + kOffCnt);
  s.scan_part = reinterpret_cast<int *>(base + kOffScan);
  cudaError_t e = launch_activate_static(s, x, keys_out, cap_blocks, count_out, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    std::string msg = std::string("zsmpm_activate_blocks_noalloc launch: ") + cudaGetErrorString(e);
    return (zsmpm_status)record_error(ZSMPM_ERR_CUDA, msg.c_str());
  }
  return ZSMPM_OK;
}
