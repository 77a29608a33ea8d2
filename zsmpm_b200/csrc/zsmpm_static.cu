// zsmpm_activate_blocks_noalloc: block activation (ComputeSparsity + EnlargeSparsity +
// ascending block order) that allocates nothing.
//
// Some callers cannot call cudaMalloc when they need this step: hosts whose own pool has
// already reserved the GPU's memory, and plug-in or real-time loops that forbid allocation
// after start-up.  For them the scratch of this entry point (hash table, dense
// bitmap, scan partials, counters) lives in a fixed file-scope device array instead of
// scene-owned buffers; the caller passes the inputs and the outputs.
//
// Limits: at most kNoAllocMaxParticles particles (the table is sized by the reference's
// rule next_2pow(max(n/512, 64)) * 16 slots, at most kNoAllocTableSlots), at most
// kNoAllocTableSlots - 20 active blocks, and an active-block bounding box of at most
// kNoAllocBitmapWords * 32 positions.  The array occupies kNoAllocScratchBytes (about 3 MB)
// on every GPU that loads the library, until the process exits.
//
// Every call shares the one array and overwrites what the previous call left there; each
// call clears the parts that must start at zero (table, counters, bitmap, status) itself.
// Calls whose work overlaps on a GPU (on different streams, or from different host threads
// without ordering) race on the array and give undefined results.
#include <cstdint>
#include <mutex>
#include <string>

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
// stand-in, not a device address.  The device address is looked up once per device with
// that device current and cached here.
constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned char *g_address[kMaxDevices] = {};

int scratch_address(int device, unsigned char **out) {
  if (device < 0 || device >= kMaxDevices)
    return record_error(ZSMPM_ERR_INVALID_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_address[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      std::string msg = std::string("cudaGetSymbolAddress of the no-alloc scratch: ") +
                        cudaGetErrorString(e);
      return record_error(ZSMPM_ERR_CUDA, msg.c_str());
    }
    g_address[device] = static_cast<unsigned char *>(p);
  }
  *out = g_address[device];
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
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) {
    std::string msg = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
    return (zsmpm_status)record_error(ZSMPM_ERR_CUDA, msg.c_str());
  }
  unsigned char *base = nullptr;
  int st = scratch_address(device, &base);
  if (st != ZSMPM_OK) return (zsmpm_status)st;

  // the table follows the reference's sizing rule, as a scene of n particles would
  int64_t expected = n / 512 < 64 ? 64 : n / 512;
  int64_t T = 1;
  while (T < expected) T <<= 1;
  T *= 16;
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
  e = launch_activate_static(s, x, keys_out, cap_blocks, count_out, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    std::string msg = std::string("zsmpm_activate_blocks_noalloc launch: ") + cudaGetErrorString(e);
    return (zsmpm_status)record_error(ZSMPM_ERR_CUDA, msg.c_str());
  }
  return ZSMPM_OK;
}
