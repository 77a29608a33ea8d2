// sm_100a kernels of the explicit MLS/APIC MPM substep.
//
// Pipeline of one substep (all launches have fixed shapes and read their sizes from
// device counters, so a substep can be captured in a CUDA graph):
//   activation  k_begin, k_insert_particle_blocks, k_enlarge, k_bitmap_prepare,
//               k_bitmap_set, scan(3), k_assign_ranks, k_neighbors
//   binning     k_bin_count, scan(3), k_cell_start, k_bin_scatter, k_bin_finalize
//   transfer    k_p2g, k_grid_update, k_g2p
// Reference operators replaced: SparsityOp.hpp:41-112 (activation), SparsityOp.hpp:115-196
// (binning), P2G.hpp:45-127, GridOp.hpp:54-164, G2P.hpp:43-84 (paths inside include/zensim).
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "zsmpm_device.cuh"
#include "zsmpm_internal.h"

namespace zsmpm {

namespace {

constexpr int kThreads = 256;
constexpr unsigned kFull = 0xffffffffu;
// Particle passes take kPass particles per thread per round: all loads first, so that several
// are in flight per thread (the passes are bound by load latency, not bandwidth).
constexpr int kPass = 4;

__device__ __forceinline__ void set_status(int *ctr, int bit) { atomicOr(&ctr[kCtrStatus], bit); }

__device__ __forceinline__ int grid_threads() { return gridDim.x * blockDim.x; }

// ----------------------------------------------------------------- hash table
// Insert with the reference's home slot and stride-127 linear probing
// (HashTable.hpp:356-374).  The slot is claimed by a 64-bit CAS on the packed key instead
// of the reference's per-slot spin lock, so no thread ever waits on another.
// Returns the insertion index when this call inserted the key, -1 when it existed, -2 when
// the table is full.
__device__ int table_insert(const scene_device &s, uint64_t key, int3 k, int *counter,
                            int index_base) {
  const int T = s.prm.table_size;
  int slot = home_slot(k.x, k.y, k.z, T);
  for (int probe = 0; probe < T; ++probe) {
    // most calls find their key already present (every warp of a block's particles asks):
    // a plain load settles those without a contended atomic
    unsigned long long prev = *reinterpret_cast<volatile unsigned long long *>(&s.pk[slot]);
    if (prev == (unsigned long long)key) return -1;
    if (prev == kEmptyKey)
      prev = atomicCAS((unsigned long long *)&s.pk[slot], (unsigned long long)kEmptyKey, (unsigned long long)key);
    if (prev == kEmptyKey) {
      const int idx = index_base + atomicAdd(counter, 1);
      s.tkeys[3 * slot + 0] = k.x;
      s.tkeys[3 * slot + 1] = k.y;
      s.tkeys[3 * slot + 2] = k.z;
      if (idx < s.prm.nb_cap) {
        s.ins_pk[idx] = key;
        s.ins_slot[idx] = slot;
        s.tidx[slot] = idx;
      } else {
        // beyond the block capacity: keep the key unqueryable so no kernel indexes past it
        set_status(s.ctr, kStatusCapacity);
        s.tidx[slot] = -1;
      }
      return idx;
    }
    if (prev == key) return -1;
    slot = (slot + 127) & (T - 1);
  }
  set_status(s.ctr, kStatusTableFull);
  return -2;
}

// HashTable::query (HashTable.hpp:444-456): index of the key or -1.
__device__ int table_query(const scene_device &s, uint64_t key, int3 k) {
  const int T = s.prm.table_size;
  int slot = home_slot(k.x, k.y, k.z, T);
  for (int probe = 0; probe < T; ++probe) {
    const uint64_t p = s.pk[slot];
    if (p == key) return s.tidx[slot];
    if (p == kEmptyKey) return -1;
    slot = (slot + 127) & (T - 1);
  }
  return -1;
}

// Stencil-origin cell and block of a position exactly as ComputeSparsity computes them
// (SparsityOp.hpp:70-77): c = floor(x * (1/dx) + 0.5) - 2, block = floor_div(c, 8).
// Returns false for NaN/Inf or positions beyond the packed key range.
__device__ __forceinline__ bool cell_of(const scene_params &p, float4 x, int3 &c, int3 &b) {
  const float fx = x.x * p.inv_dx + 0.5f, fy = x.y * p.inv_dx + 0.5f, fz = x.z * p.inv_dx + 0.5f;
  const float lim = (float)(kKeyLimit * 8);
  if (!(fabsf(fx) < lim && fabsf(fy) < lim && fabsf(fz) < lim)) return false;
  c = make_int3((int)floorf(fx) - 2, (int)floorf(fy) - 2, (int)floorf(fz) - 2);
  b = make_int3(block_of_cell(c.x), block_of_cell(c.y), block_of_cell(c.z));
  return true;
}

// x / dx, as G2P and G2P2G compute the particle's position in cells (G2P.hpp:56-58,
// G2P2G.hpp): a multiplication by 1/dx where dx is a power of two (the same number, since both
// scale by a power of two exactly), else the correctly rounded division.  (In P2G the same
// branch measured slower.)
__device__ __forceinline__ float over_dx(const scene_params &p, float x) {
  return p.dx_pow2 ? x * p.inv_dx : __fdiv_rn(x, p.dx);
}

// Batched scenes: the slot of a scene, the slot coordinate of a key component (keys of a
// scene lie in [32 slot - 4, 32 slot + 28)), and the scene-local block of a key.
__device__ __forceinline__ int3 slot_of_scene(int sc) { return make_int3(sc & 7, (sc >> 3) & 7, sc >> 6); }
__device__ __forceinline__ int slot_coord(int k) { return (k + kBatchMargin) / kBatchSlot; }
__device__ __forceinline__ int scene_of_key(int3 k) {
  return slot_coord(k.x) + 8 * slot_coord(k.y) + 64 * slot_coord(k.z);
}
__device__ __forceinline__ int3 local_block(const scene_params &p, int3 k) {
  if (!p.batch) return k;
  return make_int3(k.x - kBatchSlot * slot_coord(k.x), k.y - kBatchSlot * slot_coord(k.y),
                   k.z - kBatchSlot * slot_coord(k.z));
}

// Cell and block of particle i in the scene's key space: cell_of, then for batched scenes a
// check that the local block leaves room for the +1 enlargement inside the slot, and the
// slot offset.
// sid: the particle's scene (batched scenes only)
__device__ __forceinline__ bool particle_cell(const scene_device &s, int sid, float4 x, int3 &c, int3 &b) {
  if (!cell_of(s.prm, x, c, b)) return false;
  if (s.prm.batch) {
    const int hi = kBatchSlot - kBatchMargin - 1;
    if (b.x < -kBatchMargin || b.x >= hi || b.y < -kBatchMargin || b.y >= hi || b.z < -kBatchMargin || b.z >= hi)
      return false;
    const int3 o = slot_of_scene(sid);
    b = make_int3(b.x + kBatchSlot * o.x, b.y + kBatchSlot * o.y, b.z + kBatchSlot * o.z);
    c = make_int3(c.x + 8 * kBatchSlot * o.x, c.y + 8 * kBatchSlot * o.y, c.z + 8 * kBatchSlot * o.z);
  }
  return true;
}

// ----------------------------------------------------------------- CTA scan helpers
template <int NT>
__device__ __forceinline__ int cta_exclusive_scan(int v, int &total, int *smem /* >= NT/32 + 1 */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < NT / 32 ? smem[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    if (lane < NT / 32) smem[lane] = w;
    if (lane == NT / 32 - 1) smem[NT / 32] = w;
  }
  __syncthreads();
  const int incl = x + (warp > 0 ? smem[warp - 1] : 0);
  total = smem[NT / 32];
  __syncthreads();
  return incl - v;
}

// ----------------------------------------------------------------- device-wide scan
// Three-phase exclusive scan over n values produced by Load(i) (n read from device memory
// at *n_ptr), kScanCtas CTAs x kThreads.  out[n] receives the total.
struct load_popc {
  const uint32_t *w;
  __device__ int operator()(int i) const { return __popc(w[i]); }
};
struct load_int {
  const int *a;
  __device__ int operator()(int i) const { return a[i]; }
};

template <class Load>
__global__ void __launch_bounds__(kThreads) k_scan_reduce(Load ld, const int *n_ptr, int *part) {
  __shared__ int sm[kThreads / 32 + 1];
  const int n = *n_ptr;
  const int chunk = (n + gridDim.x - 1) / gridDim.x;
  const int lo = min(n, (int)blockIdx.x * chunk), hi = min(n, lo + chunk);
  int acc = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) acc += ld(i);
  int total;
  cta_exclusive_scan<kThreads>(acc, total, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kThreads) k_scan_partials(int *part, int parts) {
  __shared__ int sm[kThreads / 32 + 1];
  const int v = threadIdx.x < parts ? part[threadIdx.x] : 0;
  int total;
  const int ex = cta_exclusive_scan<kThreads>(v, total, sm);
  if (threadIdx.x < parts) part[threadIdx.x] = ex;
  if (threadIdx.x == 0) part[parts] = total;
}

template <class Load>
__global__ void __launch_bounds__(kThreads) k_scan_down(Load ld, const int *n_ptr, const int *part,
                                                         int *out) {
  __shared__ int sm[kThreads / 32 + 1];
  const int n = *n_ptr;
  const int chunk = (n + gridDim.x - 1) / gridDim.x;
  const int lo = min(n, (int)blockIdx.x * chunk), hi = min(n, lo + chunk);
  int run = part[blockIdx.x];
  for (int base = lo; base < hi; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = i < hi ? ld(i) : 0;
    int total;
    const int ex = cta_exclusive_scan<kThreads>(v, total, sm);
    if (i < hi) out[i] = run + ex;
    run += total;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = part[gridDim.x];
}

template <class Load>
cudaError_t device_scan(Load ld, const int *n_ptr, int *part, int *out, cudaStream_t st) {
  k_scan_reduce<<<kScanCtas, kThreads, 0, st>>>(ld, n_ptr, part);
  k_scan_partials<<<1, kThreads, 0, st>>>(part, kScanCtas);
  k_scan_down<<<kScanCtas, kThreads, 0, st>>>(ld, n_ptr, part, out);
  return cudaGetLastError();
}

// ----------------------------------------------------------------- activation
// Resets the hash table (CleanSparsity, SparsityOp.hpp:41-55) and the per-substep counters.
__global__ void __launch_bounds__(kThreads) k_begin(scene_device s) {
  const int T = s.prm.table_size;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += grid_threads()) {
    s.pk[i] = kEmptyKey;
    s.tkeys[3 * i + 0] = 0x7fffffff;
    s.tkeys[3 * i + 1] = 0x7fffffff;
    s.tkeys[3 * i + 2] = 0x7fffffff;
    s.tidx[i] = -1;
    s.tstatus[i] = -1;
  }
  if (blockIdx.x == 0 && threadIdx.x < kCtrCount) {
    const int t = threadIdx.x;
    // k_bitmap_prepare resets the two mask counters; the binning clears the mover count
    // the learned G2P's queue counters stay for a closure pass that runs beside this substep's
    // activation and binning (the learned G2P clears the queue before it fills it)
    if (t == kCtrStatus || t == kCtrMaskFrom || t == kCtrMaskBad || t == kCtrMovers || t == kCtrQueue ||
        t == kCtrQueueSubstep)
      return;
    if (t == kCtrUseMasks) {
      s.ctr[t] = s.ctr[kCtrMaskBad] == 0 ? s.ctr[kCtrMaskFrom] : 0;
      return;
    }
    if (t == kCtrIncBin) {
      // the move masks are valid exactly when the last G2P listed every particle that left
      // its cell, so the binning can merge those into the last binning's order
      s.ctr[t] = (s.ctr[kCtrMaskBad] == 0 && s.ctr[kCtrMaskFrom] > 0) ? 1 : 0;
      return;
    }
    if (t == kCtrSubstep) {
      s.ctr[t] += 1;
      return;
    }
    int v = 0;
    if (t >= kCtrBoxLo && t < kCtrBoxLo + 3) v = 0x7fffffff;
    if (t >= kCtrBoxHi && t < kCtrBoxHi + 3) v = -0x7fffffff;
    s.ctr[t] = v;
  }
}

// ComputeSparsity (SparsityOp.hpp:58-86): one insert per distinct block key of a warp.
__global__ void __launch_bounds__(kThreads) k_insert_particle_blocks(scene_device s) {
  if (s.ctr[kCtrUseMasks] > 0) return;  // k_insert_moved_blocks inserts this substep's blocks
  const int lane = threadIdx.x & 31;
  const int n = s.prm.n;
  int3 lo = make_int3(0x7fffffff, 0x7fffffff, 0x7fffffff);
  int3 hi = make_int3(-0x7fffffff, -0x7fffffff, -0x7fffffff);
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int warps = grid_threads() >> 5;
  for (int base0 = warp_global * 32 * kPass; base0 < n; base0 += warps * 32 * kPass) {
    float4 xs[kPass];
    int sids[kPass];
#pragma unroll
    for (int u = 0; u < kPass; ++u) {
      const int i = base0 + u * 32 + lane;
      xs[u] = i < n ? s.cur.xm[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      sids[u] = (s.prm.batch && i < n) ? s.cur.sid[i] : 0;
    }
#pragma unroll
    for (int u = 0; u < kPass; ++u) {
      const int i = base0 + u * 32 + lane;
      uint64_t key = kEmptyKey - 1 - lane;  // distinct per lane when invalid
      int3 c, b = make_int3(0, 0, 0);
      bool valid = false;
      if (i < n) {
        if (particle_cell(s, sids[u], xs[u], c, b)) {
          key = pack_key(b.x, b.y, b.z);
          valid = true;
        } else {
          set_status(s.ctr, kStatusOutOfDomain);
        }
      }
      const unsigned peers = __match_any_sync(kFull, key);
      if (valid && lane == __ffs(peers) - 1) {
        table_insert(s, key, b, &s.ctr[kCtrParticleBlocks], 0);
        lo = make_int3(min(lo.x, b.x), min(lo.y, b.y), min(lo.z, b.z));
        hi = make_int3(max(hi.x, b.x), max(hi.y, b.y), max(hi.z, b.z));
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo.x = min(lo.x, __shfl_xor_sync(kFull, lo.x, o));
    lo.y = min(lo.y, __shfl_xor_sync(kFull, lo.y, o));
    lo.z = min(lo.z, __shfl_xor_sync(kFull, lo.z, o));
    hi.x = max(hi.x, __shfl_xor_sync(kFull, hi.x, o));
    hi.y = max(hi.y, __shfl_xor_sync(kFull, hi.y, o));
    hi.z = max(hi.z, __shfl_xor_sync(kFull, hi.z, o));
  }
  if (lane == 0 && lo.x != 0x7fffffff) {
    atomicMin(&s.ctr[kCtrBoxLo + 0], lo.x);
    atomicMin(&s.ctr[kCtrBoxLo + 1], lo.y);
    atomicMin(&s.ctr[kCtrBoxLo + 2], lo.z);
    atomicMax(&s.ctr[kCtrBoxHi + 0], hi.x);
    atomicMax(&s.ctr[kCtrBoxHi + 1], hi.y);
    atomicMax(&s.ctr[kCtrBoxHi + 2], hi.z);
  }
}

// ComputeSparsity from the move masks the last G2P wrote: the blocks the particles of each
// previous block ended in (the same set of keys as the particle pass finds, since G2P computes
// each particle's block from the position it stores).  Runs instead of the particle pass
// after a G2P in which no particle left its block's 3^3 neighbourhood.
__global__ void __launch_bounds__(kThreads) k_insert_moved_blocks(scene_device s) {
  const int nold = s.ctr[kCtrUseMasks];
  if (nold == 0) return;
  // the previous binning's block keys by their index then (k_assign_ranks renumbers blk_pk)
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nold; b += grid_threads()) s.old_pk[b] = s.blk_pk[b];
  int3 lo = make_int3(0x7fffffff, 0x7fffffff, 0x7fffffff);
  int3 hi = make_int3(-0x7fffffff, -0x7fffffff, -0x7fffffff);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nold * 27; t += grid_threads()) {
    const int b = t / 27, j = t % 27;
    if (!((s.bmask[b] >> j) & 1u)) continue;
    const int3 k = unpack_key(s.blk_pk[b]);
    const int3 nk = make_int3(k.x + j / 9 - 1, k.y + (j / 3) % 3 - 1, k.z + j % 3 - 1);
    table_insert(s, pack_key(nk.x, nk.y, nk.z), nk, &s.ctr[kCtrParticleBlocks], 0);
    lo = make_int3(min(lo.x, nk.x), min(lo.y, nk.y), min(lo.z, nk.z));
    hi = make_int3(max(hi.x, nk.x), max(hi.y, nk.y), max(hi.z, nk.z));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo.x = min(lo.x, __shfl_xor_sync(kFull, lo.x, o));
    lo.y = min(lo.y, __shfl_xor_sync(kFull, lo.y, o));
    lo.z = min(lo.z, __shfl_xor_sync(kFull, lo.z, o));
    hi.x = max(hi.x, __shfl_xor_sync(kFull, hi.x, o));
    hi.y = max(hi.y, __shfl_xor_sync(kFull, hi.y, o));
    hi.z = max(hi.z, __shfl_xor_sync(kFull, hi.z, o));
  }
  if ((threadIdx.x & 31) == 0 && lo.x != 0x7fffffff) {
    atomicMin(&s.ctr[kCtrBoxLo + 0], lo.x);
    atomicMin(&s.ctr[kCtrBoxLo + 1], lo.y);
    atomicMin(&s.ctr[kCtrBoxLo + 2], lo.z);
    atomicMax(&s.ctr[kCtrBoxHi + 0], hi.x);
    atomicMax(&s.ctr[kCtrBoxHi + 1], hi.y);
    atomicMax(&s.ctr[kCtrBoxHi + 2], hi.z);
  }
}

// EnlargeSparsity{lo=0, hi=2} (SparsityOp.hpp:88-112): the +{0,1}^3 neighbours of every
// particle block, so that the 3x3x3 stencil of every particle lands in active blocks.
__global__ void __launch_bounds__(kThreads) k_enlarge(scene_device s) {
  const int npb = min(s.ctr[kCtrParticleBlocks], s.prm.nb_cap);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npb * 7; t += grid_threads()) {
    const int i = t / 7, o = t % 7 + 1;
    const int3 k = unpack_key(s.ins_pk[i]);
    const int3 nk = make_int3(k.x + (o >> 2), k.y + ((o >> 1) & 1), k.z + (o & 1));
    table_insert(s, pack_key(nk.x, nk.y, nk.z), nk, &s.ctr[kCtrEnlarged], npb);
  }
}

// Total block count, capacity checks and the dense bounding box of the bitmap that ranks
// the blocks in ascending (bx, by, bz) order.
__global__ void k_bitmap_prepare(scene_device s) {
  if (threadIdx.x != 0) return;
  s.ctr[kCtrMaskFrom] = 0;  // the masks are spent: the ranks below renumber the blocks
  s.ctr[kCtrMaskBad] = 0;
  int nb = s.ctr[kCtrParticleBlocks] + s.ctr[kCtrEnlarged];
  // HashTable.hpp:369 flags an insertion index >= T - 20, i.e. more than T - 20 blocks
  if (nb > s.prm.table_size - 20) set_status(s.ctr, kStatusTableFull);
  if (nb > s.prm.nb_cap) {
    set_status(s.ctr, kStatusCapacity);
    nb = s.prm.nb_cap;
  }
  s.ctr[kCtrBlocks] = nb;
  *s.view_cnt = nb;
  int words = 0;
  if (nb > 0) {
    const long long ex = (long long)s.ctr[kCtrBoxHi + 0] - s.ctr[kCtrBoxLo + 0] + 2;
    const long long ey = (long long)s.ctr[kCtrBoxHi + 1] - s.ctr[kCtrBoxLo + 1] + 2;
    const long long ez = (long long)s.ctr[kCtrBoxHi + 2] - s.ctr[kCtrBoxLo + 2] + 2;
    const long long vol = ex * ey * ez;
    const long long w = (vol + 31) / 32;
    if (w > s.prm.bitmap_cap) {
      set_status(s.ctr, kStatusBitmap);
      s.ctr[kCtrBlocks] = 0;
      *s.view_cnt = 0;
    } else {
      words = (int)w;
    }
  }
  s.ctr[kCtrWords] = words;
}

__device__ __forceinline__ long long dense_id(const scene_device &s, int3 k) {
  const long long ey = (long long)s.ctr[kCtrBoxHi + 1] - s.ctr[kCtrBoxLo + 1] + 2;
  const long long ez = (long long)s.ctr[kCtrBoxHi + 2] - s.ctr[kCtrBoxLo + 2] + 2;
  return (((long long)k.x - s.ctr[kCtrBoxLo + 0]) * ey + ((long long)k.y - s.ctr[kCtrBoxLo + 1])) * ez +
         ((long long)k.z - s.ctr[kCtrBoxLo + 2]);
}

__global__ void __launch_bounds__(kThreads) k_bitmap_set(scene_device s) {
  const int nb = s.ctr[kCtrWords] > 0 ? s.ctr[kCtrBlocks] : 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += grid_threads()) {
    const long long d = dense_id(s, unpack_key(s.ins_pk[i]));
    atomicOr(&s.bitmap[d >> 5], 1u << (d & 31));
  }
}

// rank = number of active keys below this one; index == rank from here on
__global__ void __launch_bounds__(kThreads) k_assign_ranks(scene_device s) {
  const int nb = s.ctr[kCtrWords] > 0 ? s.ctr[kCtrBlocks] : 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += grid_threads()) {
    const uint64_t key = s.ins_pk[i];
    const int3 k = unpack_key(key);
    const long long d = dense_id(s, k);
    const uint32_t w = s.bitmap[d >> 5];
    const int rank = s.word_prefix[d >> 5] + __popc(w & ((1u << (d & 31)) - 1u));
    s.tidx[s.ins_slot[i]] = rank;
    s.blk_pk[rank] = key;
    s.active_keys[3 * rank + 0] = k.x;
    s.active_keys[3 * rank + 1] = k.y;
    s.active_keys[3 * rank + 2] = k.z;
  }
}

// neighbour table b + {0,1}^3 (index dx*4 + dy*2 + dz); clears the bitmap for next time
__global__ void __launch_bounds__(kThreads) k_neighbors(scene_device s) {
  const int nb = s.ctr[kCtrBlocks];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nb * 8; t += grid_threads()) {
    const int b = t >> 3, o = t & 7;
    const int3 k = unpack_key(s.blk_pk[b]);
    const int3 nk = make_int3(k.x + (o >> 2), k.y + ((o >> 1) & 1), k.z + (o & 1));
    s.nbr[t] = table_query(s, pack_key(nk.x, nk.y, nk.z), nk);
  }
  const int words = s.ctr[kCtrWords];
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += grid_threads()) s.bitmap[w] = 0u;
}

// ----------------------------------------------------------------- binning
// Per particle: its block index and stencil-origin cell; counts per cell (rank within the
// cell from the atomic) and per block (warp-aggregated).
__device__ __forceinline__ bool incremental_binning(const scene_device &s) {
  return s.ctr[kCtrIncBin] != 0 && !s.prm.bin_full;
}

__global__ void __launch_bounds__(kThreads) k_bin_count(scene_device s) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    s.ctr[kCtrOrderFront] = 0;  // k_cell_start fills work_order
    s.ctr[kCtrOrderBack] = 0;
    // the persistent kernels of this binning and of the transfers after it start from their
    // first block (a second binning after one activation must not find them spent)
    s.ctr[kCtrWork + kWorkCellStart] = 0;
    s.ctr[kCtrWork + kWorkFinalize] = 0;
    s.ctr[kCtrWork + kWorkP2G] = 0;
    s.ctr[kCtrWork + kWorkG2P] = 0;
    s.ctr[kCtrDirty] = 0;
  }
  if (incremental_binning(s)) return;  // k_inc_stayers and k_inc_movers count this substep
  const int lane = threadIdx.x & 31;
  const int n = s.prm.n;
  const int nb = s.ctr[kCtrBlocks];
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int warps = grid_threads() >> 5;
  for (int base0 = warp_global * 32 * kPass; base0 < n; base0 += warps * 32 * kPass) {
   float4 xs[kPass];
   int sids[kPass];
#pragma unroll
   for (int u = 0; u < kPass; ++u) {
     const int i = base0 + u * 32 + lane;
     xs[u] = i < n ? s.cur.xm[i] : make_float4(0.f, 0.f, 0.f, 0.f);
     sids[u] = (s.prm.batch && i < n) ? s.cur.sid[i] : 0;
   }
#pragma unroll
   for (int u = 0; u < kPass; ++u) {
    const int i = base0 + u * 32 + lane;
    uint64_t key = kEmptyKey - 1 - lane;
    int3 c = make_int3(0, 0, 0), b = make_int3(0, 0, 0);
    bool valid = false;
    if (i < n && particle_cell(s, sids[u], xs[u], c, b)) {
      key = pack_key(b.x, b.y, b.z);
      valid = true;
    }
    const unsigned peers = __match_any_sync(kFull, key);
    const int leader = __ffs(peers) - 1;
    int blk = -1;
    if (valid && lane == leader) blk = table_query(s, key, b);
    blk = __shfl_sync(kFull, blk, leader);
    if (valid && (blk < 0 || blk >= nb)) set_status(s.ctr, kStatusMissingBlock);
    const bool ok = valid && blk >= 0 && blk < nb;
    // block counts, one atomic per distinct block of the warp
    const unsigned bpeers = __match_any_sync(kFull, ok ? blk : -1 - lane);
    if (ok && lane == __ffs(bpeers) - 1) atomicAdd(&s.block_count[blk], __popc(bpeers));
    // cell counts, one atomic per distinct cell of the warp (particles arrive in the previous
    // binning's order, so a warp spans a few cells); ranks within the warp follow lane order
    const int cell = ((c.x - 8 * b.x) << 6) | ((c.y - 8 * b.y) << 3) | (c.z - 8 * b.z);
    const uint32_t k32 = ok ? (uint32_t)blk * 512u + (uint32_t)cell : 0xffffffffu - (uint32_t)lane;
    const unsigned cpeers = __match_any_sync(kFull, k32);
    const int cleader = __ffs(cpeers) - 1;
    int cbase = 0;
    if (ok && lane == cleader) {
      cbase = atomicAdd(&s.cell_count[k32], __popc(cpeers));
      // cell counts share their word with the incremental binning's arrival count (high 16 bits)
      if (cbase + __popc(cpeers) > 0xffff) set_status(s.ctr, kStatusCapacity);
    }
    cbase = __shfl_sync(kFull, cbase, cleader);
    if (i < n) {
      s.key32[i] = ok ? k32 : 0xffffffffu;
      s.rnk[i] = ok ? cbase + __popc(cpeers & lanemask_lt()) : 0;
    }
   }
  }
}

// Persistent per-block CTA loop helper.
__device__ __forceinline__ int grab_block(int *counter, int *s_b) {
  __syncthreads();
  if (threadIdx.x == 0) *s_b = atomicAdd(counter, 1);
  __syncthreads();
  return *s_b;
}

// cell-major offsets of every cell's particle list
__global__ void __launch_bounds__(512) k_cell_start(scene_device s) {
  __shared__ int sm[512 / 32 + 1];
  __shared__ int s_b;
  const int nb = s.ctr[kCtrBlocks];
  for (;;) {
    const int b = grab_block(&s.ctr[kCtrWork + kWorkCellStart], &s_b);
    if (b >= nb) break;
    // low 16 bits: particles counted in place (every particle of a full binning, the stayers of
    // an incremental one); high 16 bits: the incremental binning's arrivals
    const int craw = s.cell_count[b * 512 + threadIdx.x];
    const int c = (craw & 0xffff) + (craw >> 16);
    int total;
    const int ex = cta_exclusive_scan<512>(c, total, sm);
    s.cell_start[b * 512 + threadIdx.x] = s.block_start[b] + ex;
    // the per-block kernels take the big blocks first, so that they end on small ones
    if (threadIdx.x == 0) {
      if (total >= kBigBlock)
        s.work_order[atomicAdd(&s.ctr[kCtrOrderFront], 1)] = b;
      else
        s.work_order[nb - 1 - atomicAdd(&s.ctr[kCtrOrderBack], 1)] = b;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_bin_scatter(scene_device s) {
  if (incremental_binning(s)) return;
  const int n = s.prm.n;
  const int stride = grid_threads();
  for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += kPass * stride) {
    uint32_t k[kPass];
    int r[kPass], cs[kPass];
#pragma unroll
    for (int u = 0; u < kPass; ++u) {
      const int i = i0 + u * stride;
      k[u] = i < n ? s.key32[i] : 0xffffffffu;
      r[u] = i < n ? s.rnk[i] : 0;
    }
#pragma unroll
    for (int u = 0; u < kPass; ++u) cs[u] = k[u] != 0xffffffffu ? s.cell_start[k[u]] : 0;
#pragma unroll
    for (int u = 0; u < kPass; ++u)
      if (k[u] != 0xffffffffu) s.tmp[cs[u] + r[u]] = i0 + u * stride;
  }
}

// Orders the list of one cell (indices into cur) by upload id, from `in` into `out` (which may
// be the same array).  Lists of up to 12 entries are sorted in registers (every index known at
// compile time): two rounds of independent loads (the list, then the ids), then an insertion
// sort of (id << 32 | index) entries; ids are unique, so this orders the cell by id.  Longer
// lists (strongly compressed cells) take an insertion sort in place in global memory.
__device__ __forceinline__ void sort_cell_by_id(const scene_device &s, const int *in, int *out, int cs, int c) {
  constexpr int kMaxList = 12;
  if (c <= kMaxList) {
    unsigned long long e[kMaxList];
#pragma unroll
    for (int r = 0; r < kMaxList; ++r) e[r] = r < c ? (unsigned long long)(uint32_t)in[cs + r] : ~0ull;
#pragma unroll
    for (int r = 0; r < kMaxList; ++r)
      if (r < c) e[r] |= (unsigned long long)(uint32_t)s.cur.id[(int)(uint32_t)e[r]] << 32;
#pragma unroll
    for (int r = 1; r < kMaxList; ++r)
      if (r < c) {
#pragma unroll
        for (int q = r; q > 0; --q) {
          const unsigned long long lo = e[q - 1], hi = e[q];
          const bool sw = lo > hi;
          e[q - 1] = sw ? hi : lo;
          e[q] = sw ? lo : hi;
        }
      }
#pragma unroll
    for (int r = 0; r < kMaxList; ++r)
      if (r < c) out[cs + r] = (int)(uint32_t)e[r];
  } else {
    int *w = const_cast<int *>(in);
    for (int r = 1; r < c; ++r) {
      const int i = w[cs + r];
      const int id = s.cur.id[i];
      int q = r;
      while (q > 0 && s.cur.id[w[cs + q - 1]] > id) {
        w[cs + q] = w[cs + q - 1];
        --q;
      }
      w[cs + q] = i;
    }
    if (out != in)
      for (int r = 0; r < c; ++r) out[cs + r] = w[cs + r];
  }
}

// Final particle order of a block (full binning): cells ascending, the particles of a cell in
// increasing upload index (a stable sort by (block, cell)).  Also zeroes the block's grid and
// the counts for the next substep.  The register sort caps the kernel at 3 CTAs of 512
// threads per SM (binning 0.71 -> 0.62 ms on the 30 M-particle sand scene against a sort in
// local memory at 4 CTAs).
__global__ void __launch_bounds__(512, 3) k_bin_finalize(scene_device s) {
  if (incremental_binning(s)) return;
  __shared__ int s_b;
  const int nb = s.ctr[kCtrBlocks];
  const int t = threadIdx.x;
  if (blockIdx.x == 0 && t == 0) {
    s.ctr[kCtrMovers] = 0;  // the next G2P lists its movers afresh
    s.ctr[kCtrBinInfo] = -1;
  }
  for (;;) {
    const int b = grab_block(&s.ctr[kCtrWork + kWorkFinalize], &s_b);
    if (b >= nb) break;
    const int c = s.cell_count[b * 512 + t];
    const int cs = s.cell_start[b * 512 + t];
    s.cell_count[b * 512 + t] = 0;
    sort_cell_by_id(s, s.tmp, s.src, cs, c);
    float4 *g = reinterpret_cast<float4 *>(s.grid + (size_t)b * kGridChannels * 512);
    g[t] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (t == 0) s.block_count[b] = 0;
  }
}

// ----------------------------------------------------------------- incremental binning
// After a G2P whose particles all stayed within their block's 3^3 neighbourhood, the particles
// are stored in the last binning's slot order, and G2P has flagged each slot whose particle
// left its cell (moved[]) and listed those slots (movers[]).  The particles that stayed
// (typically 98-99%) keep their relative order: it is already (cell, upload id) within their
// cell, and the block order is ascending keys both times.  So the new order is the stayers of
// every old cell, placed in order at the start of the same cell's new range, with the movers
// appended behind them and only the cells that received movers sorted again by id.  The result
// equals the full binning's order bit for bit.
//   k_inc_map            per old block: its index in the new activation
//   k_inc_stayers        per old cell: its stayers -> cell_count (low 16 bits) of the cell in
//                        the block's new index, and the block's total
//   k_inc_movers         per mover: its new cell, arrival rank (high 16 bits of cell_count)
//   (scan, k_cell_start) as in the full binning
//   k_inc_place_stayers  per old cell: src of its stayers
//   k_inc_place_movers   per mover: src behind the stayers of its cell
//   k_inc_sort           per cell that received movers: sorted by id
//   k_inc_finalize       per new cell: counts and grid zeroed

// the new index of every old block (one query per block, before the per-block passes)
__global__ void __launch_bounds__(kThreads) k_inc_map(scene_device s) {
  if (!incremental_binning(s)) return;
  const int nold = s.ctr[kCtrUseMasks];
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nold; b += grid_threads()) {
    const uint64_t key = s.old_pk[b];
    s.new_of_old[b] = table_query(s, key, unpack_key(key));
  }
}

// The stayers of one old cell j = b * 512 + c: its slot range in the previous binning and the
// number of its particles that did not move out (the flags of a cell are a few adjacent bytes)
__device__ __forceinline__ int2 prev_cell_range(const scene_device &s, int j) {
  const int b = j >> 9, c = j & 511;
  const int cs = s.cell_start_prev[j];
  const int ce = c < 511 ? s.cell_start_prev[j + 1] : s.block_start_prev[b + 1];
  return make_int2(cs, ce);
}

__global__ void __launch_bounds__(kThreads) k_inc_stayers(scene_device s) {
  if (!incremental_binning(s)) return;
  const int nold = s.ctr[kCtrUseMasks], nb = s.ctr[kCtrBlocks];
  const long long cells = (long long)nold * 512;  // a warp covers 32 cells of one block
  const int lane = threadIdx.x & 31;
  for (long long j0 = blockIdx.x * (long long)blockDim.x; j0 < cells; j0 += grid_threads()) {
    const long long j = j0 + threadIdx.x;
    const bool in = j < cells;
    int stay = 0, nbi = -1;
    if (in) {
      const int2 r = prev_cell_range(s, (int)j);
      int slot = r.x;
      for (; slot + 4 <= r.y; slot += 4) {
        const uint8_t a = s.moved[slot], b1 = s.moved[slot + 1], c = s.moved[slot + 2], d = s.moved[slot + 3];
        stay += (a == 0) + (b1 == 0) + (c == 0) + (d == 0);
      }
      for (; slot < r.y; ++slot) stay += s.moved[slot] == 0;
      nbi = s.new_of_old[(int)(j >> 9)];
      if (stay > 0xffff) set_status(s.ctr, kStatusCapacity);  // shares its word with the arrivals
      if (nbi >= 0 && nbi < nb)
        s.cell_count[nbi * 512 + (int)(j & 511)] = stay;
      else if (stay > 0)
        set_status(s.ctr, kStatusMissingBlock);
    }
    const int wsum = __reduce_add_sync(kFull, stay);
    if (lane == 0 && wsum > 0 && nbi >= 0 && nbi < nb) atomicAdd(&s.block_count[nbi], wsum);
  }
}

__global__ void __launch_bounds__(kThreads) k_inc_movers(scene_device s) {
  if (!incremental_binning(s)) return;
  const int nmov = min(s.ctr[kCtrMovers], s.prm.mover_cap);
  const int nb = s.ctr[kCtrBlocks];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nmov; k += grid_threads()) {
    const int slot = s.movers[k];
    int3 c, b;
    int2 pos = make_int2(-1, 0);
    if (particle_cell(s, s.prm.batch ? s.cur.sid[slot] : 0, s.cur.xm[slot], c, b)) {
      const int blk = table_query(s, pack_key(b.x, b.y, b.z), b);
      if (blk >= 0 && blk < nb) {
        const int k32 = blk * 512 + (((c.x - 8 * b.x) << 6) | ((c.y - 8 * b.y) << 3) | (c.z - 8 * b.z));
        const int old = atomicAdd(&s.cell_count[k32], 1 << 16);
        atomicAdd(&s.block_count[blk], 1);
        pos = make_int2(k32, old >> 16);
        if ((old >> 16) >= 0x7fff) set_status(s.ctr, kStatusCapacity);
        // the first arrival lists the cell for k_inc_sort (at most one entry per mover)
        if ((old >> 16) == 0) s.dirty[atomicAdd(&s.ctr[kCtrDirty], 1)] = k32;
      }
    }
    if (pos.x < 0) set_status(s.ctr, kStatusMissingBlock);
    s.mover_pos[k] = pos;
  }
}

__global__ void __launch_bounds__(kThreads) k_inc_place_stayers(scene_device s) {
  if (!incremental_binning(s)) return;
  const int nold = s.ctr[kCtrUseMasks], nb = s.ctr[kCtrBlocks];
  const long long cells = (long long)nold * 512;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < cells; j += grid_threads()) {
    const int nbi = s.new_of_old[(int)(j >> 9)];
    if (nbi < 0 || nbi >= nb) continue;
    const int2 r = prev_cell_range(s, (int)j);
    int dst = s.cell_start[nbi * 512 + (int)(j & 511)];
    // four flags loaded together per round (a cell holds a few adjacent slots)
    for (int slot = r.x; slot < r.y; slot += 4) {
      uint8_t f[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) f[u] = slot + u < r.y ? s.moved[slot + u] : (uint8_t)1;
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (f[u] == 0) s.src[dst++] = slot + u;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_inc_place_movers(scene_device s) {
  if (!incremental_binning(s)) return;
  const int nmov = min(s.ctr[kCtrMovers], s.prm.mover_cap);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nmov; k += grid_threads()) {
    const int2 pos = s.mover_pos[k];
    if (pos.x < 0) continue;
    s.src[s.cell_start[pos.x] + (s.cell_count[pos.x] & 0xffff) + pos.y] = s.movers[k];
  }
}

// the cells that received movers, in upload-id order (stayers and arrivals merged)
__global__ void __launch_bounds__(kThreads) k_inc_sort(scene_device s) {
  if (!incremental_binning(s)) return;
  const int nd = min(s.ctr[kCtrDirty], s.prm.mover_cap);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nd; k += grid_threads()) {
    const int j = s.dirty[k];
    const int craw = s.cell_count[j];
    const int c = (craw & 0xffff) + (craw >> 16);
    if (c > 1) sort_cell_by_id(s, s.src, s.src, s.cell_start[j], c);
  }
}

__global__ void __launch_bounds__(kThreads) k_inc_finalize(scene_device s) {
  if (!incremental_binning(s)) return;
  const int nb = s.ctr[kCtrBlocks];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    s.ctr[kCtrBinInfo] = min(s.ctr[kCtrMovers], s.prm.mover_cap);
    s.ctr[kCtrMovers] = 0;  // the next G2P lists its movers afresh (k_inc_place_movers has read them)
  }
  const long long cells = (long long)nb * 512;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < cells; j += grid_threads()) {
    s.cell_count[j] = 0;
    const int b = (int)(j >> 9), cell = (int)(j & 511);
#pragma unroll
    for (int ch = 0; ch < kGridChannels; ++ch) s.grid[((size_t)b * kGridChannels + ch) * 512 + cell] = 0.f;
    if (cell == 0) s.block_count[b] = 0;
  }
}

// ----------------------------------------------------------------- P2G
// One CTA per block (persistent).  The block's 512 cells are processed in chunks of 64:
//  1. the CTA gathers the chunk's particles, two per thread with their loads issued together,
//     and stages, per particle, its 3x3 B-spline weights, m and the affine terms (q, A dx) in
//     shared memory as six float4 fields laid out [field][rank][cell], rows padded by one
//     float4: lanes reading one rank of consecutive cells read 512 contiguous bytes, and the
//     ranks of one cell, which consecutive lanes write, start 4 banks apart;
//  2. one thread per (cell, channel) sums the cell's particles into 27 registers -- all
//     particles of a cell share the same 27 stencil nodes -- and adds them to a halo of the
//     grid in shared memory.
// Ranks are staged R at a time: a chunk with a cell of more particles runs phases 1-2 again for
// the next ranks (a round), so that no particle needs the slow per-node path for lack of
// staging room and the staging stays small enough for several CTAs per SM.
// The halo holds the nodes the block's particles reach: a particle binned in cell c of the
// block has its stencil origin at c + 1 (SparsityOp.hpp:72-77 against P2G.hpp:62-66), so its
// nodes lie in [8b + 1, 8b + 11) per axis; the halo spans exactly that in x and y and
// [8b, 8b + 12) in z, so that the flush moves whole 16-byte quads of the neighbour blocks.
// Grid channels: m and p = sum W (m v + A (x_i - x_p)), the reference's mv + rhs
// (P2G.hpp:108-125) with A = m C - (4 dt/dx^2) tau precomputed by G2P.
// The staging depth is a tile choice of the autotuner: R particles per cell are staged per
// round, with the register budget cut for the CTAs per SM that R's shared memory allows --
// 8 ranks (55 KB) for 4 CTAs per SM, 12 (72 KB, the default) for 3, 16 (88 KB) for 2.
// ZSMPM_P2G_STAGE_F = 1 (compile-time) stages the particle's fractional position in the cell
// instead of its nine weights (phase 2 recomputes them: more arithmetic, a third less shared
// memory).
#ifndef ZSMPM_P2G_STAGE_F
#define ZSMPM_P2G_STAGE_F 1
#endif
constexpr int kP2GChunk = 64;     // cells per chunk
constexpr int kP2GRanksDefault = 12;  // particles per cell staged per round, unless tuned
constexpr bool kP2GStageF = ZSMPM_P2G_STAGE_F != 0;
constexpr int kP2GRow = kP2GChunk + 1;  // padded row of float4: rank r of cell c at bank 4 (r + c) % 32
constexpr int kP2GThreads = 256;  // 4 channels x 64 cells
constexpr int kP2GMap = 1024;     // slots of a chunk mapped to their cell (more: binary search)
constexpr int kP2GHx = 10, kP2GHy = 10, kP2GHz = 12;  // halo extents (x, y from 8b + 1; z from 8b)
constexpr int kP2GHaloNodes = kP2GHx * kP2GHy * kP2GHz;

struct p2g_particle {
  float m, w[3][3], f[3], q[3], ax[3], ay[3], az[3];
  int hb[3];  // stencil origin relative to the block's first cell 8b (1..8 when binned in it)
};

// quadratic B-spline weights of the nodes 0, 1, 2 of a stencil at fractional position f
// (InterpolationKernel.hpp:93-130)
__device__ __forceinline__ void bspline_weights(float f, float *w) {
  w[0] = 0.5f * (1.5f - f) * (1.5f - f);
  const float f1 = f - 1.f;
  w[1] = 0.75f - f1 * f1;
  const float f2 = 0.5f + f1;
  w[2] = 0.5f * f2 * f2;
}

// The node weights of the cell-centric pair (P2C2GTransfer): a particle's tent weights to the
// centers of its two cells per axis, 1/2 - fx and 1/2 + fx with fx = x/dx - floor(x/dx + 1/2),
// each passed half to either corner, over the nodes base .. base + 2 (base = floor(x/dx + 1/2)
// - 1, f = x/dx - base = fx + 1).
__device__ __forceinline__ void cell_weights(float f, float *w) {
  w[0] = 0.75f - 0.5f * f;
  w[1] = 0.5f;
  w[2] = 0.5f * f - 0.25f;
}

struct p2g_raw {
  float4 xm, v;
  float A[9];
};

__device__ __forceinline__ void p2g_load(const scene_device &s, const float *affine, int i, p2g_raw &r) {
  r.xm = s.cur.xm[i];
  r.v = s.cur.v[i];
#pragma unroll
  for (int k = 0; k < 9; ++k) r.A[k] = affine[mat_at(k, i)];
}

// kCell: the cell-centric pair's weights and stencil origin; with_mass = false leaves the mass
// and the m v term out (P2C2GTransferForce)
template <bool kCell>
__device__ __forceinline__ void p2g_prepare(const scene_params &p, const p2g_raw &r, int ox, int oy, int oz,
                                            p2g_particle &pp, bool with_mass) {
  // APIC: x / dx as P2G.hpp:62 divides (a multiplication when dx is a power of two, the same
  // number).  The cell pair: the index bucket floor(x * (1/dx) + 1/2) as the binning keys it.
  float X[3];
  if (kCell) {
    X[0] = r.xm.x * p.inv_dx, X[1] = r.xm.y * p.inv_dx, X[2] = r.xm.z * p.inv_dx;
  } else {
    X[0] = over_dx(p, r.xm.x), X[1] = over_dx(p, r.xm.y), X[2] = over_dx(p, r.xm.z);
  }
  float lp[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float base = kCell ? floorf(X[d] + 0.5f) - 1.f : floorf(X[d] - 0.5f);
    const float f = X[d] - base;
    pp.hb[d] = (int)base - (d == 0 ? ox : d == 1 ? oy : oz);
    pp.f[d] = f;
    if (kCell)
      cell_weights(f, pp.w[d]);
    else
      bspline_weights(f, pp.w[d]);
    lp[d] = f * p.dx;
  }
  pp.m = with_mass ? r.xm.w : 0.f;
  const float vel[3] = {r.v.x, r.v.y, r.v.z};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    pp.q[d] = pp.m * vel[d] - (r.A[d] * lp[0] + r.A[3 + d] * lp[1] + r.A[6 + d] * lp[2]);
    pp.ax[d] = r.A[d] * p.dx;
    pp.ay[d] = r.A[3 + d] * p.dx;
    pp.az[d] = r.A[6 + d] * p.dx;
  }
}

// Every node of one particle by itself: shared atomics into the halo when its stencil lies in
// it, else global atomics into the grid blocks b + {0,1}^3 (a stencil origin that rounding
// put one cell off the binned cell, possible when dx is not a power of two).
__device__ __forceinline__ void p2g_direct(const scene_device &s, float *sh, const p2g_particle &pp, int b) {
  const int hx = pp.hb[0] - 1, hy = pp.hb[1] - 1, hz = pp.hb[2];
  const bool in_halo = hx >= 0 && hx <= kP2GHx - 3 && hy >= 0 && hy <= kP2GHy - 3 && hz >= 0 && hz <= kP2GHz - 3;
  const bool in_reach = pp.hb[0] >= 0 && pp.hb[0] <= 13 && pp.hb[1] >= 0 && pp.hb[1] <= 13 && pp.hb[2] >= 0 &&
                        pp.hb[2] <= 13;
  if (!in_halo && !in_reach) {
    set_status(s.ctr, kStatusMissingBlock);
    return;
  }
  for (int ii = 0; ii < 3; ++ii)
    for (int jj = 0; jj < 3; ++jj)
      for (int kk = 0; kk < 3; ++kk) {
        const float W = pp.w[0][ii] * pp.w[1][jj] * pp.w[2][kk];
        float v[4];
        v[0] = W * pp.m;
#pragma unroll
        for (int d = 0; d < 3; ++d)
          v[1 + d] = W * (pp.q[d] + (float)ii * pp.ax[d] + (float)jj * pp.ay[d] + (float)kk * pp.az[d]);
        if (in_halo) {
          const int h = ((hx + ii) * kP2GHy + (hy + jj)) * kP2GHz + hz + kk;
#pragma unroll
          for (int c = 0; c < 4; ++c) atomicAdd(&sh[c * kP2GHaloNodes + h], v[c]);
        } else {
          const int X = pp.hb[0] + ii, Y = pp.hb[1] + jj, Z = pp.hb[2] + kk;  // cells from 8b
          if (X >= 16 || Y >= 16 || Z >= 16) {
            set_status(s.ctr, kStatusMissingBlock);
            continue;
          }
          const int tb = s.nbr[b * 8 + ((X >> 3) << 2) + ((Y >> 3) << 1) + (Z >> 3)];
          if (tb < 0) {
            set_status(s.ctr, kStatusMissingBlock);
            continue;
          }
          const int cell = ((X & 7) << 6) | ((Y & 7) << 3) | (Z & 7);
#pragma unroll
          for (int c = 0; c < 4; ++c) atomicAdd(&s.grid[((size_t)tb * kGridChannels + c) * 512 + cell], v[c]);
        }
      }
}

// float4 fields: w00 w01 w02 w10 | w11 w12 w20 w21 | w22 m | (q ax ay az) x 3, or with the
// fractional position: fx fy fz m | (q ax ay az) x 3
constexpr int kP2GVec = kP2GStageF ? 4 : 6;
constexpr int kP2GQ = kP2GVec - 3;  // first momentum field
constexpr size_t p2g_smem_bytes(int ranks) {
  return sizeof(float) * kGridChannels * kP2GHaloNodes + sizeof(float4) * kP2GVec * ranks * kP2GRow +
         sizeof(int) * 2 * (kP2GChunk + 1) + sizeof(int) * 4 + sizeof(unsigned char) * 2 * kP2GMap;
}

// the weights and the mass of staged rank r of cell cl
template <bool kCell, int R>
__device__ __forceinline__ void staged_weights(const float4 (*stg)[R][kP2GRow], int r, int cl, float (&w)[3][3],
                                               float &m) {
  if (kP2GStageF) {
    const float4 fm = stg[0][r][cl];
    if (kCell) {
      cell_weights(fm.x, w[0]);
      cell_weights(fm.y, w[1]);
      cell_weights(fm.z, w[2]);
    } else {
      bspline_weights(fm.x, w[0]);
      bspline_weights(fm.y, w[1]);
      bspline_weights(fm.z, w[2]);
    }
    m = fm.w;
  } else {
    const float4 wa = stg[0][r][cl], wb = stg[1][r][cl], wc = stg[2][r][cl];
    w[0][0] = wa.x, w[0][1] = wa.y, w[0][2] = wa.z;
    w[1][0] = wa.w, w[1][1] = wb.x, w[1][2] = wb.y;
    w[2][0] = wb.z, w[2][1] = wb.w, w[2][2] = wc.x;
    m = wc.y;
  }
}

// kCell: P2C2GTransfer of the cell-centric pair (below) with the pair's node weights and
// affine term; `affine` is the affine term (A = m C - (4 dt/dx^2) tau for APIC), with_mass = 0
// leaves the mass channel and the m v term out.  R staged ranks per round, registers cut for
// MinCtas CTAs per SM.
template <bool kCell, int R, int MinCtas>
__global__ void __launch_bounds__(kP2GThreads, MinCtas) k_p2g(scene_device s, const float *affine, int with_mass) {
  extern __shared__ __align__(16) float p2g_smem[];
  float *sh = p2g_smem;
  auto stg = reinterpret_cast<float4(*)[R][kP2GRow]>(p2g_smem + kGridChannels * kP2GHaloNodes);
  int *s_cs = reinterpret_cast<int *>(p2g_smem + kGridChannels * kP2GHaloNodes +
                                      4 * kP2GVec * R * kP2GRow);
  int *const s_wmax = s_cs + 2 * (kP2GChunk + 1);  // per chunk parity: the largest cell count of each half
  unsigned char *const s_map0 = reinterpret_cast<unsigned char *>(s_wmax + 4);
  __shared__ int s_b;
  const int nb = s.ctr[kCtrBlocks];
  const int t = threadIdx.x;
  const int my_cell = t & (kP2GChunk - 1), my_ch = t >> 6;
  // the halo starts zeroed; each block's flush zeroes the quads it sends, so the next block
  // finds it zeroed again (the first barrier of grab_block orders both)
  for (int q = t; q < kGridChannels * kP2GHaloNodes; q += blockDim.x) sh[q] = 0.f;
  for (;;) {
    const int w = grab_block(&s.ctr[kCtrWork + kWorkP2G], &s_b);
    if (w >= nb) break;
    const int b = s.work_order[w];
    const int start = s.block_start[b], end = s.block_start[b + 1];
    if (start == end) continue;
    const int3 bk = local_block(s.prm, unpack_key(s.blk_pk[b]));
    const int ox = bk.x * 8, oy = bk.y * 8, oz = bk.z * 8;
    int *const s_cs0 = s_cs;
    // cell starts of chunk k in s_cs0 + (k & 1) * (kP2GChunk + 1), its slot -> cell map in
    // s_map0 + (k & 1) * kP2GMap and its largest cell count in s_wmax[2 (k & 1) ..]; the next
    // chunk's are filled during this chunk's last phase 2, so a round needs two barriers
    auto fill = [&](int chunk_to_fill) {
      if (t <= kP2GChunk) {
        const int c = chunk_to_fill * kP2GChunk + t;
        s_cs0[(chunk_to_fill & 1) * (kP2GChunk + 1) + t] = c < 512 ? s.cell_start[b * 512 + c] : end;
      }
      if (t < kP2GChunk) {
        const int c = chunk_to_fill * kP2GChunk + t;
        const int cs = s.cell_start[b * 512 + c];
        const int ce = c + 1 < 512 ? s.cell_start[b * 512 + c + 1] : end;
        const int base = s.cell_start[b * 512 + chunk_to_fill * kP2GChunk];
        unsigned char *m = s_map0 + (chunk_to_fill & 1) * kP2GMap;
        for (int q = cs - base; q < ce - base && q < kP2GMap; ++q) m[q] = (unsigned char)t;
        const int wmax = __reduce_max_sync(kFull, ce - cs);
        if ((t & 31) == 0) s_wmax[2 * (chunk_to_fill & 1) + (t >> 5)] = wmax;
      }
    };
    fill(0);
    // the shallow (8-rank) staging, which the tuner picks for sparse cells: the slot-map entries
    // of this thread's first two slots of the next chunk are loaded during the current chunk's
    // last sums, so that the next phase 1 waits for one load instead of two (-1: not loaded).
    // At 8 ranks this measured 1.035 against 1.067 ms on the 16 M snow scene; at 12 ranks it
    // was slower.
    constexpr bool kPrefetchSrc = R == 8;
    int pre1 = -1, pre2 = -1;
    for (int chunk = 0; chunk < 512 / kP2GChunk; ++chunk) {
      const int cell0 = chunk * kP2GChunk;
      const int par = chunk & 1;
      int *s_cs = s_cs0 + par * (kP2GChunk + 1);
      const unsigned char *s_map = s_map0 + par * kP2GMap;
      for (int round = 0;; ++round) {
        __syncthreads();  // previous staging consumed, this chunk's starts loaded, halo zeroed
        const int maxc = max(s_wmax[2 * par], s_wmax[2 * par + 1]);
        const int rlo = round * R;
        const bool last = rlo + R >= maxc;
        // ---- phase 1: consecutive threads take consecutive slots (coalesced gathers); the
        // slots whose rank falls in this round's window are staged
        const int c0 = s_cs[0], c1 = s_cs[kP2GChunk];
        auto cell_of_slot = [&](int slot) {
          int lo = 0;  // the cell of this slot: the last cell whose start is <= slot
          if (slot - c0 < kP2GMap) {
            lo = s_map[slot - c0];
          } else {
            int hi = kP2GChunk;
            while (hi - lo > 1) {
              const int mid = (lo + hi) >> 1;
              if (s_cs[mid] <= slot) lo = mid;
              else hi = mid;
            }
          }
          return lo;
        };
        auto stage_one = [&](int cl, int r, const p2g_particle &pp) {
          const int cell = cell0 + cl;
          const int ex = (cell >> 6) + 1, ey = ((cell >> 3) & 7) + 1, ez = (cell & 7) + 1;
          if (pp.hb[0] != ex || pp.hb[1] != ey || pp.hb[2] != ez) {
            // a stencil origin that rounding moved off the cell: this particle by itself, and a
            // zero-mass stand-in in its staging place
            p2g_direct(s, sh, pp, b);
            for (int f = 0; f < kP2GVec; ++f) stg[f][r][cl] = make_float4(0.f, 0.f, 0.f, 0.f);
            return;
          }
          if (kP2GStageF) {
            stg[0][r][cl] = make_float4(pp.f[0], pp.f[1], pp.f[2], pp.m);
          } else {
            stg[0][r][cl] = make_float4(pp.w[0][0], pp.w[0][1], pp.w[0][2], pp.w[1][0]);
            stg[1][r][cl] = make_float4(pp.w[1][1], pp.w[1][2], pp.w[2][0], pp.w[2][1]);
            stg[2][r][cl] = make_float4(pp.w[2][2], pp.m, 0.f, 0.f);
          }
#pragma unroll
          for (int d = 0; d < 3; ++d)
            stg[kP2GQ + d][r][cl] = make_float4(pp.q[d], pp.ax[d], pp.ay[d], pp.az[d]);
        };
        for (int slot = c0 + t; slot < c1; slot += 2 * blockDim.x) {
          const int slot2 = slot + blockDim.x;
          const int cl1 = cell_of_slot(slot), r1 = slot - s_cs[cl1] - rlo;
          const bool in1 = r1 >= 0 && r1 < R;
          int cl2 = 0, r2 = -1;
          if (slot2 < c1) {
            cl2 = cell_of_slot(slot2);
            r2 = slot2 - s_cs[cl2] - rlo;
          }
          const bool in2 = r2 >= 0 && r2 < R;
          if (!in1 && !in2) continue;
          p2g_raw ra, rb;
          if (kPrefetchSrc) {
            int src1, src2;
            if (round == 0 && slot == c0 + t && pre1 >= 0) {
              src1 = pre1;
              src2 = slot2 < c1 ? pre2 : pre1;
            } else {
              src1 = s.src[slot];
              src2 = slot2 < c1 ? s.src[slot2] : src1;
            }
            p2g_load(s, affine, in1 ? src1 : src2, ra);
            p2g_load(s, affine, in2 ? src2 : src1, rb);
          } else {
            p2g_load(s, affine, s.src[in1 ? slot : slot2], ra);
            p2g_load(s, affine, s.src[in2 ? slot2 : slot], rb);
          }
          p2g_particle pp;
          if (in1) {
            p2g_prepare<kCell>(s.prm, ra, ox, oy, oz, pp, with_mass != 0);
            stage_one(cl1, r1, pp);
          }
          if (in2) {
            p2g_prepare<kCell>(s.prm, rb, ox, oy, oz, pp, with_mass != 0);
            stage_one(cl2, r2, pp);
          }
        }
        __syncthreads();
        if (last && chunk + 1 < 512 / kP2GChunk) fill(chunk + 1);
        if (kPrefetchSrc) {
          pre1 = pre2 = -1;
          if (last && chunk + 1 < 512 / kP2GChunk) {
            const int c0n = s.cell_start[b * 512 + (chunk + 1) * kP2GChunk];
            const int c1n = chunk + 2 < 512 / kP2GChunk ? s.cell_start[b * 512 + (chunk + 2) * kP2GChunk] : end;
            if (c0n + t < c1n) pre1 = s.src[c0n + t];
            if (c0n + t + (int)blockDim.x < c1n) pre2 = s.src[c0n + t + blockDim.x];
          }
        }
        // ---- phase 2: thread (cell, channel) sums the staged particles of its cell
        const int cnt = min(s_cs[my_cell + 1] - s_cs[my_cell] - rlo, R);
        if (cnt > 0) {
          float acc[27];
#pragma unroll
          for (int n = 0; n < 27; ++n) acc[n] = 0.f;
          const int d = my_ch - 1;  // p channel index, -1 for mass
          if (my_ch == 0) {
            // mass: W m (the warp is channel-uniform)
            for (int r = 0; r < cnt; ++r) {
              float w[3][3], m;
              staged_weights<kCell, R>(stg, r, my_cell, w, m);
#pragma unroll
              for (int ii = 0; ii < 3; ++ii) {
                const float wm = w[0][ii] * m;
#pragma unroll
                for (int jj = 0; jj < 3; ++jj) {
                  const float wij = wm * w[1][jj];
#pragma unroll
                  for (int kk = 0; kk < 3; ++kk) {
                    const int n = (ii * 3 + jj) * 3 + kk;
                    acc[n] = fmaf(wij, w[2][kk], acc[n]);
                  }
                }
              }
            }
          } else {
            // momentum: W (q + ii ax + jj ay + kk az), in cell units of the node offset
            for (int r = 0; r < cnt; ++r) {
              float w[3][3], m_unused;
              staged_weights<kCell, R>(stg, r, my_cell, w, m_unused);
              const float4 qa = stg[kP2GQ + d][r][my_cell];
              const float q = qa.x, ax = qa.y, ay = qa.z, az = qa.w;
              // wz (qij + kk az) = wz qij + cz[kk], cz = (0, wz1 az, 2 wz2 az): two operations
              // per node
              const float cz1 = w[2][1] * az, cz2 = 2.f * w[2][2] * az;
#pragma unroll
              for (int ii = 0; ii < 3; ++ii) {
                const float qi = q + (float)ii * ax;
#pragma unroll
                for (int jj = 0; jj < 3; ++jj) {
                  const float qij = qi + (float)jj * ay;
                  const float wij = w[0][ii] * w[1][jj];
                  const int n = (ii * 3 + jj) * 3;
                  acc[n] = fmaf(wij, w[2][0] * qij, acc[n]);
                  acc[n + 1] = fmaf(wij, fmaf(w[2][1], qij, cz1), acc[n + 1]);
                  acc[n + 2] = fmaf(wij, fmaf(w[2][2], qij, cz2), acc[n + 2]);
                }
              }
            }
          }
          // cell (lx, ly, lz): stencil origin (lx + 1, ly + 1, lz + 1) from 8b, halo node
          // (lx, ly, lz + 1)
          const int cell = cell0 + my_cell;
          const int hx = cell >> 6, hy = (cell >> 3) & 7, hz = (cell & 7) + 1;
          float *dst = sh + my_ch * kP2GHaloNodes;
#pragma unroll
          for (int ii = 0; ii < 3; ++ii)
#pragma unroll
            for (int jj = 0; jj < 3; ++jj)
#pragma unroll
              for (int kk = 0; kk < 3; ++kk)
                atomicAdd(&dst[((hx + ii) * kP2GHy + (hy + jj)) * kP2GHz + hz + kk], acc[(ii * 3 + jj) * 3 + kk]);
        }
        if (last) break;
      }
    }
    __syncthreads();
    // flush: items (ch, hx, hy, quad) over 4 x 10 x 10 x 3; halo node (hx, hy, 4 quad + j) is
    // the grid cell (8b + 1 + hx, 8b + 1 + hy, 8b + 4 quad + j)
    for (int it = t; it < kGridChannels * kP2GHx * kP2GHy * 3; it += blockDim.x) {
      const int quad = it % 3, hy = (it / 3) % kP2GHy, hx = (it / (3 * kP2GHy)) % kP2GHx,
                ch = it / (3 * kP2GHy * kP2GHx);
      float4 *src4 = reinterpret_cast<float4 *>(&sh[((ch * kP2GHx + hx) * kP2GHy + hy) * kP2GHz + quad * 4]);
      const float4 q4 = *src4;
      if (q4.x == 0.f && q4.y == 0.f && q4.z == 0.f && q4.w == 0.f) continue;
      *src4 = make_float4(0.f, 0.f, 0.f, 0.f);
      const int X = hx + 1, Y = hy + 1;
      const int tt = (X >= 8 ? 4 : 0) | (Y >= 8 ? 2 : 0) | (quad == 2 ? 1 : 0);
      const int tb = s.nbr[b * 8 + tt];
      if (tb < 0) {
        set_status(s.ctr, kStatusMissingBlock);
        continue;
      }
      const int cell = ((X & 7) << 6) | ((Y & 7) << 3) | ((quad * 4) & 7);
      red_add_v4(s.grid + ((size_t)tb * kGridChannels + ch) * 512 + cell, q4.x, q4.y, q4.z, q4.w);
    }
  }
}

// ----------------------------------------------------------------- the cell-centric pair
// P2C2GTransfer (simulation/transfer/P2C2G.hpp:27-189) and G2C2PTransfer with its Pre and Post
// passes (G2C2P.hpp:36-278), the fixed-corotated branch.  Both go through the grid cells: the
// particles within dx of a cell's center x_c (per axis) carry the tent weight
// W = prod (1 - |x_c - x_p| / dx), and a cell passes its sums to its 8 corner nodes (and takes
// its velocity from them) with weight 1/8.  A particle's cells are those of the index buckets
// floor(x / dx + 0.5) in {c, c + 1}^3 around it.  The cells are linear stages between the
// particles and the nodes, so each node receives sum_p w_p (m v + A (x_i - x_p)) with the
// composed node weights of cell_weights, and each particle takes sum_i w_i v_i: P2C2G runs as
// the staged P2G kernel with those weights (k_p2g<true>) and G2C2P as a variant of the G2P
// kernel (k_g2p<..., true>), both without per-particle atomics.  (A literal cell-gather P2C2G,
// one thread per cell walking its 8 buckets, measured 5.1 ms against 1.5 ms for P2G on 30 M
// particles: its loads are dependent and scattered.)
//
// Per particle the pair carries x, m, v, F and B (the reference's C attribute) and, written at
// the end of G2C2P for the next P2C2G, the affine term
//   A = (m B - dt V0 P(F) F^T) Dinv,   Dinv_k = 2 / (dx^2 - 2 r_k^2),  r = x - dx round(x / dx),
// columns k scaled (P2C2G.hpp:86-146); it is the same array the APIC path keeps its affine
// momentum in.

// Dinv of one position component, as P2C2G.hpp:87-91 and PostG2C2PTransfer compute it
__device__ __forceinline__ float cell_dinv(const scene_params &p, float x) {
  const float r = x - floorf(x * p.inv_dx + 0.5f) * p.dx;
  return 2.f / (p.dx * p.dx - 2.f * r * r);
}

// The pair's per-particle affine term A of the stored state, in the particle order of cur:
// part 0 the whole term (P2C2GTransfer; the cell-scheme counterpart of k_prime), 1 the momentum
// part m B Dinv (P2C2GTransferMomentum), 2 the force part -dt V0 P F^T Dinv (P2C2GTransferForce).
__global__ void __launch_bounds__(kThreads) k_cell_affine(scene_device s, int part, float *out) {
  if (part == 0 && blockIdx.x == 0 && threadIdx.x == 0) s.ctr[kCtrMaskFrom] = 0;
  const scene_params &p = s.prm;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += grid_threads()) {
    const float4 xm = s.cur.xm[i];
    const float dinv[3] = {cell_dinv(p, xm.x), cell_dinv(p, xm.y), cell_dinv(p, xm.z)};
    float F[9], tau[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = s.cur.F[mat_at(k, i)];
    float pl = 0.f;
    if (part != 1) constitutive(p.mat, F, pl, tau);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const float mB = part == 2 ? 0.f : xm.w * s.cur.C[mat_at(k, i)];
      const float f = part == 1 ? 0.f : p.dt * tau[k];
      out[mat_at(k, i)] = (mB - f) * dinv[k / 3];
    }
  }
}

// ----------------------------------------------------------------- grid update
// ComputeGridBlockVelocity with the rhs term (v = (mv + rhs)/m + g dt; GridOp.hpp:93-99
// restated) and ApplyBoundaryConditionOnGridBlocks with six planes wall_cells*dx inside
// the unit box (GridOp.hpp:136-161, Collider.h:98-105).
__device__ __forceinline__ void apply_walls(const scene_params &p, const float pos[3], float v[3]) {
  if (p.wall_type == 3) return;
  const float lo = (float)p.wall_cells * p.dx, hi = 1.f - (float)p.wall_cells * p.dx;
#pragma unroll
  for (int w = 0; w < 6; ++w) {
    const int axis = w >> 1;
    const float sgn = (w & 1) ? -1.f : 1.f;
    const float sd = sgn * (pos[axis] - ((w & 1) ? hi : lo));
    if (!(sd < 0.f)) continue;
    if (p.wall_type == 0) {
      v[0] = v[1] = v[2] = 0.f;
    } else {
      const float proj = sgn * v[axis];
      if (p.wall_type == 1 || proj < 0.f) v[axis] = v[axis] - proj * sgn;
    }
  }
}

// the scene's colliders after its walls, then its sparse level sets, each in list order
__device__ __forceinline__ void apply_colliders(const scene_params &p, int count, int nls, const float pos[3],
                                             float v[3]) {
  for (int k = 0; k < count; ++k) collider_resolve(p.colliders[k], pos, v);
  for (int k = 0; k < nls; ++k) levelset_resolve(p.levelsets[k], pos, v);
}

__global__ void __launch_bounds__(kThreads) k_grid_update(scene_device s) {
  const scene_params &p = s.prm;
  const int nb = s.ctr[kCtrBlocks];
  const long long total = (long long)nb * 512;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += grid_threads()) {
    const int b = (int)(t >> 9), cell = (int)(t & 511);
    float *g = s.grid + (size_t)b * kGridChannels * 512 + cell;
    const float m = g[0];
    if (m == 0.f) continue;
    const float inv = 1.f / m;
    float v[3] = {g[512] * inv + p.gravity[0] * p.dt, g[1024] * inv + p.gravity[1] * p.dt,
                  g[1536] * inv + p.gravity[2] * p.dt};
    if (m > 0.f) {
      const int3 k = local_block(p, unpack_key(s.blk_pk[b]));
      const float pos[3] = {((float)k.x * 8.f + (float)(cell >> 6)) * p.dx,
                            ((float)k.y * 8.f + (float)((cell >> 3) & 7)) * p.dx,
                            ((float)k.z * 8.f + (float)(cell & 7)) * p.dx};
      apply_walls(p, pos, v);
    }
    g[512] = v[0];
    g[1024] = v[1];
    g[1536] = v[2];
  }
}

// The scene's colliders and level sets, after the walls of k_grid_update, on every node with
// positive mass (their own launch, so that k_grid_update keeps its registers; without colliders
// every CTA returns at once).
__global__ void __launch_bounds__(kThreads) k_grid_boundaries(scene_device s) {
  const scene_params &p = s.prm;
  const int ncol = p.ncolliders ? min(*p.ncolliders, kMaxColliders) : 0;
  const int nls = p.nlevelsets ? min(*p.nlevelsets, kMaxLevelsets) : 0;
  if (ncol + nls == 0) return;
  const long long total = (long long)s.ctr[kCtrBlocks] * 512;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += grid_threads()) {
    const int b = (int)(t >> 9), cell = (int)(t & 511);
    float *g = s.grid + (size_t)b * kGridChannels * 512 + cell;
    if (!(g[0] > 0.f)) continue;
    const int3 k = local_block(p, unpack_key(s.blk_pk[b]));
    const float pos[3] = {((float)k.x * 8.f + (float)(cell >> 6)) * p.dx,
                          ((float)k.y * 8.f + (float)((cell >> 3) & 7)) * p.dx,
                          ((float)k.z * 8.f + (float)(cell & 7)) * p.dx};
    float v[3] = {g[512], g[1024], g[1536]};
    apply_colliders(p, ncol, nls, pos, v);
    g[512] = v[0];
    g[1024] = v[1];
    g[1536] = v[2];
  }
}

// ----------------------------------------------------------------- G2P
// One CTA per block (persistent): stage the 12^3 halo of grid velocities in shared memory,
// then per particle gather v and C (G2P.hpp:56-66), advect, update F = (I + dt C) F
// (G2P.hpp:76-78), run the constitutive update and write the particle to its binned slot
// in the next buffer set, so that storage order follows the binning of this substep.
// Particles are taken 32 per warp and the whole warp steps together (lanes past the block's
// end run on a copy of its first particle and write nothing): the SVD's early exit is a
// warp-wide vote, and the learned closure's tensor-core MLP runs across the warp.  While a
// warp computes one batch, cp.async copies its next batch's state (x|m, F, plastic, id) into
// the warp's other prefetch buffer, and the slot map entry of the batch after that is loaded,
// so the gathers of the particle state wait on no load (1.86 -> 1.72 ms on the 30 M-particle
// sand scene).

// trial-state features of the closure: log singular values and the model's three
// material/state features
__device__ __forceinline__ void closure_features(const material_dev &mat, const float *S, float plastic,
                                                 float *feat) {
#pragma unroll
  for (int i = 0; i < 3; ++i) feat[i] = logf(fmaxf(fabsf(S[i]), 1e-4f));
  if (mat.model == 1) {
    feat[3] = mat.friction_deg;
    feat[4] = mat.cohesion;
    feat[5] = plastic;
  } else {
    feat[3] = mat.theta_c;
    feat[4] = mat.theta_s;
    feat[5] = logf(plastic);
  }
}

__device__ __forceinline__ principal_result plain_principal(const material_dev &mat, const float *S,
                                                            const float *l, float plastic) {
  if (mat.model == 1)
    return dp_principal(mat.mu, mat.lambda, mat.cohesion, mat.beta, mat.volume_correction, mat.yield_surface, l,
                        plastic);
  return snow_principal(mat.mu, mat.lambda, mat.hardening, mat.theta_c, mat.theta_s, S, plastic);
}

// The learned constitutive update (committed ordering), G2P's part.
//
// The network replaces the return-mapping branch, i.e. the projection of a trial state that
// lies outside the yield surface.  Which branch a trial state takes is decided here exactly,
// by the tests of the plain map: Drucker-Prager (compute_stress_sand) projects to the tip when
// tr >= 0 and onto the cone when tr < 0 and dgamma > 0, and is elastic otherwise; snow clamps
// the singular values that leave [1 - theta_c, 1 + theta_s].  Elastic states keep their strain
// and the tip takes its closed form, here.  A projection inside the network's training hull is
// queued (raw features, U, V, S, the plastic state and the binned slot): after G2P the
// tcgen05 kernel runs the network over the queue in 128-row tiles, and k_closure_finish forms
// the projected state, its stress by the model's own formula (Hencky for Drucker-Prager,
// hardened fixed corotated for snow) and writes F, the affine momentum and the plastic state.
// Projections outside the hull, or beyond the queue's capacity, take the plain map here.
// Returns true when the particle was queued (its F, A and plastic state are then not written
// by G2P).
__device__ __forceinline__ bool learned_update(const scene_device &s, const material_dev &mat, const closure_dev &cd,
                                               float *F, float &plastic, float *tau, bool active, int slot, int sid,
                                               int id, float m, const float *Cm, unsigned &all_updates) {
  float U[9], S[3], V[9];
  svd3<true>(F, U, S, V);
  float feat[6];
  closure_features(mat, S, plastic, feat);
  bool project = false;
  float H[3], pl_new = plastic;
  if (mat.model == 1) {
    float eps[3], eh[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) eps[i] = feat[i] - mat.cohesion;
    const float sum_eps = eps[0] + eps[1] + eps[2];
    const float tr = sum_eps + plastic;
#pragma unroll
    for (int i = 0; i < 3; ++i) eh[i] = eps[i] - tr / 3.f;
    const float ehn = sqrtf(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2]);
    const float smu = 2.f * mat.mu;
    if (tr >= 0.f) {
#pragma unroll
      for (int i = 0; i < 3; ++i) H[i] = mat.cohesion;
      if (mat.volume_correction) pl_new = mat.beta * sum_eps + plastic;
    } else {
      pl_new = 0.f;
      const float dg = ehn + (3.f * mat.lambda + smu) / smu * tr * mat.yield_surface;
      project = dg > 0.f;
#pragma unroll
      for (int i = 0; i < 3; ++i) H[i] = feat[i];
    }
  } else {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      project = project || S[i] < 1.f - mat.theta_c || S[i] > 1.f + mat.theta_s;
      H[i] = feat[i];
    }
  }
  bool in_hull = true;
#pragma unroll
  for (int k = 0; k < kMlpIn; ++k) in_hull = in_hull && feat[k] >= cd.in_min[k] && feat[k] <= cd.in_max[k];
  bool queued = false;
  const bool want = active && project && in_hull;
  const unsigned wq = __ballot_sync(0xffffffffu, want);
  all_updates += __popc(__ballot_sync(0xffffffffu, active));
  if (wq) {
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == __ffs(wq) - 1) base = atomicAdd(&s.ctr[kCtrQueue], __popc(wq));
    base = __shfl_sync(0xffffffffu, base, __ffs(wq) - 1);
    if (want) {
      const long long k = base + __popc(wq & lanemask_lt());
      if (k < s.aux.qcap) {
        float *fr = s.aux.q_feat + 6 * k;
#pragma unroll
        for (int i = 0; i < 6; ++i) fr[i] = feat[i];
        float *u = s.aux.q_uvs + kQueueFloats * k;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
          u[i] = U[i];
          u[9 + i] = V[i];
        }
        u[18] = S[0];
        u[19] = S[1];
        u[20] = S[2];
        u[21] = plastic;
        // the particle's mass and C, for the affine momentum (so that the finish reads only the
        // queue)
        u[22] = m;
#pragma unroll
        for (int i = 0; i < 9; ++i) u[23 + i] = Cm[i];
        s.aux.q_slot[k] = make_int2(slot, sid);
        s.aux.q_id[k] = id;
        queued = true;
      }
    }
  }
  if (queued) return true;
  float Ns[3], tp[3];
  if (active && project) {
    // outside the hull (or a full queue): the plain map
    const principal_result r = plain_principal(mat, S, feat, plastic);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      tp[i] = r.tau[i];
      Ns[i] = r.Ns[i];
    }
    pl_new = r.plastic;
    atomicAdd(&cd.audit[5], 1.0);
  } else if (mat.model == 1) {
#pragma unroll
    for (int i = 0; i < 3; ++i) Ns[i] = expf(H[i]);
    const float trl = H[0] + H[1] + H[2];
#pragma unroll
    for (int i = 0; i < 3; ++i) tp[i] = 2.f * mat.mu * H[i] + mat.lambda * trl;
  } else {
#pragma unroll
    for (int i = 0; i < 3; ++i) Ns[i] = S[i];  // inside the clamp box: no projection, Jp unchanged
    const float e = expf(mat.hardening * (1.f - plastic));
    float Ph[3];
    fc_principal(mat.mu * e, mat.lambda * e, Ns, Ph);
#pragma unroll
    for (int i = 0; i < 3; ++i) tp[i] = Ph[i] * Ns[i];
  }
  plastic = pl_new;
  const float d[3] = {tp[0] * mat.volume, tp[1] * mat.volume, tp[2] * mat.volume};
  mul_diag_t(tau, U, d, U);
  mul_diag_t(F, U, Ns, V);
  return false;
}

// The learned update's second part, for the projections the network has given (after the
// tcgen05 pass over the queue): projected state, its stress, F, the affine momentum and the
// plastic state written to the particle's binned slot; one projection in audit_period is
// checked against the plain map (double accumulators).
__global__ void __launch_bounds__(kThreads) k_closure_finish(scene_device s) {
  const closure_dev &cd = s.aux.cd;
  const int nq = (int)min((long long)s.ctr[kCtrQueue], s.aux.qcap);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (nq > 0) atomicAdd(&cd.audit[6], (double)nq);
    // a bounded tensor-core wait of the network pass that gave up is the scene's error too
    if (cd.tc_status && *cd.tc_status) set_status(s.ctr, kStatusTimeout);
  }
  const int substep = s.ctr[kCtrQueueSubstep];  // of the G2P that queued the rows
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nq; k += grid_threads()) {
    const int2 sl = s.aux.q_slot[k];
    const int slot = sl.x;
    const material_dev mat = s.prm.batch ? s.prm.mats[sl.y] : s.prm.mat;
    const float *u = s.aux.q_uvs + kQueueFloats * (size_t)k;
    float U[9], V[9], S[3], feat[6], y[6];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      U[i] = u[i];
      V[i] = u[9 + i];
    }
    S[0] = u[18];
    S[1] = u[19];
    S[2] = u[20];
    const float plastic = u[21];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      feat[i] = s.aux.q_feat[6 * (size_t)k + i];
      y[i] = s.aux.q_out[6 * (size_t)k + i];
    }
    float H[3], Ns[3], tp[3], pl_new;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      H[i] = feat[i] + y[i];
      Ns[i] = expf(H[i]);
    }
    if (mat.model == 1) {
      pl_new = 0.f;  // the cone branch (tr < 0) resets logJp, as compute_stress_sand does
      const float trl = H[0] + H[1] + H[2];
#pragma unroll
      for (int i = 0; i < 3; ++i) tp[i] = 2.f * mat.mu * H[i] + mat.lambda * trl;
    } else {
      pl_new = plastic * (S[0] * S[1] * S[2] / fmaxf(Ns[0] * Ns[1] * Ns[2], 1e-6f));
      const float e = expf(mat.hardening * (1.f - pl_new));
      float Ph[3];
      fc_principal(mat.mu * e, mat.lambda * e, Ns, Ph);
#pragma unroll
      for (int i = 0; i < 3; ++i) tp[i] = Ph[i] * Ns[i];
    }
    const int id = s.aux.q_id[k];
    if (cd.audit_period > 0 &&
        ((unsigned)id * 2654435761u + (unsigned)substep * 40503u) % (unsigned)cd.audit_period == 0u) {
      const principal_result r = plain_principal(mat, S, feat, plastic);
      float d2 = 0.f, t2 = 0.f;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        d2 += (tp[i] - r.tau[i]) * (tp[i] - r.tau[i]);
        t2 += r.tau[i] * r.tau[i];
      }
      const float floor_stress = 1e-4f * (3.f * mat.lambda + 2.f * mat.mu);
      const float rel = sqrtf(d2) / (sqrtf(t2) + floor_stress);
      // non-negative doubles order like their bit patterns, so the max is an integer max
      atomicAdd(&cd.audit[0], 1.0);
      atomicAdd(&cd.audit[1], (double)rel);
      atomicMax(reinterpret_cast<unsigned long long *>(&cd.audit[2]),
                (unsigned long long)__double_as_longlong((double)rel));
      atomicAdd(&cd.audit[3], (double)d2);
      atomicAdd(&cd.audit[4], (double)t2);
    }
    const float dd[3] = {tp[0] * mat.volume, tp[1] * mat.volume, tp[2] * mat.volume};
    float tau[9], Fn[9];
    mul_diag_t(tau, U, dd, U);
    mul_diag_t(Fn, U, Ns, V);
    const float m = u[22];
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      s.nxt.F[mat_at(c, slot)] = Fn[c];
      s.nxt.A[mat_at(c, slot)] = m * u[23 + c] - s.prm.kappa * tau[c];
    }
    if (s.nxt.plastic) s.nxt.plastic[slot] = pl_new;
  }
}

// Shared memory of k_g2p: the velocity halo, one float4 (vx, vy, vz, vz) per node so that a
// node is one 16-byte load (z twice: the gather's pairs are (x, y) and (z, z)); then per warp
// two prefetch buffers of 32 particles, each laid out as x|m float4[32], F[9][32],
// plastic[32], id[32] (kG2PPrefetch floats).
constexpr int kG2PPrefetch = 4 * 32 + 9 * 32 + 32 + 32;
constexpr size_t g2p_smem_bytes(int nt) {
  return sizeof(float4) * kHaloCells + sizeof(float) * 2 * kG2PPrefetch * (size_t)(nt / 32);
}

// cp.async (sm_80 and later): copies that land in shared memory while the warp computes
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// kLearned: the closure's network gives the return map's projections (queued for the tcgen05
// pass, 256 threads only); kBatch: batched scenes (per-block scene material, scene-local block
// origin); NT threads per CTA.  The variants are register-capped for 3 (256 threads) or 5 (128
// threads) resident CTAs per SM: the kernel is issue- and latency-bound, and the extra warps
// hide more latency than the cap costs (2.41 -> 2.09 ms on the 30 M-particle sand scene, no
// spills).
// kCell: G2C2PTransfer with PreG2C2PTransfer and PostG2C2PTransfer (the cell-centric pair,
// fixed corotated), gathered per particle: a particle takes sum_c W_c/8 v_i over the 8 corners i
// of its cells c, i.e. the node weights (3/4 - f/2, 1/2, f/2 - 1/4) per axis over the same three
// nodes as the quadratic stencil (f = x/dx - base, base = floor(x/dx + 1/2) - 1), and
// B = sum W v_i (x_i - x_p)^T; then F <- (I + dt B Dinv) F, x += v dt, and the affine term A of
// the next P2C2G from the new state.
template <bool kLearned, bool kBatch, int NT, bool kCell = false>
__global__ void __launch_bounds__(NT, NT == 256 ? 3 : 5) k_g2p(scene_device s) {
  static_assert(!kLearned || NT == kThreads, "learned G2P runs at 256 threads");
  static_assert(!kCell || (!kLearned && !kBatch), "the cell-centric pair runs on single fixed-corotated scenes");
  extern __shared__ __align__(16) float g2p_smem[];
  float4 *svf = reinterpret_cast<float4 *>(g2p_smem);
  __shared__ int s_b;
  __shared__ material_dev s_mat;
  __shared__ unsigned s_moved;  // the block's move mask
  const scene_params &p = s.prm;
  const int nb = s.ctr[kCtrBlocks];
  const int substep = s.ctr[kCtrSubstep];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    s.ctr[kCtrMaskFrom] = nb;
    if (kLearned) s.ctr[kCtrQueueSubstep] = substep;  // for the closure pass's audit sampling
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float *const pf = g2p_smem + 4 * kHaloCells + warp * 2 * kG2PPrefetch;
  unsigned all_updates = 0;  // learned closure: particle updates of this warp
  // the lane's particle of a batch into prefetch buffer `buf` (lanes past the block's end copy
  // the block's first particle)
  auto prefetch = [&](int buf, int i) {
    float *b = pf + buf * kG2PPrefetch;
    cp_async16(b + 4 * lane, &s.cur.xm[i]);
#pragma unroll
    for (int k = 0; k < 9; ++k) cp_async4(b + 128 + 32 * k + lane, &s.cur.F[mat_at(k, i)]);
    if (s.cur.plastic) cp_async4(b + 416 + lane, &s.cur.plastic[i]);
    cp_async4(b + 448 + lane, &s.cur.id[i]);
    cp_async_commit();
  };
  for (;;) {
    const int w = grab_block(&s.ctr[kCtrWork + kWorkG2P], &s_b);
    if (w >= nb) break;
    const int b = s.work_order[w];
    const int start = s.block_start[b], end = s.block_start[b + 1];
    if (start == end) {
      if (threadIdx.x == 0) s.bmask[b] = 0u;
      continue;
    }
    const int3 gk = unpack_key(s.blk_pk[b]);
    if (kBatch && threadIdx.x == 0) s_mat = p.mats[scene_of_key(gk)];
    if (threadIdx.x == 0) s_moved = 0u;
    // halo load: items (hx, hy, quad) over 12 x 12 x 3; each reads four consecutive cells of
    // the three velocity channels (16-byte loads) and writes four float4 nodes
    for (int it = threadIdx.x; it < kHalo * kHalo * 3; it += NT) {
      const int quad = it % 3, hy = (it / 3) % kHalo, hx = it / (3 * kHalo);
      const int t = (hx >= 8 ? 4 : 0) | (hy >= 8 ? 2 : 0) | (quad == 2 ? 1 : 0);
      const int tb = s.nbr[b * 8 + t];
      float4 vx = make_float4(0.f, 0.f, 0.f, 0.f), vy = vx, vz = vx;
      if (tb >= 0) {
        const int cell = ((hx & 7) << 6) | ((hy & 7) << 3) | ((quad * 4) & 7);
        const float *g = s.grid + ((size_t)tb * kGridChannels + 1) * 512 + cell;
        vx = *reinterpret_cast<const float4 *>(g);
        vy = *reinterpret_cast<const float4 *>(g + 512);
        vz = *reinterpret_cast<const float4 *>(g + 1024);
      }
      float4 *dst = svf + (hx * kHalo + hy) * kHalo + quad * 4;
      dst[0] = make_float4(vx.x, vy.x, vz.x, vz.x);
      dst[1] = make_float4(vx.y, vy.y, vz.y, vz.y);
      dst[2] = make_float4(vx.z, vy.z, vz.z, vz.z);
      dst[3] = make_float4(vx.w, vy.w, vz.w, vz.w);
    }
    __syncthreads();
    const int3 bk = kBatch ? local_block(p, gk) : gk;
    const int org[3] = {bk.x * 8, bk.y * 8, bk.z * 8};
    // each warp takes batches of 32 slots; the next batch's particles are copied into the
    // warp's other prefetch buffer while this batch computes
    int buf = 0;
    int i = 0, inext = 0;  // the particle of this batch and of the next
    const int base0 = start + warp * 32;
    if (base0 < end) {
      i = s.src[base0 + lane < end ? base0 + lane : start];
      prefetch(0, i);
      if (base0 + NT < end) inext = s.src[base0 + NT + lane < end ? base0 + NT + lane : start];
    }
    for (int base = start + warp * 32; base < end; base += NT) {
      const int slot = base + lane;
      // every lane of the warp stays in the loop (lanes past the block's end work on a copy of
      // its first particle and store nothing): the SVD's early exit is a warp-wide vote
      const bool active = slot < end;
      const bool more = base + NT < end;  // warp-uniform
      // the batch after next: its slot map load has a whole batch to land
      const int nslot2 = base + 2 * NT + lane;
      const int inext2 = base + 2 * NT < end ? s.src[nslot2 < end ? nslot2 : start] : 0;
      cp_async_wait_all();  // this batch's copies (the only group in flight)
      const float *pb = pf + buf * kG2PPrefetch;
      float4 xm = reinterpret_cast<const float4 *>(pb)[lane];
      const int icur = i;
      if (more) prefetch(buf ^ 1, inext);
      buf ^= 1;
      i = inext;
      inext = inext2;
      int hb[3];
      float w[3][3], f[3];
      if (kCell) {
        // the index bucket floor(x / dx + 1/2) as the binning computes it; its cells are
        // bucket - 1 and bucket, their corners the nodes bucket - 1 .. bucket + 1
        const float X[3] = {xm.x * p.inv_dx, xm.y * p.inv_dx, xm.z * p.inv_dx};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float bs = floorf(X[d] + 0.5f) - 1.f;
          f[d] = X[d] - bs;
          hb[d] = (int)bs - org[d];
          w[d][0] = 0.75f - 0.5f * f[d];
          w[d][1] = 0.5f;
          w[d][2] = 0.5f * f[d] - 0.25f;
        }
      } else {
        const float X[3] = {over_dx(p, xm.x), over_dx(p, xm.y), over_dx(p, xm.z)};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float bs = floorf(X[d] - 0.5f);
          f[d] = X[d] - bs;
          hb[d] = (int)bs - org[d];
          w[d][0] = 0.5f * (1.5f - f[d]) * (1.5f - f[d]);
          const float f1 = f[d] - 1.f;
          w[d][1] = 0.75f - f1 * f1;
          const float f2 = 0.5f + f1;
          w[d][2] = 0.5f * f2 * f2;
        }
      }
      const bool inside = hb[0] >= 0 && hb[0] <= kHalo - 3 && hb[1] >= 0 && hb[1] <= kHalo - 3 &&
                          hb[2] >= 0 && hb[2] <= kHalo - 3;
      if (active && !inside) set_status(s.ctr, kStatusMissingBlock);
      // the cell this slot was binned in, as the binning computed it from the same position
      const int sid = kBatch ? s.cur.sid[icur] : 0;
      int3 cell_old = make_int3(0x7fffffff, 0, 0), blk_old;
      if (active && !particle_cell(s, sid, xm, cell_old, blk_old)) cell_old.x = 0x7fffffff;
      float vel[3] = {0.f, 0.f, 0.f};
      float B[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // sum W v (node - f)^T
      if (inside) {
        // paired FP32 arithmetic (fma.rn.f32x2): the x and y components of a node go as one
        // pair, and z as the pair (z, z) that the halo stores in the fourth slot, taking the
        // weights (wz, wz (k - fz)); every lane of a pair is the same correctly rounded
        // operation as the scalar form
        float2 wzp[3], wdp[3], wzz[3];  // (wz, wz), (wzd, wzd), (wz, wzd) of node k
#pragma unroll
        for (int kk = 0; kk < 3; ++kk) {
          const float wz = w[2][kk], wzd = wz * ((float)kk - f[2]);
          wzp[kk] = make_float2(wz, wz);
          wdp[kk] = make_float2(wzd, wzd);
          wzz[kk] = make_float2(wz, wzd);
        }
        float2 vxy = make_float2(0.f, 0.f), bxy0 = vxy, bxy3 = vxy, bxy6 = vxy;
#pragma unroll
        for (int ii = 0; ii < 3; ++ii) {
          const float dxi = (float)ii - f[0];
#pragma unroll
          for (int jj = 0; jj < 3; ++jj) {
            const float dyj = (float)jj - f[1];
            const float wij = w[0][ii] * w[1][jj];
            const int hrow = ((hb[0] + ii) * kHalo + (hb[1] + jj)) * kHalo + hb[2];
            // separable accumulation over k: s0 = sum_k wz v, s1 = sum_k wz (k - fz) v, the
            // xy parts as pairs and the z parts as the pair (s0z, s1z)
            float2 s0 = make_float2(0.f, 0.f), s1 = s0, sz = s0;
#pragma unroll
            for (int kk = 0; kk < 3; ++kk) {
              const float4 node = svf[hrow + kk];
              const float2 nxy = make_float2(node.x, node.y), nzz = make_float2(node.z, node.w);
              s0 = __ffma2_rn(wzp[kk], nxy, s0);
              s1 = __ffma2_rn(wdp[kk], nxy, s1);
              sz = __ffma2_rn(wzz[kk], nzz, sz);
            }
            const float2 wij2 = make_float2(wij, wij);
            const float2 axy = __fmul2_rn(wij2, s0);
            vxy = __fadd2_rn(vxy, axy);
            bxy0 = __ffma2_rn(axy, make_float2(dxi, dxi), bxy0);
            bxy3 = __ffma2_rn(axy, make_float2(dyj, dyj), bxy3);
            bxy6 = __ffma2_rn(wij2, s1, bxy6);
            const float az = wij * sz.x;
            vel[2] += az;
            B[2] = fmaf(az, dxi, B[2]);
            B[5] = fmaf(az, dyj, B[5]);
            B[8] = fmaf(wij, sz.y, B[8]);
          }
        }
        vel[0] = vxy.x, vel[1] = vxy.y;
        B[0] = bxy0.x, B[1] = bxy0.y, B[3] = bxy3.x, B[4] = bxy3.y, B[6] = bxy6.x, B[7] = bxy6.y;
      }
      float C[9];  // APIC: C = (4/dx^2) sum W v (x_i - x_p)^T; the cell pair: B = sum W v (x_i - x_p)^T
#pragma unroll
      for (int k = 0; k < 9; ++k) C[k] = B[k] * (kCell ? p.dx : p.four_over_dx);
      // the cell pair updates F with B Dinv at the position before the move
      // (PostG2C2PTransfer); APIC with C
      float Cs[9];
      if (kCell) {
        const float dold[3] = {cell_dinv(p, xm.x), cell_dinv(p, xm.y), cell_dinv(p, xm.z)};
#pragma unroll
        for (int k = 0; k < 9; ++k) Cs[k] = C[k] * dold[k / 3];
      } else {
#pragma unroll
        for (int k = 0; k < 9; ++k) Cs[k] = C[k];
      }
      xm.x += vel[0] * p.dt;
      xm.y += vel[1] * p.dt;
      xm.z += vel[2] * p.dt;
      {
        // the block of the new position, as the next activation computes it from the stored
        // x, recorded relative to this block for k_insert_moved_blocks; and whether the
        // particle left the cell it was binned in, for the next (incremental) binning
        unsigned bit = 0u;
        bool moved_far = false, left_cell = false;
        if (active) {
          int3 c2, b2;
          if (particle_cell(s, sid, xm, c2, b2)) {
            const int ox = b2.x - gk.x, oy = b2.y - gk.y, oz = b2.z - gk.z;
            if (ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1 && oz >= -1 && oz <= 1)
              bit = 1u << ((ox + 1) * 9 + (oy + 1) * 3 + (oz + 1));
            else
              moved_far = true;
            left_cell = c2.x != cell_old.x || c2.y != cell_old.y || c2.z != cell_old.z;
          } else {
            moved_far = true;  // the particle pass of the next activation reports it
          }
          s.moved[slot] = (uint8_t)(left_cell || moved_far);
        }
        const unsigned wbits = __reduce_or_sync(kFull, bit);
        if (lane == 0 && wbits) atomicOr(&s_moved, wbits);
        bool bad = moved_far;
        const unsigned leavers = __ballot_sync(kFull, left_cell && !moved_far);
        if (leavers) {
          int base = 0;
          if (lane == 0) base = atomicAdd(&s.ctr[kCtrMovers], __popc(leavers));
          base = __shfl_sync(kFull, base, 0);
          if ((leavers >> lane) & 1u) {
            const int k = base + __popc(leavers & lanemask_lt());
            if (k < p.mover_cap)
              s.movers[k] = slot;
            else
              bad = true;  // list full: the next substep bins every particle
          }
        }
        if (__any_sync(kFull, bad) && lane == 0) s.ctr[kCtrMaskBad] = 1;
      }
      // F, the plastic state and the id from the prefetch buffer, read after the gather so
      // that they take no registers during it (the buffer is next written by the prefetch of
      // the following batch)
      float F[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) F[k] = pb[128 + 32 * k + lane];
      float pl = s.cur.plastic ? pb[416 + lane] : 0.f;
      const int id = __float_as_int(pb[448 + lane]);
      // F <- (I + dt C) F
      float Fn[9];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r)
          Fn[3 * c + r] = F[3 * c + r] + p.dt * (Cs[r] * F[3 * c] + Cs[3 + r] * F[3 * c + 1] + Cs[6 + r] * F[3 * c + 2]);
      // trial-state log for the closure's training set
      if (!kBatch && s.aux.log_period > 0 && active && p.mat.model != 0 &&
          ((unsigned)id + (unsigned)substep) % (unsigned)s.aux.log_period == 0u) {
        float U[9], S[3], V[9], feat[6];
        svd3(Fn, U, S, V);
        closure_features(p.mat, S, pl, feat);
        const unsigned long long k = atomicAdd(s.aux.log_count, 1ull);
        if ((long long)k < s.aux.log_cap)
          for (int q = 0; q < 6; ++q) s.aux.log_buf[6 * k + q] = feat[q];
      }
      float tau[9];
      // in a batch the closure serves the scenes of its material model (uniform over a CTA: a
      // block belongs to one scene); a queued projection's F, A and plastic state are written
      // by k_closure_finish
      bool queued = false;
      if (kLearned && (!kBatch || s_mat.model == s.aux.cd.model))
        queued = learned_update(s, kBatch ? s_mat : p.mat, s.aux.cd, Fn, pl, tau, active, slot, sid, id, xm.w, C,
                                all_updates);
      else if (kBatch)
        constitutive<true>(s_mat, Fn, pl, tau);
      else
        constitutive<true>(p.mat, Fn, pl, tau);
      if (!active) continue;
      s.nxt.xm[slot] = xm;
      s.nxt.v[slot] = make_float4(vel[0], vel[1], vel[2], 0.f);
#pragma unroll
      for (int k = 0; k < 9; ++k) s.nxt.C[mat_at(k, slot)] = C[k];
      if (kCell) {
        // the affine term of the next P2C2G, from the new position and F (P2C2G.hpp:86-146)
        const float dnew[3] = {cell_dinv(p, xm.x), cell_dinv(p, xm.y), cell_dinv(p, xm.z)};
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          s.nxt.A[mat_at(k, slot)] = (xm.w * C[k] - p.dt * tau[k]) * dnew[k / 3];
          s.nxt.F[mat_at(k, slot)] = Fn[k];
        }
        if (s.nxt.plastic) s.nxt.plastic[slot] = pl;
      } else if (!queued) {
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          s.nxt.A[mat_at(k, slot)] = xm.w * C[k] - p.kappa * tau[k];
          s.nxt.F[mat_at(k, slot)] = Fn[k];
        }
        if (s.nxt.plastic) s.nxt.plastic[slot] = pl;
      }
      s.nxt.id[slot] = id;
      if (kBatch) s.nxt.sid[slot] = sid;
    }
    __syncthreads();
    if (threadIdx.x == 0) s.bmask[b] = s_moved;
  }
  if (kLearned && lane == 0 && all_updates) atomicAdd(&s.aux.cd.audit[7], (double)all_updates);
}

// ----------------------------------------------------------------- G2P2G and the implicit system
// G2P2GTransfer (simulation/transfer/G2P2G.hpp:49-142), the force operator of the implicit
// solve (simulation/mpm/ImplicitMPM.hpp:34-61).  One CTA per block (persistent); the velocity
// field is staged in a 12^3 halo of float4 nodes.  The block's 512 cells are processed in
// chunks of 64, in two phases as in P2G:
//  1. consecutive threads take consecutive particles of the chunk: gather C, form the trial
//     F = (I + dt C) F, evaluate the stress on a copy of the state (nothing is written back),
//     and stage the particle's weights and its force in the affine form
//     f(node) = W (q + ii a_x + jj a_y + kk a_z), (a_x a_y a_z) = (4/dx) tau, q = -(4/dx) tau f,
//     which equals W (4/dx^2) tau (x_i - x_p) with node offsets (ii, jj, kk) in cells;
//  2. one thread per (cell, component) sums the staged particles of its cell into 27
//     registers (all particles of a cell share the 27 nodes) and adds them to a 12^3 force
//     halo in shared memory, which is flushed into f with 16-byte reductions.
// Against one shared atomic per particle, node and component (81 per particle, limited by the
// shared-atomic rate) the staging takes the kernel from 3.6 to 2.95 ms on 30 M particles.
// v and f are node-major over the active blocks in canonical order, v[(block*512 + cell)*3 + d]:
// the layout of a dof_view<space, 3> over a Vector (types/View.h:77-168).
constexpr int kG2P2GThreads = 256;
constexpr int kG2P2GChunk = 64;
constexpr int kG2P2GRanks = 11;   // particles per cell staged per chunk (more scatter directly)
constexpr int kG2P2GFields = 21;  // w[9], q[3], ax[3], ay[3], az[3]
constexpr int kG2P2GRow = kG2P2GChunk + 1;
constexpr int kG2P2GMap = 1024;   // slots of a chunk mapped to their cell (more: binary search)
constexpr size_t kG2P2GSmem = sizeof(float4) * kHaloCells + sizeof(float) * 3 * kHaloCells +
                              sizeof(float) * kG2P2GFields * kG2P2GRanks * kG2P2GRow +
                              sizeof(int) * 2 * (kG2P2GChunk + 1) + 2 * kG2P2GMap;

__global__ void __launch_bounds__(kG2P2GThreads, 2)
    k_g2p2g(scene_device s, const float *__restrict__ vin, float *__restrict__ fout, long long ndofs, float dt,
            const int *skip) {
  if (skip && *skip) return;
  extern __shared__ __align__(16) float gg_smem[];
  float4 *svf = reinterpret_cast<float4 *>(gg_smem);
  float *sf = gg_smem + 4 * kHaloCells;  // [3][kHaloCells]
  auto stg = reinterpret_cast<float(*)[kG2P2GRanks][kG2P2GRow]>(sf + 3 * kHaloCells);
  int *const s_cs0 = reinterpret_cast<int *>(sf + 3 * kHaloCells + kG2P2GFields * kG2P2GRanks * kG2P2GRow);
  unsigned char *const s_map0 = reinterpret_cast<unsigned char *>(s_cs0 + 2 * (kG2P2GChunk + 1));
  __shared__ int s_b;
  const scene_params &p = s.prm;
  const int nb = s.ctr[kCtrBlocks];
  if ((long long)nb * 1536 > ndofs) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_status(s.ctr, kStatusCapacity);
    return;
  }
  const int t = threadIdx.x;
  const int my_cell = t % kG2P2GChunk, my_ch = t / kG2P2GChunk;
  // the force halo starts zeroed; each block's flush zeroes the quads it sends (as in k_p2g)
  for (int q = t; q < 3 * kHaloCells; q += kG2P2GThreads) sf[q] = 0.f;
  for (;;) {
    const int w = grab_block(&s.ctr[kCtrWork + kWorkG2P2G], &s_b);
    if (w >= nb) break;
    const int b = s.work_order[w];
    const int start = s.block_start[b], end = s.block_start[b + 1];
    if (start == end) continue;
    // velocity halo: items (hx, hy, quad) over 12 x 12 x 3; four consecutive nodes are 12
    // consecutive floats (three 16-byte loads)
    for (int it = t; it < kHalo * kHalo * 3; it += kG2P2GThreads) {
      const int quad = it % 3, hy = (it / 3) % kHalo, hx = it / (3 * kHalo);
      const int tb = s.nbr[b * 8 + ((hx >= 8 ? 4 : 0) | (hy >= 8 ? 2 : 0) | (quad == 2 ? 1 : 0))];
      float4 a = make_float4(0.f, 0.f, 0.f, 0.f), c = a, d = a;
      if (tb >= 0) {
        const int cell = ((hx & 7) << 6) | ((hy & 7) << 3) | ((quad * 4) & 7);
        const float4 *g = reinterpret_cast<const float4 *>(vin + ((size_t)tb * 512 + cell) * 3);
        a = g[0];
        c = g[1];
        d = g[2];
      }
      float4 *dst = svf + (hx * kHalo + hy) * kHalo + quad * 4;
      dst[0] = make_float4(a.x, a.y, a.z, 0.f);
      dst[1] = make_float4(a.w, c.x, c.y, 0.f);
      dst[2] = make_float4(c.z, c.w, d.x, 0.f);
      dst[3] = make_float4(d.y, d.z, d.w, 0.f);
    }
    const int3 bk = unpack_key(s.blk_pk[b]);
    const int org[3] = {bk.x * 8, bk.y * 8, bk.z * 8};
    // cell starts of chunk k in s_cs0 + (k & 1) * (kG2P2GChunk + 1) and its slot -> cell map in
    // s_map0 + (k & 1) * kG2P2GMap; the next chunk's are filled during this chunk's phase 2
    auto fill = [&](int k) {
      if (t <= kG2P2GChunk) {
        const int nc = k * kG2P2GChunk + t;
        s_cs0[(k & 1) * (kG2P2GChunk + 1) + t] = nc < 512 ? s.cell_start[b * 512 + nc] : end;
      }
      if (t < kG2P2GChunk) {
        const int c = k * kG2P2GChunk + t;
        const int cs = s.cell_start[b * 512 + c];
        const int ce = c + 1 < 512 ? s.cell_start[b * 512 + c + 1] : end;
        const int base = s.cell_start[b * 512 + k * kG2P2GChunk];
        unsigned char *m = s_map0 + (k & 1) * kG2P2GMap;
        for (int q = cs - base; q < ce - base && q < kG2P2GMap; ++q) m[q] = (unsigned char)t;
      }
    };
    fill(0);
    for (int chunk = 0; chunk < 512 / kG2P2GChunk; ++chunk) {
      const int cell0 = chunk * kG2P2GChunk;
      __syncthreads();  // halos ready, previous staging consumed, this chunk's starts and map in place
      const int *s_cs = s_cs0 + (chunk & 1) * (kG2P2GChunk + 1);
      const unsigned char *s_map = s_map0 + (chunk & 1) * kG2P2GMap;
      const int c0 = s_cs[0], c1 = s_cs[kG2P2GChunk];
      // ---- phase 1 (the whole CTA steps together: the SVD's early exit is a warp vote, so
      // lanes past the chunk's end run on a copy of its first particle and stage nothing)
      for (int base = c0; base < c1; base += kG2P2GThreads) {
        const int slot = base + t;
        const bool active = slot < c1;
        const int i = s.src[active ? slot : c0];
        const float4 xm = s.cur.xm[i];
        float F[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) F[k] = s.cur.F[mat_at(k, i)];
        float pl = s.cur.plastic ? s.cur.plastic[i] : 0.f;
        const float X[3] = {over_dx(p, xm.x), over_dx(p, xm.y), over_dx(p, xm.z)};
        int hb[3];
        float w[3][3], f[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float bs = floorf(X[d] - 0.5f);
          f[d] = X[d] - bs;
          hb[d] = (int)bs - org[d];
          w[d][0] = 0.5f * (1.5f - f[d]) * (1.5f - f[d]);
          const float f1 = f[d] - 1.f;
          w[d][1] = 0.75f - f1 * f1;
          const float f2 = 0.5f + f1;
          w[d][2] = 0.5f * f2 * f2;
        }
        const bool inside = hb[0] >= 0 && hb[0] <= kHalo - 3 && hb[1] >= 0 && hb[1] <= kHalo - 3 &&
                            hb[2] >= 0 && hb[2] <= kHalo - 3;
        if (active && !inside) set_status(s.ctr, kStatusMissingBlock);
        float B[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // sum W v (node - f)^T
        if (inside) {
#pragma unroll
          for (int ii = 0; ii < 3; ++ii) {
            const float dxi = (float)ii - f[0];
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) {
              const float dyj = (float)jj - f[1];
              const float wij = w[0][ii] * w[1][jj];
              const int hrow = ((hb[0] + ii) * kHalo + (hb[1] + jj)) * kHalo + hb[2];
              float s0[3] = {0.f, 0.f, 0.f}, s1[3] = {0.f, 0.f, 0.f};
#pragma unroll
              for (int kk = 0; kk < 3; ++kk) {
                const float wz = w[2][kk], wzd = wz * ((float)kk - f[2]);
                const float4 node = svf[hrow + kk];
                s0[0] += wz * node.x;
                s0[1] += wz * node.y;
                s0[2] += wz * node.z;
                s1[0] += wzd * node.x;
                s1[1] += wzd * node.y;
                s1[2] += wzd * node.z;
              }
#pragma unroll
              for (int d = 0; d < 3; ++d) {
                const float a = wij * s0[d];
                B[d] += a * dxi;
                B[3 + d] += a * dyj;
                B[6 + d] += wij * s1[d];
              }
            }
          }
        }
        // trial F = (I + dt C) F (G2P2G.hpp:103-105), C = B 4/dx
        float Fn[9];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int r = 0; r < 3; ++r)
            Fn[3 * c + r] = F[3 * c + r] + dt * p.four_over_dx *
                                               (B[r] * F[3 * c] + B[3 + r] * F[3 * c + 1] + B[6 + r] * F[3 * c + 2]);
        float tau[9];
        constitutive<true>(p.mat, Fn, pl, tau);
        if (!active) continue;
        float ax[3], ay[3], az[3], q[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          ax[d] = tau[d] * p.four_over_dx;
          ay[d] = tau[3 + d] * p.four_over_dx;
          az[d] = tau[6 + d] * p.four_over_dx;
          q[d] = -(ax[d] * f[0] + ay[d] * f[1] + az[d] * f[2]);
        }
        int lo = 0;  // the cell of this slot: the last cell whose start is <= slot
        if (slot - c0 < kG2P2GMap) {
          lo = s_map[slot - c0];
        } else {
          int hi = kG2P2GChunk;
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_cs[mid] <= slot) lo = mid;
            else hi = mid;
          }
        }
        const int cl = lo, r = slot - s_cs[lo], cell = cell0 + cl;
        const bool on_cell = hb[0] == (cell >> 6) + 1 && hb[1] == ((cell >> 3) & 7) + 1 && hb[2] == (cell & 7) + 1;
        if (r >= kG2P2GRanks || !on_cell) {
          // beyond the staged ranks, or a stencil origin that rounding moved off the cell:
          // scatter directly and stage a zero stand-in
          if (inside)
            for (int ii = 0; ii < 3; ++ii)
              for (int jj = 0; jj < 3; ++jj)
                for (int kk = 0; kk < 3; ++kk) {
                  const float W = w[0][ii] * w[1][jj] * w[2][kk];
                  const int h = ((hb[0] + ii) * kHalo + (hb[1] + jj)) * kHalo + hb[2] + kk;
#pragma unroll
                  for (int d = 0; d < 3; ++d)
                    atomicAdd(&sf[d * kHaloCells + h],
                              W * (q[d] + (float)ii * ax[d] + (float)jj * ay[d] + (float)kk * az[d]));
                }
          if (r < kG2P2GRanks)
            for (int fl = 0; fl < kG2P2GFields; ++fl) stg[fl][r][cl] = 0.f;
          continue;
        }
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) stg[3 * a + c][r][cl] = w[a][c];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          stg[9 + d][r][cl] = q[d];
          stg[12 + d][r][cl] = ax[d];
          stg[15 + d][r][cl] = ay[d];
          stg[18 + d][r][cl] = az[d];
        }
      }
      __syncthreads();
      if (chunk + 1 < 512 / kG2P2GChunk) fill(chunk + 1);
      // ---- phase 2: thread (cell, component) sums the staged particles of its cell
      const int cnt = my_ch < 3 ? min(s_cs[my_cell + 1] - s_cs[my_cell], kG2P2GRanks) : 0;
      if (cnt > 0) {
        const int d = my_ch;
        float acc[27];
#pragma unroll
        for (int n = 0; n < 27; ++n) acc[n] = 0.f;
        for (int r = 0; r < cnt; ++r) {
          float w[3][3];
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) w[a][c] = stg[3 * a + c][r][my_cell];
          const float q = stg[9 + d][r][my_cell];
          const float ax = stg[12 + d][r][my_cell];
          const float ay = stg[15 + d][r][my_cell];
          const float az = stg[18 + d][r][my_cell];
          const float cz1 = w[2][1] * az, cz2 = 2.f * w[2][2] * az;  // as in k_p2g
#pragma unroll
          for (int ii = 0; ii < 3; ++ii) {
            const float qi = q + (float)ii * ax;
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) {
              const float qij = qi + (float)jj * ay;
              const float wij = w[0][ii] * w[1][jj];
              const int n = (ii * 3 + jj) * 3;
              acc[n] = fmaf(wij, w[2][0] * qij, acc[n]);
              acc[n + 1] = fmaf(wij, fmaf(w[2][1], qij, cz1), acc[n + 1]);
              acc[n + 2] = fmaf(wij, fmaf(w[2][2], qij, cz2), acc[n + 2]);
            }
          }
        }
        const int cell = cell0 + my_cell;
        const int ex = (cell >> 6) + 1, ey = ((cell >> 3) & 7) + 1, ez = (cell & 7) + 1;
        float *dst = sf + d * kHaloCells;
#pragma unroll
        for (int ii = 0; ii < 3; ++ii)
#pragma unroll
          for (int jj = 0; jj < 3; ++jj)
#pragma unroll
            for (int kk = 0; kk < 3; ++kk)
              atomicAdd(&dst[((ex + ii) * kHalo + (ey + jj)) * kHalo + ez + kk], acc[(ii * 3 + jj) * 3 + kk]);
      }
    }
    __syncthreads();
    // flush: items (hx, hy, quad); four nodes x three components = three 16-byte reductions
    for (int it = t; it < kHalo * kHalo * 3; it += kG2P2GThreads) {
      const int quad = it % 3, hy = (it / 3) % kHalo, hx = it / (3 * kHalo);
      const int h = (hx * kHalo + hy) * kHalo + quad * 4;
      float v[12];
#pragma unroll
      for (int n = 0; n < 4; ++n)
#pragma unroll
        for (int d = 0; d < 3; ++d) v[3 * n + d] = sf[d * kHaloCells + h + n];
      bool any = false;
#pragma unroll
      for (int k = 0; k < 12; ++k) any = any || v[k] != 0.f;
      if (!any) continue;
#pragma unroll
      for (int d = 0; d < 3; ++d) *reinterpret_cast<float4 *>(&sf[d * kHaloCells + h]) = make_float4(0.f, 0.f, 0.f, 0.f);
      const int tb = s.nbr[b * 8 + ((hx >= 8 ? 4 : 0) | (hy >= 8 ? 2 : 0) | (quad == 2 ? 1 : 0))];
      if (tb < 0) {
        set_status(s.ctr, kStatusMissingBlock);
        continue;
      }
      const int cell = ((hx & 7) << 6) | ((hy & 7) << 3) | ((quad * 4) & 7);
      float *dst = fout + ((size_t)tb * 512 + cell) * 3;
      red_add_v4(dst, v[0], v[1], v[2], v[3]);
      red_add_v4(dst + 4, v[4], v[5], v[6], v[7]);
      red_add_v4(dst + 8, v[8], v[9], v[10], v[11]);
    }
  }
}

// dof entries of the active blocks (nb * 512 * 3), or 0 with the capacity status when the
// caller's vectors are shorter
__device__ __forceinline__ long long dof_count(const scene_device &s, long long ndofs) {
  const long long total = (long long)s.ctr[kCtrBlocks] * 1536;
  if (total <= ndofs) return total;
  if (blockIdx.x == 0 && threadIdx.x == 0) set_status(s.ctr, kStatusCapacity);
  return 0;
}

// ImplicitMPMSystem::ForceDtSqrPlusMass (ImplicitMPM.hpp:17-33): where the grid mass of the
// node is positive, out = (f dt^2 + m) dv, with f = out on entry.
__global__ void __launch_bounds__(kThreads) k_implicit_mass(scene_device s, const float *__restrict__ dv,
                                                             float *__restrict__ out, float dt, long long ndofs,
                                                             const int *skip) {
  if (skip && *skip) return;
  const long long total = dof_count(s, ndofs);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += grid_threads()) {
    const long long node = i / 3;
    const float m = s.grid[(node >> 9) * kGridChannels * 512 + (node & 511)];
    if (m > 0.f) out[i] = (out[i] * dt * dt + m) * dv[i];
  }
}

// ImplicitMPMSystem::Projector (ImplicitMPM.hpp:63-97) with the scene's six walls: nodes with
// positive mass get the walls' collision response, all others are zeroed.
__global__ void __launch_bounds__(kThreads) k_implicit_project(scene_device s, float *__restrict__ dof,
                                                                long long ndofs, const int *skip) {
  if (skip && *skip) return;
  const scene_params &p = s.prm;
  const long long total = dof_count(s, ndofs) / 3;
  const int ncol = p.ncolliders ? min(*p.ncolliders, kMaxColliders) : 0;
  const int nls = p.nlevelsets ? min(*p.nlevelsets, kMaxLevelsets) : 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += grid_threads()) {
    const int b = (int)(t >> 9), cell = (int)(t & 511);
    float *v = dof + t * 3;
    if (s.grid[(size_t)b * kGridChannels * 512 + cell] > 0.f) {
      const int3 k = unpack_key(s.blk_pk[b]);
      const float pos[3] = {((float)k.x * 8.f + (float)(cell >> 6)) * p.dx,
                            ((float)k.y * 8.f + (float)((cell >> 3) & 7)) * p.dx,
                            ((float)k.z * 8.f + (float)(cell & 7)) * p.dx};
      float vel[3] = {v[0], v[1], v[2]};
      apply_walls(p, pos, vel);
      if (ncol + nls > 0) apply_colliders(p, ncol, nls, pos, vel);
      v[0] = vel[0];
      v[1] = vel[1];
      v[2] = vel[2];
    } else {
      v[0] = v[1] = v[2] = 0.f;
    }
  }
}

// ImplicitMPMSystem::DivPernodeMass (ImplicitMPM.hpp:126-137): out = in / m where the grid
// mass is positive; other entries of out are left as they are.
__global__ void __launch_bounds__(kThreads) k_implicit_precondition(scene_device s, const float *__restrict__ in,
                                                                     float *__restrict__ out, long long ndofs,
                                                                     const int *skip) {
  if (skip && *skip) return;
  const long long total = dof_count(s, ndofs);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += grid_threads()) {
    const long long node = i / 3;
    const float m = s.grid[(node >> 9) * kGridChannels * 512 + (node & 511)];
    if (m > 0.f) out[i] = in[i] / m;
  }
}

// ConjugateGradient::solve (math/linear/ConjugateGradient.hpp:69-172) on the device.  The
// scalars (r.q, alpha, beta, the stopping test) live in a cg_state in device memory, so no
// step needs the host: every kernel of an iteration returns at once when the iteration's
// check found the solve finished.  Dot products sum float products per thread and warp, and
// the warp sums in double.
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__global__ void __launch_bounds__(kThreads) k_cg_fill0(scene_device s, float *__restrict__ v, long long ndofs,
                                                        const int *skip) {
  if (skip && *skip) return;
  const long long total = dof_count(s, ndofs);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += grid_threads()) v[i] = 0.f;
}

// r = b - Ax (ConjugateGradient.hpp:97-98)
__global__ void __launch_bounds__(kThreads) k_cg_residual(scene_device s, const float *__restrict__ b,
                                                           const float *__restrict__ ax, float *__restrict__ r,
                                                           long long ndofs) {
  const long long total = dof_count(s, ndofs);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += grid_threads())
    r[i] = b[i] - ax[i];
}

__global__ void __launch_bounds__(kThreads) k_cg_copy(scene_device s, const float *__restrict__ src,
                                                       float *__restrict__ dst, long long ndofs) {
  const long long total = dof_count(s, ndofs);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += grid_threads()) dst[i] = src[i];
}

__global__ void __launch_bounds__(kThreads) k_cg_dot(scene_device s, const float *__restrict__ a,
                                                      const float *__restrict__ b, long long ndofs, cg_state *cs) {
  if (cs->done) return;
  const long long total = dof_count(s, ndofs);
  float acc = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += grid_threads())
    acc += a[i] * b[i];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc != 0.f) atomicAdd(&cs->acc, (double)acc);
}

// after the first r.q: the norm and the tolerance min(relTol * norm, tol) (:115-117)
__global__ void k_cg_init(cg_state *cs, float tol, float rel_tol) {
  const float z = (float)cs->acc;
  cs->acc = 0.0;
  cs->ztrk = z;
  cs->norm = sqrtf(z);
  cs->local_tol = fminf(rel_tol * cs->norm, tol);
  cs->iter = 0;
  cs->done = 0;
}

// the loop head (:118-122): stop at the tolerance or after max_iters iterations
__global__ void k_cg_check(cg_state *cs, int max_iters) {
  if (cs->done) return;
  if (cs->iter >= max_iters || cs->norm <= cs->local_tol) cs->done = 1;
}

__global__ void k_cg_alpha(cg_state *cs) {
  if (cs->done) return;
  cs->alpha = cs->ztrk / (float)cs->acc;  // alpha = zTrk / (Ap . p)  (:134)
  cs->acc = 0.0;
}

// x = alpha p + x, r = -alpha Ap + r (:137-143)
__global__ void __launch_bounds__(kThreads) k_cg_update_xr(scene_device s, float *__restrict__ x, float *__restrict__ r,
                                                            const float *__restrict__ p, const float *__restrict__ ap,
                                                            long long ndofs, const cg_state *cs) {
  if (cs->done) return;
  const float alpha = cs->alpha;
  const long long total = dof_count(s, ndofs);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += grid_threads()) {
    x[i] = alpha * p[i] + x[i];
    r[i] = -alpha * ap[i] + r[i];
  }
}

// zTrk = q.r, beta = zTrk / zTrkLast, norm = sqrt(zTrk), one iteration done (:156-170)
__global__ void k_cg_beta(cg_state *cs) {
  if (cs->done) return;
  const float last = cs->ztrk;
  cs->ztrk = (float)cs->acc;
  cs->acc = 0.0;
  cs->beta = cs->ztrk / last;
  cs->norm = sqrtf(cs->ztrk);
  cs->iter += 1;
}

// p = beta p + q (:163)
__global__ void __launch_bounds__(kThreads) k_cg_update_p(scene_device s, float *__restrict__ p,
                                                           const float *__restrict__ q, long long ndofs,
                                                           const cg_state *cs) {
  if (cs->done) return;
  const float beta = cs->beta;
  const long long total = dof_count(s, ndofs);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += grid_threads())
    p[i] = beta * p[i] + q[i];
}

// ----------------------------------------------------------------- import / export
// scene of upload index i: the last scene whose start is <= i
__device__ __forceinline__ int scene_of_index(const scene_params &p, int i) {
  int lo = 0, hi = p.nscenes;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (p.scene_start[mid] <= i) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void k_import(scene_device s, const float *m, const float *x, const float *v,
                         const float *C, const float *F, const float *pl, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += grid_threads()) {
    int model = s.prm.mat.model;
    if (s.prm.batch) {
      const int sc = scene_of_index(s.prm, i);
      s.cur.sid[i] = sc;
      model = s.prm.mats[sc].model;
    }
    const float plastic_default = model == 2 ? 1.f : 0.f;
    s.cur.xm[i] = make_float4(x[3 * i], x[3 * i + 1], x[3 * i + 2], m[i]);
    s.cur.v[i] = v ? make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      s.cur.C[mat_at(k, i)] = C ? C[9 * (size_t)i + k] : 0.f;
      s.cur.F[mat_at(k, i)] = F ? F[9 * (size_t)i + k] : ((k & 3) == 0 ? 1.f : 0.f);
    }
    if (s.cur.plastic) s.cur.plastic[i] = pl ? pl[i] : plastic_default;
    s.cur.id[i] = i;
  }
}

__global__ void k_import_tv(scene_device s, const float *base, int nchn, int om, int ox, int ov,
                            int oC, int oF, int opl, int n) {
  const float plastic_default = s.prm.mat.model == 2 ? 1.f : 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += grid_threads()) {
    const size_t tile = (size_t)(i / 32) * nchn * 32 + (i % 32);
    auto at = [&](int chn) { return base[tile + (size_t)chn * 32]; };
    s.cur.xm[i] = make_float4(at(ox), at(ox + 1), at(ox + 2), at(om));
    s.cur.v[i] = ov >= 0 ? make_float4(at(ov), at(ov + 1), at(ov + 2), 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      s.cur.C[mat_at(k, i)] = oC >= 0 ? at(oC + k) : 0.f;
      s.cur.F[mat_at(k, i)] = oF >= 0 ? at(oF + k) : ((k & 3) == 0 ? 1.f : 0.f);
    }
    if (s.cur.plastic) s.cur.plastic[i] = opl >= 0 ? at(opl) : plastic_default;
    s.cur.id[i] = i;
  }
}

// stress of the stored state; A = m C - kappa tau (what the previous G2P would have written)
__global__ void k_prime(scene_device s) {
  if (blockIdx.x == 0 && threadIdx.x == 0) s.ctr[kCtrMaskFrom] = 0;  // new particles: no move masks
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.prm.n; i += grid_threads()) {
    float F[9], tau[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = s.cur.F[mat_at(k, i)];
    float pl = s.cur.plastic ? s.cur.plastic[i] : 0.f;
    if (s.prm.batch)
      constitutive(s.prm.mats[s.cur.sid[i]], F, pl, tau);
    else
      constitutive(s.prm.mat, F, pl, tau);
    const float m = s.cur.xm[i].w;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      s.cur.F[mat_at(k, i)] = F[k];
      s.cur.A[mat_at(k, i)] = m * s.cur.C[mat_at(k, i)] - s.prm.kappa * tau[k];
    }
    if (s.cur.plastic) s.cur.plastic[i] = pl;
  }
}

__global__ void k_export(scene_device s, float *m, float *x, float *v, float *C, float *F, float *pl) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.prm.n; i += grid_threads()) {
    const int o = s.cur.id[i];
    const float4 xm = s.cur.xm[i], vv = s.cur.v[i];
    if (m) m[o] = xm.w;
    if (x) {
      x[3 * (size_t)o] = xm.x;
      x[3 * (size_t)o + 1] = xm.y;
      x[3 * (size_t)o + 2] = xm.z;
    }
    if (v) {
      v[3 * (size_t)o] = vv.x;
      v[3 * (size_t)o + 1] = vv.y;
      v[3 * (size_t)o + 2] = vv.z;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      if (C) C[9 * (size_t)o + k] = s.cur.C[mat_at(k, i)];
      if (F) F[9 * (size_t)o + k] = s.cur.F[mat_at(k, i)];
    }
    if (pl) pl[o] = s.cur.plastic ? s.cur.plastic[i] : 0.f;
  }
}

__global__ void k_export_tv(scene_device s, float *base, int nchn, int om, int ox, int ov, int oC,
                            int oF, int opl) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.prm.n; i += grid_threads()) {
    const int o = s.cur.id[i];
    const size_t tile = (size_t)(o / 32) * nchn * 32 + (o % 32);
    auto at = [&](int chn) -> float & { return base[tile + (size_t)chn * 32]; };
    const float4 xm = s.cur.xm[i], vv = s.cur.v[i];
    if (om >= 0) at(om) = xm.w;
    if (ox >= 0) {
      at(ox) = xm.x;
      at(ox + 1) = xm.y;
      at(ox + 2) = xm.z;
    }
    if (ov >= 0) {
      at(ov) = vv.x;
      at(ov + 1) = vv.y;
      at(ov + 2) = vv.z;
    }
    for (int k = 0; k < 9; ++k) {
      if (oC >= 0) at(oC + k) = s.cur.C[mat_at(k, i)];
      if (oF >= 0) at(oF + k) = s.cur.F[mat_at(k, i)];
    }
    if (opl >= 0) at(opl) = s.cur.plastic ? s.cur.plastic[i] : 0.f;
  }
}

__global__ void k_export_order(scene_device s, int *order) {
  // order[slot] = upload id of the particle that the binning placed in `slot`
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < s.prm.n; t += grid_threads())
    order[t] = s.cur.id[s.src[t]];
}

__global__ void k_svd_batch(const float *A, float *U, float *S, float *V, long long count) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count; i += grid_threads()) {
    float a[9], u[9], sg[3], v[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = A[9 * i + k];
    svd3(a, u, sg, v);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      U[9 * i + k] = u[k];
      V[9 * i + k] = v[k];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) S[3 * i + k] = sg[k];
  }
}

__global__ void k_constitutive_batch(material_dev mat, float *F, float *pl, float *tau, long long count) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count; i += grid_threads()) {
    float f[9], t[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = F[9 * i + k];
    float p = pl ? pl[i] : 0.f;
    constitutive(mat, f, p, t);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      F[9 * i + k] = f[k];
      tau[9 * i + k] = t[k];
    }
    if (pl) pl[i] = p;
  }
}

// ----------------------------------------------------------------- allocation-free activation
// Kernels used only by zsmpm_activate_blocks_noalloc (zsmpm_static.cu): particle positions
// come as the reference's Particles "x" layout (3 floats per particle) instead of the
// scene's float4 buffer, and the result is copied out to the caller's arrays.

// Zeroes the bitmap and the status word of the static scratch before a call.
__global__ void __launch_bounds__(kThreads) k_static_reset(scene_device s) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < s.prm.bitmap_cap; w += grid_threads())
    s.bitmap[w] = 0u;
  if (blockIdx.x == 0 && threadIdx.x == 0) s.ctr[kCtrStatus] = 0;
}

// ComputeSparsity over AoS positions, one insert per distinct block key of a warp.
__global__ void __launch_bounds__(kThreads) k_insert_aos(scene_device s, const float *x) {
  const int lane = threadIdx.x & 31;
  const int n = s.prm.n;
  int3 lo = make_int3(0x7fffffff, 0x7fffffff, 0x7fffffff);
  int3 hi = make_int3(-0x7fffffff, -0x7fffffff, -0x7fffffff);
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int warps = grid_threads() >> 5;
  for (int base = warp_global * 32; base < n; base += warps * 32) {
    const int i = base + lane;
    uint64_t key = kEmptyKey - 1 - lane;
    int3 c, b = make_int3(0, 0, 0);
    bool valid = false;
    if (i < n) {
      const float4 pos = make_float4(x[3 * (size_t)i], x[3 * (size_t)i + 1], x[3 * (size_t)i + 2], 0.f);
      if (cell_of(s.prm, pos, c, b)) {
        key = pack_key(b.x, b.y, b.z);
        valid = true;
      } else {
        set_status(s.ctr, kStatusOutOfDomain);
      }
    }
    const unsigned peers = __match_any_sync(kFull, key);
    if (valid && lane == __ffs(peers) - 1) {
      table_insert(s, key, b, &s.ctr[kCtrParticleBlocks], 0);
      lo = make_int3(min(lo.x, b.x), min(lo.y, b.y), min(lo.z, b.z));
      hi = make_int3(max(hi.x, b.x), max(hi.y, b.y), max(hi.z, b.z));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo.x = min(lo.x, __shfl_xor_sync(kFull, lo.x, o));
    lo.y = min(lo.y, __shfl_xor_sync(kFull, lo.y, o));
    lo.z = min(lo.z, __shfl_xor_sync(kFull, lo.z, o));
    hi.x = max(hi.x, __shfl_xor_sync(kFull, hi.x, o));
    hi.y = max(hi.y, __shfl_xor_sync(kFull, hi.y, o));
    hi.z = max(hi.z, __shfl_xor_sync(kFull, hi.z, o));
  }
  if (lane == 0 && lo.x != 0x7fffffff) {
    atomicMin(&s.ctr[kCtrBoxLo + 0], lo.x);
    atomicMin(&s.ctr[kCtrBoxLo + 1], lo.y);
    atomicMin(&s.ctr[kCtrBoxLo + 2], lo.z);
    atomicMax(&s.ctr[kCtrBoxHi + 0], hi.x);
    atomicMax(&s.ctr[kCtrBoxHi + 1], hi.y);
    atomicMax(&s.ctr[kCtrBoxHi + 2], hi.z);
  }
}

// Copies the sorted keys out; count_out = block count, or -1 (table full / capacity /
// bounding box), -2 (more blocks than cap), -3 (a position was NaN/Inf or out of range).
__global__ void __launch_bounds__(kThreads) k_export_keys(scene_device s, int *keys_out, int cap,
                                                           int *count_out) {
  const int st = s.ctr[kCtrStatus];
  const int nb = s.ctr[kCtrBlocks];
  int code = nb;
  if (st & kStatusOutOfDomain) code = -3;
  else if (st & (kStatusTableFull | kStatusCapacity | kStatusBitmap)) code = -1;
  else if (nb > cap) code = -2;
  if (blockIdx.x == 0 && threadIdx.x == 0) *count_out = code;
  if (code < 0) return;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * nb; t += grid_threads())
    keys_out[t] = s.active_keys[t];
}

// SM count of the current device, looked up once per device ordinal.  Two host threads that
// look up the same device at once store the same value, so the atomics need no lock.
constexpr int kMaxDevices = 64;
std::atomic<int> g_num_sms[kMaxDevices];
int num_sms() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) dev = -1;
  int n = dev >= 0 ? g_num_sms[dev].load(std::memory_order_relaxed) : 0;
  if (n <= 0) {
    if (dev < 0 || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
    else
      g_num_sms[dev].store(n, std::memory_order_relaxed);
  }
  return n;
}

}  // namespace

// ----------------------------------------------------------------- launchers
cudaError_t launch_activate(scene_device &s, cudaStream_t st) {
  const int sm = num_sms();
  k_begin<<<sm * 4, kThreads, 0, st>>>(s);
  k_insert_particle_blocks<<<sm * 16, kThreads, 0, st>>>(s);
  k_insert_moved_blocks<<<sm * 2, kThreads, 0, st>>>(s);
  k_enlarge<<<sm * 2, kThreads, 0, st>>>(s);
  k_bitmap_prepare<<<1, 32, 0, st>>>(s);
  k_bitmap_set<<<sm * 2, kThreads, 0, st>>>(s);
  cudaError_t e = device_scan(load_popc{s.bitmap}, &s.ctr[kCtrWords], s.scan_part, s.word_prefix, st);
  if (e != cudaSuccess) return e;
  k_assign_ranks<<<sm * 2, kThreads, 0, st>>>(s);
  k_neighbors<<<sm * 2, kThreads, 0, st>>>(s);
  return cudaGetLastError();
}

// Both binnings are enqueued; each kernel returns at once unless the device counter
// kCtrIncBin (set by the activation) selects its path, so one CUDA graph serves both.
cudaError_t launch_bin(scene_device &s, cudaStream_t st) {
  const int sm = num_sms();
  k_bin_count<<<sm * 16, kThreads, 0, st>>>(s);
  k_inc_map<<<sm, kThreads, 0, st>>>(s);
  k_inc_stayers<<<sm * 8, kThreads, 0, st>>>(s);
  k_inc_movers<<<sm * 4, kThreads, 0, st>>>(s);
  cudaError_t e = device_scan(load_int{s.block_count}, &s.ctr[kCtrBlocks], s.scan_part, s.block_start, st);
  if (e != cudaSuccess) return e;
  k_cell_start<<<sm * 4, 512, 0, st>>>(s);
  k_bin_scatter<<<sm * 16, kThreads, 0, st>>>(s);
  k_inc_place_stayers<<<sm * 8, kThreads, 0, st>>>(s);
  k_inc_place_movers<<<sm * 4, kThreads, 0, st>>>(s);
  k_bin_finalize<<<sm * 3, 512, 0, st>>>(s);
  k_inc_sort<<<sm * 2, kThreads, 0, st>>>(s);
  k_inc_finalize<<<sm * 8, kThreads, 0, st>>>(s);
  return cudaGetLastError();
}

// per-device kernel attributes; called once per scene with its device current, before any
// capture of its launches
cudaError_t prepare_kernels() {
  cudaError_t e = cudaSuccess;
  auto p2g_attrs = [&](const void *fn, int ranks) {
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p2g_smem_bytes(ranks));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  };
  p2g_attrs((const void *)k_p2g<false, 8, 4>, 8);
  p2g_attrs((const void *)k_p2g<false, 12, 3>, 12);
  p2g_attrs((const void *)k_p2g<false, 16, 2>, 16);
  p2g_attrs((const void *)k_p2g<true, 8, 4>, 8);
  p2g_attrs((const void *)k_p2g<true, 12, 3>, 12);
  p2g_attrs((const void *)k_p2g<true, 16, 2>, 16);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_g2p2g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kG2P2GSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_g2p<true, true, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)g2p_smem_bytes(kThreads));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_g2p<true, false, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)g2p_smem_bytes(kThreads));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_g2p<false, true, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)g2p_smem_bytes(kThreads));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_g2p<false, false, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)g2p_smem_bytes(kThreads));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_g2p<false, true, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)g2p_smem_bytes(128));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_g2p<false, false, 128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)g2p_smem_bytes(128));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_g2p<false, false, kThreads, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)g2p_smem_bytes(kThreads));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_g2p<false, false, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)g2p_smem_bytes(128));
}

// the staged P2G kernel of the scene's staging depth (p2g_ranks: 8, 12 or 16; 0 = 12)
template <bool kCell>
static void launch_staged_p2g(scene_device &s, const float *affine, int with_mass, cudaStream_t st) {
  const int ranks = s.prm.p2g_ranks > 0 ? s.prm.p2g_ranks : kP2GRanksDefault;
  const int dflt = ranks == 8 ? 4 : ranks == 16 ? 2 : 3;
  const int grid = num_sms() * (s.prm.p2g_ctas_per_sm > 0 ? s.prm.p2g_ctas_per_sm : dflt);
  if (ranks == 8)
    k_p2g<kCell, 8, 4><<<grid, kP2GThreads, p2g_smem_bytes(8), st>>>(s, affine, with_mass);
  else if (ranks == 16)
    k_p2g<kCell, 16, 2><<<grid, kP2GThreads, p2g_smem_bytes(16), st>>>(s, affine, with_mass);
  else
    k_p2g<kCell, 12, 3><<<grid, kP2GThreads, p2g_smem_bytes(12), st>>>(s, affine, with_mass);
}

cudaError_t launch_p2g(scene_device &s, cudaStream_t st) {
  if (s.prm.transfer == kTransferCell) return launch_p2c2g(s, 0, st);
  launch_staged_p2g<false>(s, s.cur.A, 1, st);
  return cudaGetLastError();
}

// part 0: P2C2GTransfer from the stored affine term; 1 (momentum) and 2 (force): the part's
// affine term is formed first, into the next buffer's A (G2C2P rewrites it)
cudaError_t launch_p2c2g(scene_device &s, int part, cudaStream_t st) {
  const float *affine = s.cur.A;
  if (part != 0) {
    k_cell_affine<<<num_sms() * 4, kThreads, 0, st>>>(s, part, s.nxt.A);
    affine = s.nxt.A;
  }
  launch_staged_p2g<true>(s, affine, part == 2 ? 0 : 1, st);
  return cudaGetLastError();
}

cudaError_t launch_grid_update(scene_device &s, cudaStream_t st) {
  k_grid_update<<<num_sms() * 8, kThreads, 0, st>>>(s);
  k_grid_boundaries<<<num_sms() * 4, kThreads, 0, st>>>(s);
  return cudaGetLastError();
}

// The learned closure's pass over the projections the last learned G2P queued: the network on
// the tensor cores, then k_closure_finish.  It writes F, the affine momentum and the plastic
// state of the queued particles only, and reads the queue counter and the substep number the
// G2P recorded, which the next substep's activation and binning leave alone: so it may run
// beside them (a deferred pass), joining before the next P2G.
cudaError_t launch_closure_pass(scene_device &s, cudaStream_t st) {
  cudaError_t e = launch_closure_rows(s.aux.cd, s.aux.q_feat, s.aux.q_out, &s.ctr[kCtrQueue], s.aux.qcap, st);
  if (e != cudaSuccess) return e;
  k_closure_finish<<<num_sms() * 4, kThreads, 0, st>>>(s);
  return cudaGetLastError();
}

cudaError_t launch_g2p(scene_device &s, cudaStream_t st, bool closure_pass) {
  const int per_sm = s.prm.g2p_ctas_per_sm > 0 ? s.prm.g2p_ctas_per_sm : 3;
  const int grid = num_sms() * per_sm;
  const bool small = s.prm.g2p_threads == 128;
  if (s.prm.transfer == kTransferCell) {
    small ? k_g2p<false, false, 128, true><<<grid, 128, g2p_smem_bytes(128), st>>>(s)
          : k_g2p<false, false, kThreads, true><<<grid, kThreads, g2p_smem_bytes(kThreads), st>>>(s);
    return cudaGetLastError();
  }
  if (s.aux.learned) {
    // G2P queues the projections (from an empty queue), the network runs over the queue on the
    // tensor cores, and k_closure_finish completes the queued particles; closure_pass = false
    // leaves the last two to a deferred launch_closure_pass
    cudaError_t e = cudaMemsetAsync(&s.ctr[kCtrQueue], 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    if (s.prm.batch)
      k_g2p<true, true, kThreads><<<grid, kThreads, g2p_smem_bytes(kThreads), st>>>(s);
    else
      k_g2p<true, false, kThreads><<<grid, kThreads, g2p_smem_bytes(kThreads), st>>>(s);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return closure_pass ? launch_closure_pass(s, st) : cudaSuccess;
  }
  if (s.prm.batch)
    small ? k_g2p<false, true, 128><<<grid, 128, g2p_smem_bytes(128), st>>>(s)
          : k_g2p<false, true, kThreads><<<grid, kThreads, g2p_smem_bytes(kThreads), st>>>(s);
  else
    small ? k_g2p<false, false, 128><<<grid, 128, g2p_smem_bytes(128), st>>>(s)
          : k_g2p<false, false, kThreads><<<grid, kThreads, g2p_smem_bytes(kThreads), st>>>(s);
  return cudaGetLastError();
}

cudaError_t launch_g2p2g(scene_device &s, const float *v, float *f, long long ndofs, float dt, const int *skip,
                         cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(&s.ctr[kCtrWork + kWorkG2P2G], 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  k_g2p2g<<<num_sms() * 2, kG2P2GThreads, kG2P2GSmem, st>>>(s, v, f, ndofs, dt, skip);
  return cudaGetLastError();
}

cudaError_t launch_implicit_mass(scene_device &s, const float *dv, float *out, float dt, long long ndofs,
                                 const int *skip, cudaStream_t st) {
  k_implicit_mass<<<num_sms() * 4, kThreads, 0, st>>>(s, dv, out, dt, ndofs, skip);
  return cudaGetLastError();
}

cudaError_t launch_implicit_project(scene_device &s, float *dof, long long ndofs, const int *skip,
                                    cudaStream_t st) {
  k_implicit_project<<<num_sms() * 4, kThreads, 0, st>>>(s, dof, ndofs, skip);
  return cudaGetLastError();
}

cudaError_t launch_implicit_precondition(scene_device &s, const float *in, float *out, long long ndofs,
                                         const int *skip, cudaStream_t st) {
  k_implicit_precondition<<<num_sms() * 4, kThreads, 0, st>>>(s, in, out, ndofs, skip);
  return cudaGetLastError();
}

// The solve's start: r = b - A x, project r, q = M r (q zeroed first), p = q, zTrk = r.q.
cudaError_t launch_cg_begin(scene_device &s, float *x, const float *b, const cg_vectors &v, long long ndofs, float dt,
                            cg_state *cs, float tol, float rel_tol, cudaStream_t st) {
  const int grid = num_sms() * 4;
  cudaError_t e = cudaMemsetAsync(cs, 0, sizeof(cg_state), st);
  if (e != cudaSuccess) return e;
  k_cg_fill0<<<grid, kThreads, 0, st>>>(s, v.ap, ndofs, nullptr);
  if ((e = launch_g2p2g(s, x, v.ap, ndofs, dt, nullptr, st)) != cudaSuccess) return e;
  if ((e = launch_implicit_mass(s, x, v.ap, dt, ndofs, nullptr, st)) != cudaSuccess) return e;
  k_cg_residual<<<grid, kThreads, 0, st>>>(s, b, v.ap, v.r, ndofs);
  if ((e = launch_implicit_project(s, v.r, ndofs, nullptr, st)) != cudaSuccess) return e;
  k_cg_fill0<<<grid, kThreads, 0, st>>>(s, v.q, ndofs, nullptr);
  if ((e = launch_implicit_precondition(s, v.r, v.q, ndofs, nullptr, st)) != cudaSuccess) return e;
  k_cg_copy<<<grid, kThreads, 0, st>>>(s, v.q, v.p, ndofs);
  k_cg_dot<<<grid, kThreads, 0, st>>>(s, v.r, v.q, ndofs, cs);
  k_cg_init<<<1, 1, 0, st>>>(cs, tol, rel_tol);
  return cudaGetLastError();
}

// One loop iteration (ConjugateGradient.hpp:118-171); does nothing once the solve is done.
cudaError_t launch_cg_iteration(scene_device &s, float *x, const cg_vectors &v, long long ndofs, float dt,
                                cg_state *cs, int max_iters, cudaStream_t st) {
  const int grid = num_sms() * 4;
  const int *done = &cs->done;
  k_cg_check<<<1, 1, 0, st>>>(cs, max_iters);
  k_cg_fill0<<<grid, kThreads, 0, st>>>(s, v.ap, ndofs, done);
  cudaError_t e = launch_g2p2g(s, v.p, v.ap, ndofs, dt, done, st);
  if (e != cudaSuccess) return e;
  if ((e = launch_implicit_mass(s, v.p, v.ap, dt, ndofs, done, st)) != cudaSuccess) return e;
  if ((e = launch_implicit_project(s, v.ap, ndofs, done, st)) != cudaSuccess) return e;
  k_cg_dot<<<grid, kThreads, 0, st>>>(s, v.ap, v.p, ndofs, cs);
  k_cg_alpha<<<1, 1, 0, st>>>(cs);
  k_cg_update_xr<<<grid, kThreads, 0, st>>>(s, x, v.r, v.p, v.ap, ndofs, cs);
  if ((e = launch_implicit_precondition(s, v.r, v.q, ndofs, done, st)) != cudaSuccess) return e;
  k_cg_dot<<<grid, kThreads, 0, st>>>(s, v.q, v.r, ndofs, cs);
  k_cg_beta<<<1, 1, 0, st>>>(cs);
  k_cg_update_p<<<grid, kThreads, 0, st>>>(s, v.p, v.q, ndofs, cs);
  return cudaGetLastError();
}

// k_begin, the two particle-block inserts (one returns at once), enlarge, prepare, set, 3 scans,
// ranks, neighbours; the binning's 14 launches (the full and the incremental path, one of
// which returns at once); p2g; grid update and boundaries; g2p
int kernels_per_substep() { return 11 + 14 + 4; }

cudaError_t launch_import(scene_device &s, const float *m, const float *x, const float *v,
                          const float *C, const float *F, const float *plastic, int n,
                          cudaStream_t st) {
  k_import<<<num_sms() * 4, kThreads, 0, st>>>(s, m, x, v, C, F, plastic, n);
  return cudaGetLastError();
}

cudaError_t launch_import_tilevector(scene_device &s, const float *base, int nchn, int off_m,
                                     int off_x, int off_v, int off_C, int off_F, int off_pl,
                                     int n, cudaStream_t st) {
  k_import_tv<<<num_sms() * 4, kThreads, 0, st>>>(s, base, nchn, off_m, off_x, off_v, off_C, off_F,
                                                  off_pl, n);
  return cudaGetLastError();
}

cudaError_t launch_prime(scene_device &s, cudaStream_t st) {
  if (s.prm.transfer == kTransferCell)
    k_cell_affine<<<num_sms() * 4, kThreads, 0, st>>>(s, 0, s.cur.A);
  else
    k_prime<<<num_sms() * 4, kThreads, 0, st>>>(s);
  return cudaGetLastError();
}

cudaError_t launch_export(const scene_device &s, float *m, float *x, float *v, float *C,
                          float *F, float *plastic, cudaStream_t st) {
  k_export<<<num_sms() * 4, kThreads, 0, st>>>(s, m, x, v, C, F, plastic);
  return cudaGetLastError();
}

cudaError_t launch_export_tilevector(const scene_device &s, float *base, int nchn, int off_m,
                                     int off_x, int off_v, int off_C, int off_F, int off_pl,
                                     cudaStream_t st) {
  k_export_tv<<<num_sms() * 4, kThreads, 0, st>>>(s, base, nchn, off_m, off_x, off_v, off_C, off_F,
                                                  off_pl);
  return cudaGetLastError();
}

cudaError_t launch_export_order(const scene_device &s, int *order, cudaStream_t st) {
  k_export_order<<<num_sms() * 4, kThreads, 0, st>>>(s, order);
  return cudaGetLastError();
}

cudaError_t launch_activate_static(scene_device &s, const float *x, int *keys_out, int cap,
                                   int *count_out, cudaStream_t st) {
  const int sm = num_sms();
  k_static_reset<<<sm, kThreads, 0, st>>>(s);
  k_begin<<<sm * 4, kThreads, 0, st>>>(s);
  k_insert_aos<<<sm * 8, kThreads, 0, st>>>(s, x);
  k_enlarge<<<sm * 2, kThreads, 0, st>>>(s);
  k_bitmap_prepare<<<1, 32, 0, st>>>(s);
  k_bitmap_set<<<sm * 2, kThreads, 0, st>>>(s);
  cudaError_t e = device_scan(load_popc{s.bitmap}, &s.ctr[kCtrWords], s.scan_part, s.word_prefix, st);
  if (e != cudaSuccess) return e;
  k_assign_ranks<<<sm * 2, kThreads, 0, st>>>(s);
  k_export_keys<<<sm, kThreads, 0, st>>>(s, keys_out, cap, count_out);
  return cudaGetLastError();
}

cudaError_t launch_exclusive_scan(const int *in, const int *n_ptr, int *part, int *out, cudaStream_t st) {
  return device_scan(load_int{in}, n_ptr, part, out, st);
}

cudaError_t launch_svd_batch(const float *A, float *U, float *S, float *V, long long count,
                             cudaStream_t st) {
  k_svd_batch<<<num_sms() * 4, kThreads, 0, st>>>(A, U, S, V, count);
  return cudaGetLastError();
}

cudaError_t launch_constitutive_batch(const material_dev &mat, float *F, float *plastic,
                                      float *tau, long long count, cudaStream_t st) {
  k_constitutive_batch<<<num_sms() * 4, kThreads, 0, st>>>(mat, F, plastic, tau, count);
  return cudaGetLastError();
}

}  // namespace zsmpm
