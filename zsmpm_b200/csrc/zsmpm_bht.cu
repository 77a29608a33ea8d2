// bht<i32,3,int,16> layout of the active block keys (container/Bht.hpp): the bucketed
// three-hash table that zpc's SparseGrid uses where the legacy operators use HashTable.
//
// The table is the one the reference's host BHTView::insert (Bht.hpp:612-665) builds when the
// keys are inserted in canonical order with default insertion indices: index == the block's
// rank, so a caller's bht queries return the library's block indices.  Rules restated from the
// reference:
//   size      evaluateTableSize(n) = next_2pow(n) * 2, then + (16 - size % 16)   (Bht.hpp:154-158)
//   hashers   three universal hashes seeded by std::mt19937(2): hashx = rng() % p (at least 1),
//             hashy = rng() % p, p = 4294967291 (Bht.hpp:165-169, Bcht.hpp:38-43)
//   hash      per component ((hashx ^ k) + hashy) % p in 32-bit arithmetic, combined by the
//             32-bit hash_combine (py_interop/HashUtils.hpp:22-40, math/Hash.hpp:17-27)
//   insert    bucket hf0(key) % (size / 16) * 16: the first empty slot if its position is at most
//             14 (threshold = bucket_size - 2), else the next hasher's bucket, three tries
//   storage   16-byte keys (x, y, z, pad) byte-filled with 0x3f when empty; status -1
//
// Two builders give the same table.  zsmpm_bht_build_host inserts one key after the other, as
// the reference does.  The device builder (bht_build_device, used by zsmpm_get_bht_view and
// zsmpm_bht_build_device) places all keys at once: under insertion in order, a key's slot is
// the number of earlier keys in the bucket it settles in, and the bucket it settles in is the
// first of its three whose count of earlier keys is at most the threshold.  Each key's choice
// therefore depends only on the choices of earlier keys, so the parallel iteration
//     choice(k) <- first c with #{j < k : bucket(j) = bucket_c(k)} <= 14
// (all keys updated from the previous iteration's choices) reaches the sequential choices of
// keys 0..t-1 after t iterations and stops, unchanged, exactly at them: a fixed point of the
// update is the sequential table.  It converges in a few iterations (a chain of overflows is
// short); after kDeviceIterations without convergence a one-thread kernel inserts the keys in
// order instead.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "zsmpm.h"
#include "zsmpm_internal.h"

namespace {

constexpr uint32_t kPrime = 4294967291u;
constexpr int kBucket = 16;
constexpr int kThreshold = kBucket - 2;
constexpr int32_t kKeySentinel = 0x3f3f3f3f;

struct hasher {
  uint32_t x, y;
  uint32_t component(int32_t k) const { return ((x ^ (uint32_t)k) + y) % kPrime; }
  uint32_t operator()(const int32_t *key) const {
    uint32_t r = component(key[0]);
    for (int d = 1; d < 3; ++d) r ^= component(key[d]) + 0x9e3779b9u + (r << 6) + (r >> 2);
    return r;
  }
};

void make_hashers(hasher hf[3]) {
  std::mt19937 rng(2);
  for (int k = 0; k < 3; ++k) {
    uint32_t x = (uint32_t)(rng() % kPrime);
    if (x < 1) x = 1;
    const uint32_t y = (uint32_t)(rng() % kPrime);
    hf[k] = {x, y};
  }
}

int64_t table_size_for(int64_t n) {
  if (n <= 0) return 0;
  int64_t p = 1;
  while (p < n) p <<= 1;
  const int64_t s = p * 2;
  return s + (kBucket - s % kBucket);
}

// keys [n][3] -> table arrays; returns the number of keys that found no slot
int build(const int32_t *keys, int64_t n, int64_t size, const hasher hf[3], int32_t *tkeys /* [size][4] */,
          int32_t *indices, int32_t *status) {
  for (int64_t i = 0; i < 4 * size; ++i) tkeys[i] = kKeySentinel;
  for (int64_t i = 0; i < size; ++i) {
    indices[i] = -1;
    status[i] = -1;
  }
  const uint32_t buckets = (uint32_t)(size / kBucket);
  int failed = 0;
  int32_t next_index = 0;
  for (int64_t k = 0; k < n; ++k) {
    const int32_t *key = keys + 3 * k;
    bool placed = false;
    for (int h = 0; h < 3 && !placed && buckets; ++h) {
      const int64_t off = (int64_t)(hf[h](key) % buckets) * kBucket;
      int load = 0;
      bool exists = false;
      for (; load < kBucket; ++load) {
        const int32_t *sk = tkeys + 4 * (off + load);
        if (sk[0] == key[0] && sk[1] == key[1] && sk[2] == key[2]) {
          exists = true;
          break;
        }
        if (sk[0] == kKeySentinel && sk[1] == kKeySentinel && sk[2] == kKeySentinel) break;
      }
      if (exists) {
        placed = true;
        break;
      }
      if (load <= kThreshold) {
        int32_t *sk = tkeys + 4 * (off + load);
        sk[0] = key[0];
        sk[1] = key[1];
        sk[2] = key[2];
        indices[off + load] = next_index++;
        placed = true;
      }
    }
    if (!placed) ++failed;
  }
  return failed;
}

zsmpm_status berr(zsmpm_status st, const std::string &m) {
  return (zsmpm_status)zsmpm::record_error(st, m.c_str());
}

// ---------------------------------------------------------------- the device builder
struct dhasher {
  uint32_t x[3], y[3];
};

__device__ __forceinline__ uint32_t dhash(const dhasher &h, int c, const int32_t *key) {
  uint32_t r = ((h.x[c] ^ (uint32_t)key[0]) + h.y[c]) % kPrime;
  for (int d = 1; d < 3; ++d) r ^= (((h.x[c] ^ (uint32_t)key[d]) + h.y[c]) % kPrime) + 0x9e3779b9u + (r << 6) + (r >> 2);
  return r;
}

__device__ __forceinline__ int grid_threads_b() { return gridDim.x * blockDim.x; }

__global__ void k_bht_reset(int32_t *tkeys, int32_t *indices, int32_t *status, int64_t size) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < size; i += grid_threads_b()) {
    reinterpret_cast<int4 *>(tkeys)[i] = make_int4(kKeySentinel, kKeySentinel, kKeySentinel, kKeySentinel);
    indices[i] = -1;
    status[i] = -1;
  }
}

// the three candidate buckets of every key; every key starts on its first
__global__ void k_bht_candidates(const int32_t *keys, int n, dhasher h, uint32_t buckets, int *cand, int *choice,
                                 int32_t *active) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += grid_threads_b()) {
    for (int c = 0; c < 3; ++c) cand[3 * k + c] = (int)(dhash(h, c, keys + 3 * k) % buckets);
    choice[k] = 0;
    for (int d = 0; d < 3; ++d) active[3 * k + d] = keys[3 * k + d];
  }
}

__global__ void k_bht_count(const int *cand, const int *choice, int n, int *count) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += grid_threads_b())
    if (choice[k] < 3) atomicAdd(&count[cand[3 * k + choice[k]]], 1);
}

__global__ void k_bht_fill(const int *cand, const int *choice, int n, const int *start, int *fill, int *list) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += grid_threads_b())
    if (choice[k] < 3) {
      const int b = cand[3 * k + choice[k]];
      list[start[b] + atomicAdd(&fill[b], 1)] = k;
    }
}

// each bucket's members in insertion order
__global__ void k_bht_sort(const int *start, int buckets, int *list) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < buckets; b += grid_threads_b()) {
    const int lo = start[b], hi = start[b + 1];
    for (int i = lo + 1; i < hi; ++i) {
      const int v = list[i];
      int j = i;
      while (j > lo && list[j - 1] > v) {
        list[j] = list[j - 1];
        --j;
      }
      list[j] = v;
    }
  }
}

// members of bucket b inserted before key k
__device__ __forceinline__ int earlier_in(const int *start, const int *list, int b, int k) {
  int lo = start[b], hi = start[b + 1];
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (list[mid] < k) lo = mid + 1;
    else hi = mid;
  }
  return lo - start[b];
}

__global__ void k_bht_choose(const int *cand, const int *choice, int n, const int *start, const int *list,
                             int *choice_next, int *changed) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += grid_threads_b()) {
    int c = 0;
    for (; c < 3; ++c)
      if (earlier_in(start, list, cand[3 * k + c], k) <= kThreshold) break;
    choice_next[k] = c;  // 3: no free slot in its three buckets
    if (c != choice[k]) atomicOr(changed, 1);
  }
}

__global__ void k_bht_place(const int32_t *keys, const int *cand, const int *choice, int n, const int *start,
                            const int *list, int32_t *tkeys, int32_t *indices, int *failed) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += grid_threads_b()) {
    if (choice[k] >= 3) {
      atomicOr(failed, 1);
      continue;
    }
    const int b = cand[3 * k + choice[k]];
    const int64_t slot = (int64_t)b * kBucket + earlier_in(start, list, b, k);
    tkeys[4 * slot + 0] = keys[3 * k + 0];
    tkeys[4 * slot + 1] = keys[3 * k + 1];
    tkeys[4 * slot + 2] = keys[3 * k + 2];
    indices[slot] = k;
  }
}

// insertion one key after the other (Bht.hpp:612-665), for the rare input on which the
// iteration has not settled
__global__ void k_bht_sequential(const int32_t *keys, int n, dhasher h, uint32_t buckets, int32_t *tkeys,
                                 int32_t *indices, int *failed) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int32_t next = 0;
  for (int k = 0; k < n; ++k) {
    const int32_t *key = keys + 3 * k;
    bool placed = false;
    for (int c = 0; c < 3 && !placed; ++c) {
      const int64_t off = (int64_t)(dhash(h, c, key) % buckets) * kBucket;
      int load = 0;
      for (; load < kBucket; ++load) {
        const int32_t *sk = tkeys + 4 * (off + load);
        if (sk[0] == key[0] && sk[1] == key[1] && sk[2] == key[2]) {
          placed = true;
          break;
        }
        if (sk[0] == kKeySentinel && sk[1] == kKeySentinel && sk[2] == kKeySentinel) break;
      }
      if (!placed && load <= kThreshold) {
        int32_t *sk = tkeys + 4 * (off + load);
        sk[0] = key[0];
        sk[1] = key[1];
        sk[2] = key[2];
        indices[off + load] = next++;
        placed = true;
      }
    }
    if (!placed) *failed = 1;
  }
}

__global__ void k_bht_finish(int n, const int *failed, int32_t *cnt_success) {
  cnt_success[0] = n;
  cnt_success[1] = *failed ? 0 : 1;
}

constexpr int kDeviceIterations = 32;

}  // namespace

namespace zsmpm {

// Builds the bht of keys[n][3] (device) into tkeys [size][4], indices and status [size]
// (device), writes active[n][3] and cnt_success[2] = (n, success); `size` from
// table_size_for.  Scratch is allocated here.  Returns ZSMPM_ERR_TABLE_FULL when a key found no
// slot (cnt_success[1] = 0 then).
int bht_build_device(const int32_t *keys, int n, int64_t size, int32_t *tkeys, int32_t *indices, int32_t *status,
                     int32_t *active, int32_t *cnt_success, uint32_t *hashers_out, cudaStream_t st) {
  hasher hf[3];
  make_hashers(hf);
  dhasher dh{};
  for (int k = 0; k < 3; ++k) {
    dh.x[k] = hf[k].x;
    dh.y[k] = hf[k].y;
    if (hashers_out) {
      hashers_out[2 * k] = hf[k].x;
      hashers_out[2 * k + 1] = hf[k].y;
    }
  }
  const uint32_t buckets = (uint32_t)(size / kBucket);
  const int grid = 1024;
  k_bht_reset<<<grid, 256, 0, st>>>(tkeys, indices, status, size);
  // scratch: cand[3n], choice[2][n], list[n], count[B], start[B + 1], fill[B], flags[2], nB[1],
  // scan partials
  const size_t nn = (size_t)std::max(n, 1), bb = (size_t)std::max<uint32_t>(buckets, 1);
  const size_t words = 3 * nn + 2 * nn + nn + bb + (bb + 1) + bb + 2 + 1 + (2 * kScanCtas + 1);
  int *scratch = nullptr;
  cudaError_t e = cudaMalloc(&scratch, sizeof(int) * words);
  if (e != cudaSuccess) return record_error(ZSMPM_ERR_CUDA, "bht scratch allocation");
  int *cand = scratch, *choice = cand + 3 * nn, *choice2 = choice + nn, *list = choice2 + nn, *count = list + nn,
      *start = count + bb, *fill = start + bb + 1, *flags = fill + bb, *nB = flags + 2, *part = nB + 1;
  const int nbuckets = (int)buckets;
  int status_code = ZSMPM_OK;
  auto fail_cuda = [&](const char *what) {
    status_code = record_error(ZSMPM_ERR_CUDA, (std::string("bht device build: ") + what + ": " +
                                                cudaGetErrorString(e)).c_str());
  };
  do {
    if ((e = cudaMemcpyAsync(nB, &nbuckets, sizeof(int), cudaMemcpyHostToDevice, st)) != cudaSuccess) {
      fail_cuda("bucket count");
      break;
    }
    if ((e = cudaMemsetAsync(flags, 0, sizeof(int) * 2, st)) != cudaSuccess) {
      fail_cuda("flags");
      break;
    }
    if (n == 0 || buckets == 0) {
      if (n > 0) cudaMemsetAsync(flags + 1, 0xff, sizeof(int), st);  // keys but no buckets: failed
      break;
    }
    k_bht_candidates<<<grid, 256, 0, st>>>(keys, n, dh, buckets, cand, choice, active);
    bool converged = false;
    for (int it = 0; it < kDeviceIterations && !converged; ++it) {
      cudaMemsetAsync(count, 0, sizeof(int) * bb, st);
      cudaMemsetAsync(fill, 0, sizeof(int) * bb, st);
      cudaMemsetAsync(flags, 0, sizeof(int), st);
      k_bht_count<<<grid, 256, 0, st>>>(cand, choice, n, count);
      if ((e = launch_exclusive_scan(count, nB, part, start, st)) != cudaSuccess) break;
      k_bht_fill<<<grid, 256, 0, st>>>(cand, choice, n, start, fill, list);
      k_bht_sort<<<grid, 256, 0, st>>>(start, nbuckets, list);
      k_bht_choose<<<grid, 256, 0, st>>>(cand, choice, n, start, list, choice2, flags);
      int changed = 0;
      if ((e = cudaMemcpyAsync(&changed, flags, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess) break;
      if ((e = cudaStreamSynchronize(st)) != cudaSuccess) break;
      std::swap(choice, choice2);
      converged = changed == 0;
    }
    if (e != cudaSuccess) {
      fail_cuda("iteration");
      break;
    }
    if (converged) {
      // the lists of the last iteration belong to these (unchanged) choices
      k_bht_place<<<grid, 256, 0, st>>>(keys, cand, choice, n, start, list, tkeys, indices, flags + 1);
    } else {
      k_bht_reset<<<grid, 256, 0, st>>>(tkeys, indices, status, size);
      k_bht_sequential<<<1, 32, 0, st>>>(keys, n, dh, buckets, tkeys, indices, flags + 1);
    }
  } while (false);
  if (status_code == ZSMPM_OK) {
    k_bht_finish<<<1, 1, 0, st>>>(n, flags + 1, cnt_success);
    int failed = 0;
    e = cudaMemcpyAsync(&failed, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
      fail_cuda("finish");
    else if (failed)
      status_code = record_error(ZSMPM_ERR_TABLE_FULL, "a key found no free slot in its three buckets");
  }
  cudaStreamSynchronize(st);
  cudaFree(scratch);
  return status_code;
}

int64_t bht_table_size(int64_t n) { return table_size_for(n); }

}  // namespace zsmpm


extern "C" {

ZSMPM_API zsmpm_status zsmpm_bht_build_host(const int32_t *keys, int32_t nkeys, int32_t expected,
                                            int32_t *table_keys, int32_t *indices, int32_t *status,
                                            int32_t cap_slots, int32_t *table_size, uint32_t *hashers) {
  if (nkeys < 0 || (nkeys > 0 && !keys) || !table_size) return berr(ZSMPM_ERR_INVALID_ARG, "bad bht arguments");
  const int64_t size = table_size_for(expected > 0 ? expected : nkeys);
  *table_size = (int32_t)size;
  hasher hf[3];
  make_hashers(hf);
  if (hashers)
    for (int k = 0; k < 3; ++k) {
      hashers[2 * k] = hf[k].x;
      hashers[2 * k + 1] = hf[k].y;
    }
  if (size > cap_slots || !table_keys || !indices || !status)
    return berr(ZSMPM_ERR_CAPACITY, "bht output arrays smaller than the table size");
  // Bht.hpp:640-644: an insertion index at or above size - 20 fails the build
  if (nkeys > 0 && (int64_t)nkeys - 1 >= size - 20)
    return berr(ZSMPM_ERR_TABLE_FULL, "bht table too small for the keys");
  if (build(keys, nkeys, size, hf, table_keys, indices, status) != 0)
    return berr(ZSMPM_ERR_TABLE_FULL, "a key found no free slot in its three buckets");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_bht_build_device(const int32_t *keys, int32_t nkeys, int32_t expected,
                                              int32_t *table_keys, int32_t *indices, int32_t *status,
                                              int32_t cap_slots, int32_t *table_size, uint32_t *hashers,
                                              void *stream) {
  if (nkeys < 0 || (nkeys > 0 && !keys) || !table_size) return berr(ZSMPM_ERR_INVALID_ARG, "bad bht arguments");
  const int64_t size = table_size_for(expected > 0 ? expected : nkeys);
  *table_size = (int32_t)size;
  if (size > cap_slots || !table_keys || !indices || !status)
    return berr(ZSMPM_ERR_CAPACITY, "bht output arrays smaller than the table size");
  if (nkeys > 0 && (int64_t)nkeys - 1 >= size - 20)
    return berr(ZSMPM_ERR_TABLE_FULL, "bht table too small for the keys");
  int32_t *extra = nullptr;  // active keys and (cnt, success), not returned by this entry point
  if (cudaMalloc(&extra, sizeof(int32_t) * (3 * (size_t)std::max(nkeys, 1) + 2)) != cudaSuccess)
    return berr(ZSMPM_ERR_CUDA, "bht scratch allocation");
  const int st = zsmpm::bht_build_device(keys, nkeys, size, table_keys, indices, status, extra,
                                         extra + 3 * (size_t)std::max(nkeys, 1), hashers,
                                         static_cast<cudaStream_t>(stream));
  cudaFree(extra);
  return (zsmpm_status)st;
}

}  // extern "C"
