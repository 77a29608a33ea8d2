// bht<i32,3,int,16> layout of the active block keys (container/Bht.hpp): the bucketed
// three-hash table that zpc's SparseGrid uses where the legacy operators use HashTable.
//
// The table is built on the host, as the reference's host BHTView::insert (Bht.hpp:612-665)
// builds it when the keys are inserted in canonical order with default insertion indices:
// index == the block's rank, so a caller's bht queries return the library's block indices.
// Rules restated from the reference:
//   size      evaluateTableSize(n) = next_2pow(n) * 2, then + (16 - size % 16)   (Bht.hpp:154-158)
//   hashers   three universal hashes seeded by std::mt19937(2): hashx = rng() % p (at least 1),
//             hashy = rng() % p, p = 4294967291 (Bht.hpp:165-169, Bcht.hpp:38-43)
//   hash      per component ((hashx ^ k) + hashy) % p in 32-bit arithmetic, combined by the
//             32-bit hash_combine (py_interop/HashUtils.hpp:22-40, math/Hash.hpp:17-27)
//   insert    bucket hf0(key) % (size / 16) * 16: the first empty slot if its position is at most
//             14 (threshold = bucket_size - 2), else the next hasher's bucket, three tries
//   storage   16-byte keys (x, y, z, pad) byte-filled with 0x3f when empty; status -1
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

}  // namespace

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

}  // extern "C"
