/* Test infrastructure (oracle): integer parts of the restatement shared by both precisions
 * -- the reference's hash table (container/HashTable.hpp) and block activation
 * (simulation/sparsity/SparsityOp.hpp), plus the restated binning order of the CUDA path.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "oracle_internal.h"

/* math/Hash.hpp:17-27 with a 64-bit seed: seed ^= val + 0x9e3779b97f4a7c15 + (seed<<12) +
 * (seed>>4), val sign-extended; HashTable.hpp:493-500 starts from key[0] and truncates
 * the 64-bit result to the 32-bit value type. */
int32_t oracle_do_hash(int32_t kx, int32_t ky, int32_t kz) {
  uint64_t seed = (uint64_t)(int64_t)kx;
  seed ^= ((uint64_t)(int64_t)ky + 0x9e3779b97f4a7c15ull + (seed << 12) + (seed >> 4));
  seed ^= ((uint64_t)(int64_t)kz + 0x9e3779b97f4a7c15ull + (seed << 12) + (seed >> 4));
  return (int32_t)(uint32_t)seed;
}

int32_t oracle_hash_slot(int32_t kx, int32_t ky, int32_t kz, int32_t table_size) {
  int32_t h = oracle_do_hash(kx, ky, kz);
  return (h % table_size + table_size) % table_size;
}

static int64_t next_2pow(int64_t n) {
  int64_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

int oracle_table_init(oracle_table *t, int expected) {
  if (expected < 1) expected = 1;
  t->size = (int32_t)(next_2pow(expected) * 16); /* HashTable.hpp:88-91 */
  t->keys = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)t->size);
  t->index = (int32_t *)malloc(sizeof(int32_t) * (size_t)t->size);
  t->active = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)t->size);
  oracle_table_clear(t);
  return t->keys && t->index && t->active ? 0 : 1;
}

void oracle_table_free(oracle_table *t) {
  free(t->keys);
  free(t->index);
  free(t->active);
  memset(t, 0, sizeof(*t));
}

/* CleanSparsity (SparsityOp.hpp:41-55): keys to INT_MAX, index to -1, count to 0 */
void oracle_table_clear(oracle_table *t) {
  for (int32_t i = 0; i != t->size; ++i) {
    t->keys[3 * i] = t->keys[3 * i + 1] = t->keys[3 * i + 2] = INT32_MAX;
    t->index[i] = -1;
  }
  t->count = 0;
}

/* Sequential insert (HashTable.hpp:376-398): linear probe with stride 127; a new key gets
 * index = count++ unless `id` >= 0 is given (ReinsertHashTable form, :232-239).  Returns
 * the slot, or -1 when the table is full. */
int32_t oracle_table_insert(oracle_table *t, const int32_t k[3], int32_t id) {
  int32_t slot = oracle_hash_slot(k[0], k[1], k[2], t->size);
  for (int32_t probes = 0; probes < t->size; ++probes) {
    int32_t *s = &t->keys[3 * slot];
    if (s[0] == INT32_MAX && s[1] == INT32_MAX && s[2] == INT32_MAX) {
      s[0] = k[0];
      s[1] = k[1];
      s[2] = k[2];
      if (id < 0) {
        id = t->count++;
        t->active[3 * id] = k[0];
        t->active[3 * id + 1] = k[1];
        t->active[3 * id + 2] = k[2];
      }
      t->index[slot] = id;
      return slot;
    }
    if (s[0] == k[0] && s[1] == k[1] && s[2] == k[2]) return slot;
    slot = (slot + 127) % t->size;
  }
  return -1;
}

/* query (HashTable.hpp:444-456); the probe wraps with the insert rule (slot+127) % T. */
int32_t oracle_table_query(const oracle_table *t, const int32_t k[3]) {
  int32_t slot = oracle_hash_slot(k[0], k[1], k[2], t->size);
  for (int32_t probes = 0; probes < t->size; ++probes) {
    const int32_t *s = &t->keys[3 * slot];
    if (s[0] == k[0] && s[1] == k[1] && s[2] == k[2]) return t->index[slot];
    if (t->index[slot] == -1) return -1;
    slot = (slot + 127) % t->size;
  }
  return -1;
}

/* ComputeSparsity (SparsityOp.hpp:70-79): coord = floor(x * (1/dx) + 0.5) - 2, then
 * floor division by the block side 8 written as (coord + (coord<0 ? -7 : 0)) / 8. */
void oracle_block_of(const float x[3], float dxinv, int32_t out[3]) {
  for (int d = 0; d != 3; ++d) {
    int32_t c = (int32_t)floorf(x[d] * dxinv + 0.5f) - 2;
    out[d] = (c + (c < 0 ? -7 : 0)) / 8;
  }
}

int oracle_activate_table(oracle_table *t, int n, const float *x, float dx, int *nparblocks) {
  const float dxinv = 1.f / dx;
  oracle_table_clear(t);
  for (int i = 0; i != n; ++i) {
    int32_t b[3];
    oracle_block_of(&x[3 * i], dxinv, b);
    if (oracle_table_insert(t, b, -1) < 0) return 2;
  }
  const int npb = t->count;
  if (nparblocks) *nparblocks = npb;
  for (int i = 0; i != npb; ++i) {
    const int32_t *k = &t->active[3 * i];
    for (int a = 0; a != 2; ++a)
      for (int b = 0; b != 2; ++b)
        for (int c = 0; c != 2; ++c) {
          int32_t nk[3] = {k[0] + a, k[1] + b, k[2] + c};
          if (oracle_table_insert(t, nk, -1) < 0) return 2;
        }
  }
  if (t->count >= t->size - 20) return 2;
  return 0;
}

static int key_less(const int32_t *a, const int32_t *b) {
  for (int d = 0; d != 3; ++d)
    if (a[d] != b[d]) return a[d] < b[d];
  return 0;
}
static int key_cmp(const void *pa, const void *pb) {
  const int32_t *a = (const int32_t *)pa, *b = (const int32_t *)pb;
  return key_less(a, b) ? -1 : (key_less(b, a) ? 1 : 0);
}

/* Canonical order: sort the active keys ascending and rebuild the table with
 * index == sorted position (ResetHashTable + ReinsertHashTable, HashTable.hpp:215-247). */
void oracle_table_canonicalize(oracle_table *t) {
  const int nb = t->count;
  qsort(t->active, (size_t)nb, sizeof(int32_t) * 3, key_cmp);
  for (int32_t i = 0; i != t->size; ++i) {
    t->keys[3 * i] = t->keys[3 * i + 1] = t->keys[3 * i + 2] = INT32_MAX;
    t->index[i] = -1;
  }
  for (int i = 0; i != nb; ++i) oracle_table_insert(t, &t->active[3 * i], i);
}

int oracle_activate(int n, const float *x, float dx, int table_expected, int cap,
                    int *out_nblocks, int *out_nparblocks, int *out_keys, int *out_slots,
                    int *out_table_size) {
  oracle_table t;
  if (oracle_table_init(&t, table_expected)) return 3;
  int npb = 0;
  int st = oracle_activate_table(&t, n, x, dx, &npb);
  *out_nblocks = t.count;
  *out_nparblocks = npb;
  *out_table_size = t.size;
  if (st == 0 && t.count > cap) st = 1;
  if (st == 0)
    for (int b = 0; b != t.count; ++b) {
      for (int d = 0; d != 3; ++d) out_keys[3 * b + d] = t.active[3 * b + d];
      /* slot of key b: probe from its home slot */
      int32_t slot = oracle_hash_slot(t.active[3 * b], t.active[3 * b + 1],
                                      t.active[3 * b + 2], t.size);
      while (!(t.keys[3 * slot] == t.active[3 * b] && t.keys[3 * slot + 1] == t.active[3 * b + 1] &&
               t.keys[3 * slot + 2] == t.active[3 * b + 2]))
        slot = (slot + 127) % t.size;
      out_slots[b] = slot;
    }
  oracle_table_free(&t);
  return st;
}

/* Binning order of the CUDA path: particles grouped by block, then by stencil-origin cell
 * ascending, particles of one cell in increasing index order (a stable sort by
 * (block, cell)); block_start[b] is the first slot of block b. */
void oracle_bin_order(int n, int nblocks, const int32_t *block, const int32_t *cell,
                      int32_t *order, int32_t *block_start) {
  const size_t ncells = (size_t)nblocks * 512;
  int32_t *first = (int32_t *)calloc(ncells + 1, sizeof(int32_t));
  int32_t *fill = (int32_t *)calloc(ncells, sizeof(int32_t));
  for (int i = 0; i != n; ++i) first[(size_t)block[i] * 512 + cell[i] + 1]++;
  for (size_t k = 0; k != ncells; ++k) first[k + 1] += first[k];
  for (int i = 0; i != n; ++i) {
    size_t k = (size_t)block[i] * 512 + cell[i];
    order[first[k] + fill[k]++] = i;
  }
  for (int b = 0; b <= nblocks; ++b) block_start[b] = first[(size_t)b * 512];
  free(fill);
  free(first);
}
