/* Test infrastructure (oracle): internal declarations shared by the oracle's C files. */
#ifndef ZSMPM_ORACLE_INTERNAL_H
#define ZSMPM_ORACLE_INTERNAL_H
#include <stdint.h>

/* Host-side replica of zs::HashTable<i32,3,int> storage: keys (i32x3 per slot, INT_MAX
 * when empty), indices (-1 when empty), the active key list and its count. */
typedef struct {
  int32_t size;
  int32_t count;
  int32_t *keys;
  int32_t *index;
  int32_t *active;
} oracle_table;

int32_t oracle_do_hash(int32_t kx, int32_t ky, int32_t kz);
int oracle_table_init(oracle_table *t, int expected);
void oracle_table_free(oracle_table *t);
void oracle_table_clear(oracle_table *t);
int32_t oracle_table_insert(oracle_table *t, const int32_t k[3], int32_t id);
int32_t oracle_table_query(const oracle_table *t, const int32_t k[3]);
void oracle_block_of(const float x[3], float dxinv, int32_t out[3]);
int oracle_activate_table(oracle_table *t, int n, const float *x, float dx, int *nparblocks);
void oracle_table_canonicalize(oracle_table *t);
float oracle_ref_sqrtf(float arg);

#endif
