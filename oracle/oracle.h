/* Test infrastructure: CPU restatement of zpc's explicit MLS/APIC MPM substep.
 *
 * This library is the CHECKER for the CUDA product path (zsmpm_b200/csrc); it is never
 * linked into, loaded by, or called from the product.  The FP32 build restates the
 * reference's per-particle arithmetic in the reference's operation order so that, under a
 * sequential schedule, it reproduces the compiled reference (oracle/_ref/zsref_cli) bit for
 * bit; the FP64 build runs the same algorithm in double precision and is the accuracy
 * yardstick that every FP32 result (CPU reference, this restatement, the GPU) is measured
 * against.  Parity pin: see tests/test_oracle_pin.py, which compares this restatement with
 * the compiled reference on seeded scenes, SVD batches and stress batches.
 *
 * Reference files followed (paths inside the zpc repository, include/zensim/...):
 *   sparsity           simulation/sparsity/SparsityOp.hpp:58-112
 *   hash table         container/HashTable.hpp:356-398 (insert), :444-456 (query),
 *                      :493-500 (do_hash), math/Hash.hpp:17-27 (hash_combine)
 *   stencil            simulation/Utils.hpp:30-189, math/curve/InterpolationKernel.hpp:51-130
 *   P2G                simulation/transfer/P2G.hpp:45-127
 *   stress             physics/ConstitutiveModel_Vol_dP.hpp:10-46 (fixed corotated),
 *                      :241-325 (Drucker-Prager sand), ConstitutiveModel.hpp:34-38 (Lame)
 *   snow projection    physics/plasticity_models/SnowPlasticity.hpp:24-32
 *   SVD (FP32)         math/matrix/SVD.hpp:15-1025 (McAdams et al. 2011 quaternion Jacobi)
 *   grid update        simulation/grid/GridOp.hpp:72-164, geometry/Collider.h:80-110
 *   colliders          geometry/Collider.h:10-200, geometry/AnalyticLevelSet.h (plane, cuboid,
 *                      sphere, cylinder), math/VecInterface.hpp (vector operation order)
 *   level-set boundary geometry/SparseLevelSet.hpp:366-374 (worldToIndex), :477-484 (value_or),
 *                      :736-752 (distance, normal), :862-875 (linear arena),
 *                      math/VecInterface.hpp:1043-1049 (xlerp), ZpcMathUtils.hpp:1779-1781
 *   G2P                simulation/transfer/G2P.hpp:43-84, math/matrix/MatrixUtils.h:136-146
 *   G2P2G              simulation/transfer/G2P2G.hpp:49-142 (implicit force operator)
 *   P2C2G / G2C2P      simulation/transfer/P2C2G.hpp:27-189, G2C2P.hpp:36-278 (cell-centric
 *                      transfers), simulation/particle/Query.tpp:8-58 (index buckets)
 * Matrices are column-major (M(i,j) = M[3j+i]) as in the reference.
 */
#ifndef ZSMPM_ORACLE_H
#define ZSMPM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_FC = 0, ORACLE_DP = 1, ORACLE_SNOW = 2 };
enum { ORACLE_MODE_COMMITTED = 0, ORACLE_MODE_REFERENCE = 1 };
enum { ORACLE_WALL_STICKY = 0, ORACLE_WALL_SLIP = 1, ORACLE_WALL_SEPARATE = 2,
       ORACLE_WALL_NONE = 3 };

/* Collider<AnalyticLevelSet<shape, f32, 3>> (geometry/Collider.h:10-200): the layout of
 * zsmpm_collider.  shape 0 plane (a origin, b normal), 1 cuboid (a min, b max), 2 sphere
 * (a center, b[0] radius), 3 cylinder (a bottom, b[0] radius, b[1] length, axis); type 0 sticky,
 * 1 slip, 2 separate; rot is the rotation R, row-major. */
typedef struct {
  int shape, type, axis, reserved;
  float a[3], b[3];
  float s, dsdt;
  float rot[9];
  float omega[3], t[3], dtdt[3];
} oracle_collider;

/* LevelSetBoundary<SparseLevelSet<3>>: block origins (multiples of 8), 512 distances per block
 * (cell x*64 + y*8 + z), the background value and the world-to-index transform
 * X = ((x - t) rinv) sinv (row vectors, row-major matrices). */
typedef struct {
  int nblocks, type;
  float background, sinv[9], rinv[9], t[3];
  const int32_t *keys;
  const float *sdf;
} oracle_levelset;

typedef struct {
  int model;             /* ORACLE_FC / ORACLE_DP / ORACLE_SNOW */
  int mode;              /* ORACLE_MODE_COMMITTED or ORACLE_MODE_REFERENCE */
  int wall_type, wall_cells;
  int table_expected;    /* HashTable expected entries (capacity next_2pow(n)*16) */
  int volume_correction; /* Drucker-Prager */
  double dx, dt, gx, gy, gz;
  double E, nu, volume;
  double friction_deg, cohesion, beta;      /* Drucker-Prager */
  double hardening, theta_c, theta_s;       /* snow */
  int ncolliders;                           /* applied after the walls, in order */
  const oracle_collider *colliders;
  int nlevelsets;                           /* applied after the colliders, in order */
  const oracle_levelset *levelsets;
} oracle_params;

/* Runs nsteps substeps on SoA/AoS host arrays in place (x, v: 3n; C, F: 9n column-major;
 * plastic: logJp for Drucker-Prager, Jp for snow).  Canonical block order (ascending
 * (bx,by,bz)).  Grid output (optional): keys[3*nb] and grid[nb][4][512] = (m, vx, vy, vz)
 * after the boundary conditions of the last substep.  Returns 0, or 1 when the grid output
 * capacity is too small, 2 when the hash table is full. */
int oracle_run_f32(const oracle_params *p, int n, const float *m, float *x, float *v,
                   float *C, float *F, float *plastic, int nsteps, int cap_blocks,
                   int *out_nblocks, int *out_keys, float *out_grid);
int oracle_run_f64(const oracle_params *p, int n, const double *m, double *x, double *v,
                   double *C, double *F, double *plastic, int nsteps, int cap_blocks,
                   int *out_nblocks, int *out_keys, double *out_grid);

/* oracle_run with the cell-centric transfer pair in place of P2G / G2P: P2C2GTransfer
 * (simulation/transfer/P2C2G.hpp:27-189) over every active (block, cell), then after the grid
 * update PreG2C2PTransfer, G2C2PTransfer and PostG2C2PTransfer (G2C2P.hpp:36-278), on the
 * index buckets of simulation/particle/Query.tpp:8-58 with displacement 0.5.  Fixed corotated
 * only (returns 6 for another model); C carries the pair's B attribute. */
int oracle_run_cell_f32(const oracle_params *p, int n, const float *m, float *x, float *v, float *C,
                        float *F, int nsteps, int cap_blocks, int *out_nblocks, int *out_keys,
                        float *out_grid);
int oracle_run_cell_f64(const oracle_params *p, int n, const double *m, double *x, double *v, double *C,
                        double *F, int nsteps, int cap_blocks, int *out_nblocks, int *out_keys,
                        double *out_grid);

/* G2P2GTransfer, the implicit force operator (simulation/transfer/G2P2G.hpp:49-142): fout
 * (zeroed first) receives sum_p W (4/dx^2) (V0 P(F*) F*^T)(x_i - x_p), F* = (I + dt C(vin)) F,
 * with the particle state left unchanged.  vin and fout hold 1536 values per block, node-major
 * [(block*512 + cell)*3 + d]; the blocks are keys[3*nb] in index order.  Returns 0, 2 when
 * the table is full, 5 when a stencil node has no block. */
int oracle_g2p2g_f32(const oracle_params *p, int n, const float *x, const float *F,
                     const float *plastic, int nb, const int32_t *keys, const float *vin,
                     float *fout);
int oracle_g2p2g_f64(const oracle_params *p, int n, const double *x, const double *F,
                     const double *plastic, int nb, const int32_t *keys, const double *vin,
                     double *fout);

/* McAdams 3x3 SVD in the reference's float operation order (A = U diag(S) V^T). */
void oracle_svd_f32(const float *A, float *U, float *S, float *V);
/* Accurate double SVD (cyclic Jacobi on A^T A), same sign conventions. */
void oracle_svd_f64(const double *A, double *U, double *S, double *V);

/* Constitutive updates on one particle.  model FC: PF = V0 P(F) F^T.  model DP: the
 * reference's compute_stress_sand, which projects F in place and updates *plastic (logJp).
 * model SNOW: Stomakhin projection of F in place, Jp accumulation in *plastic, then fixed
 * corotated stress with hardened Lame parameters. */
void oracle_stress_f32(const oracle_params *p, float *F, float *plastic, float *PF);
void oracle_stress_f64(const oracle_params *p, double *F, double *plastic, double *PF);

/* Block activation exactly as ComputeSparsity + EnlargeSparsity under a sequential
 * schedule: keys in insertion order and the slot each key occupies. */
int oracle_activate(int n, const float *x, float dx, int table_expected, int cap,
                    int *out_nblocks, int *out_nparblocks, int *out_keys, int *out_slots,
                    int *out_table_size);

/* The reference's HashTable home slot of a block key, (do_hash(k) % T + T) % T. */
int32_t oracle_hash_slot(int32_t kx, int32_t ky, int32_t kz, int32_t table_size);

/* Particle binning order of the CUDA path, restated: given per-particle block ranks and
 * local stencil cells (0..511), returns order[] (slot -> particle index), a stable sort by
 * (block, cell), plus block_start[nblocks+1]. */
void oracle_bin_order(int n, int nblocks, const int32_t *block, const int32_t *cell,
                      int32_t *order, int32_t *block_start);

#ifdef __cplusplus
}
#endif
#endif
