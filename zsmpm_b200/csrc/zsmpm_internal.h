// Internal host/device interface between the C ABI layer (zsmpm_api.cu) and the kernels
// (zsmpm_kernels.cu).  Not part of the public ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "zsmpm_device.cuh"
#include "zsmpm_mlp.cuh"

struct zsmpm_closure;

namespace zsmpm {

// One particle buffer set.  Vectors are float4 (x,y,z,m) / (vx,vy,vz,0).  3x3 matrices (C, A,
// F) are stored in tiles of 32 particles: component k (column-major) of particle i at
// mat_at(k, i) = ((i / 32) * 9 + k) * 32 + i % 32, the layout of one 3x3 property of a
// TileVector<float, 32>.  A warp's load of one component is 128 contiguous bytes, as with one
// array per component, and its nine components of 32 particles are 1152 contiguous bytes: one
// DRAM stream per matrix rather than nine (the G2P writes three matrices per particle).
// A matrix array holds 9 * mat_capacity(cap) floats.
__host__ __device__ __forceinline__ size_t mat_at(int k, size_t i) {
  return ((i >> 5) * 9 + (size_t)k) * 32 + (i & 31);
}
__host__ __device__ __forceinline__ int64_t mat_capacity(int64_t cap) { return (cap + 31) & ~int64_t(31); }

struct particle_buffers {
  float4 *xm = nullptr;
  float4 *v = nullptr;
  float *C = nullptr;
  float *A = nullptr;  // affine momentum m C - (4 dt / dx^2) tau, consumed by P2G
  float *F = nullptr;
  float *plastic = nullptr;  // logJp (DP) or Jp (snow); null for fixed corotated
  int *id = nullptr;         // upload index
  int *sid = nullptr;        // scene of the particle (batched scenes only)
};

// Batched scenes share one key space: scene s owns a slot of kBatchSlot blocks per axis at
// slot coordinates (s & 7, (s >> 3) & 7, s >> 6); its particles keep local positions and its
// blocks lie in [-kBatchMargin, kBatchSlot - kBatchMargin) per axis before the slot offset.
constexpr int kBatchSlot = 32;
constexpr int kBatchMargin = 4;
constexpr int kBatchMaxScenes = 1 << 16;

// Device counters (int32), zeroed at the start of every substep except the status word, the
// substep counter and the learned G2P's queue counters.
enum counter_slot : int {
  kCtrParticleBlocks = 0,  // blocks inserted from particles (insertion indices [0, npb))
  kCtrEnlarged = 1,        // blocks inserted by the enlargement
  kCtrBlocks = 2,          // total active blocks of this substep
  kCtrStatus = 3,          // sticky status bits (kStatus*)
  kCtrBoxLo = 4,           // 3 ints: bounding box of particle blocks
  kCtrBoxHi = 7,           // 3 ints
  kCtrWords = 10,          // bitmap words in use
  kCtrWork = 11,           // 8 work counters for persistent kernels
  kCtrSubstep = 20,        // substeps begun since the scene was created (audit/log sampling)
  kCtrMaskFrom = 21,       // blocks whose move masks the last G2P wrote (0: none since the upload)
  kCtrMaskBad = 22,        // 1: a particle of the last G2P left its block's 3^3 neighbourhood
  kCtrUseMasks = 23,       // this activation inserts from the move masks of that many blocks
  kCtrOrderFront = 24,     // blocks of at least kBigBlock particles placed at the front of work_order
  kCtrOrderBack = 25,      // the others, placed from the back
  kCtrMovers = 26,         // particles the last G2P listed as having left their cell (cleared by the binning)
  kCtrIncBin = 27,         // 1: this substep's binning merges the movers into the last binning's order
  kCtrBinInfo = 28,        // the last binning: -1 full, else the number of movers it merged
  kCtrDirty = 29,          // cells the incremental binning's movers arrived in (to be sorted by id)
  kCtrQueue = 30,          // projections the last learned G2P queued for the closure's network
  kCtrQueueSubstep = 31,   // the substep number of that G2P (the closure pass samples its audit by it)
  kCtrCount = 32
};
enum work_slot : int {
  kWorkCellStart = 0,
  kWorkFinalize = 1,
  kWorkP2G = 2,
  kWorkG2P = 3,
  kWorkGrid = 4,
  kWorkG2P2G = 5  // reset by its own launcher (the operator runs many times per activation)
};

struct scene_params {
  int n;          // particles
  int cap;        // particle capacity (matrix component stride)
  int nb_cap;     // block capacity
  int table_size; // hash table slots (power of two)
  int bitmap_cap; // bitmap words available
  float dx, inv_dx, dt, kappa, four_over_dx;
  int dx_pow2;    // dx is a power of two: x / dx is exactly x * inv_dx
  float gravity[3];
  int wall_type, wall_cells;
  material_dev mat;
  // batched scenes
  int batch;                        // 1: particles carry a scene id, keys carry the scene slot
  int nscenes;
  const material_dev *mats;         // [nscenes] per-scene materials (device)
  const int *scene_start;           // [nscenes + 1] upload-index ranges of the scenes (device)
  // colliders after the walls (device; the count is read at run time, so updates need no new graph)
  const collider_dev *colliders;
  const int *ncolliders;
  // sparse level-set boundaries after the colliders (device, count read at run time)
  const levelset_dev *levelsets;
  const int *nlevelsets;
  // launch shapes (set by the autotuner; 0 = default)
  int g2p_threads;                  // 128 or 256
  int g2p_ctas_per_sm, p2g_ctas_per_sm;
  int p2g_ranks;                    // P2G staging depth per round: 8, 12 or 16 (0 = 12)
  // incremental binning
  int mover_cap;                    // entries of the mover list
  int bin_full;                     // 1: this binning launch recounts every particle
  int transfer;                     // kTransferApic (P2G / G2P) or kTransferCell (P2C2G / G2C2P)
};

constexpr int kTransferApic = 0, kTransferCell = 1;

// floats of a queue entry: U 9, V 9, S 3, plastic state, m, C 9
constexpr int kQueueFloats = 32;

// G2P options beside the plain path: the learned closure and the trial-state log.
struct g2p_aux {
  int learned = 0;            // 1: the closure's MLP replaces the return map's projection
  closure_dev cd{};           // its weights, normalisation, hull and audit accumulators
  // the projections G2P hands to the network: raw features [qcap][6], network outputs
  // [qcap][6], [qcap][kQueueFloats] U V S, the plastic state, m and C, (binned slot, scene)
  // [qcap] and the upload index [qcap]
  float *q_feat = nullptr, *q_out = nullptr, *q_uvs = nullptr;
  int2 *q_slot = nullptr;
  int *q_id = nullptr;
  long long qcap = 0;
  float *log_buf = nullptr;   // [log_cap][6] raw closure features of sampled particles
  long long log_cap = 0;
  int log_period = 0;         // one particle in log_period per substep (0 = off)
  unsigned long long *log_count = nullptr;
};

struct scene_device {
  scene_params prm;
  g2p_aux aux;
  particle_buffers cur, nxt;
  // hash table (HashTableView-compatible arrays + packed keys used for CAS/probing)
  uint64_t *pk = nullptr;
  int *tkeys = nullptr;   // [T][3]
  int *tidx = nullptr;    // [T]
  int *tstatus = nullptr; // [T]
  int *active_keys = nullptr; // [nb_cap][3] sorted keys (view)
  int *view_cnt = nullptr;    // active block count (view)
  uint64_t *ins_pk = nullptr; // [nb_cap] keys by insertion index
  int *ins_slot = nullptr;    // [nb_cap]
  uint64_t *blk_pk = nullptr; // [nb_cap] keys by final block index
  uint32_t *bmask = nullptr;  // [nb_cap] per block: bit (ox+1)*9+(oy+1)*3+(oz+1) set when one of its
                              // particles ended G2P in block + (ox, oy, oz)
  int *nbr = nullptr;         // [nb_cap][8]
  uint32_t *bitmap = nullptr; // [bitmap_cap]
  int *word_prefix = nullptr; // [bitmap_cap]
  int *ctr = nullptr;         // [kCtrCount]
  // binning
  int *block_count = nullptr; // [nb_cap]
  int *block_start = nullptr; // [nb_cap + 1]
  int *cell_count = nullptr;  // [nb_cap * 512]
  int *cell_start = nullptr;  // [nb_cap * 512]
  uint32_t *key32 = nullptr;  // [cap]
  int *rnk = nullptr;         // [cap]
  int *tmp = nullptr;         // [cap]
  int *src = nullptr;         // [cap] slot -> index in cur
  // the previous binning's cell and block starts (the binning alternates between two sets, so
  // that an incremental binning reads the last one while it writes its own)
  int *cell_start_prev = nullptr;  // [nb_cap * 512]
  int *block_start_prev = nullptr; // [nb_cap + 1]
  uint64_t *old_pk = nullptr;      // [nb_cap] keys of the previous binning's blocks, by their index then
  int *new_of_old = nullptr;       // [nb_cap] their indices in the current activation (-1: gone)
  uint8_t *moved = nullptr;        // [cap] per slot of the last binning: 1 when G2P moved the particle out
                                   // of its cell (or out of reach of the move masks)
  int *movers = nullptr;           // [mover_cap] slots of the particles that left their cell
  int2 *mover_pos = nullptr;       // [mover_cap] (new cell index b * 512 + cell, arrival rank in it)
  int *dirty = nullptr;            // [mover_cap] new cells that received movers
  int *work_order = nullptr;  // [nb_cap] blocks in the order the per-block kernels take them
  int *scan_part = nullptr;   // [2 * kScanCtas + 1]
  float *grid = nullptr;      // [nb_cap][4][512]
};

constexpr int kScanCtas = 256;
constexpr int kBigBlock = 2048;  // particles from which a block goes to the front of work_order

// sets per-device kernel attributes (dynamic shared memory sizes); call with the device current
cudaError_t prepare_kernels();
// launchers (all asynchronous on `st`)
cudaError_t launch_activate(scene_device &s, cudaStream_t st);
cudaError_t launch_bin(scene_device &s, cudaStream_t st);
cudaError_t launch_p2g(scene_device &s, cudaStream_t st);
// P2C2G of the cell-centric pair: part 0 all, 1 the momentum part, 2 the force part
cudaError_t launch_p2c2g(scene_device &s, int part, cudaStream_t st);
cudaError_t launch_grid_update(scene_device &s, cudaStream_t st);
cudaError_t launch_g2p(scene_device &s, cudaStream_t st, bool closure_pass = true);
cudaError_t launch_closure_pass(scene_device &s, cudaStream_t st);
int kernels_per_substep();
// the implicit system (ImplicitMPM.hpp) over node-major dof vectors [nb * 512 * 3]; a kernel
// returns at once when `skip` (device, may be null) holds a nonzero value
cudaError_t launch_g2p2g(scene_device &s, const float *v, float *f, long long ndofs, float dt, const int *skip,
                         cudaStream_t st);
cudaError_t launch_implicit_mass(scene_device &s, const float *dv, float *out, float dt, long long ndofs,
                                 const int *skip, cudaStream_t st);
cudaError_t launch_implicit_project(scene_device &s, float *dof, long long ndofs, const int *skip,
                                    cudaStream_t st);
cudaError_t launch_implicit_precondition(scene_device &s, const float *in, float *out, long long ndofs,
                                         const int *skip, cudaStream_t st);

// ConjugateGradient::solve state on the device
struct cg_state {
  double acc;        // dot product accumulator (zeroed by its consumer)
  float ztrk, norm, local_tol, alpha, beta;
  int done, iter;
};
struct cg_vectors {
  float *r, *p, *q, *ap;  // residual, search direction, preconditioned residual, A p
};
cudaError_t launch_cg_begin(scene_device &s, float *x, const float *b, const cg_vectors &v, long long ndofs, float dt,
                            cg_state *cs, float tol, float rel_tol, cudaStream_t st);
cudaError_t launch_cg_iteration(scene_device &s, float *x, const cg_vectors &v, long long ndofs, float dt,
                                cg_state *cs, int max_iters, cudaStream_t st);

// upload / download helpers: staging is AoS (x: 3n, C/F: 9n), see zsmpm_particle_arrays
cudaError_t launch_import(scene_device &s, const float *m, const float *x, const float *v,
                          const float *C, const float *F, const float *plastic, int n,
                          cudaStream_t st);
cudaError_t launch_import_tilevector(scene_device &s, const float *base, int nchn, int off_m,
                                     int off_x, int off_v, int off_C, int off_F, int off_pl,
                                     int n, cudaStream_t st);
cudaError_t launch_prime(scene_device &s, cudaStream_t st);
cudaError_t launch_export(const scene_device &s, float *m, float *x, float *v, float *C,
                          float *F, float *plastic, cudaStream_t st);
cudaError_t launch_export_tilevector(const scene_device &s, float *base, int nchn, int off_m,
                                     int off_x, int off_v, int off_C, int off_F, int off_pl,
                                     cudaStream_t st);
cudaError_t launch_export_order(const scene_device &s, int *order, cudaStream_t st);
// block activation of AoS positions into a caller-provided scene_device view (used by the
// allocation-free entry point); writes the sorted keys and the count (or a negative code)
cudaError_t launch_activate_static(scene_device &s, const float *x, int *keys_out, int cap,
                                   int *count_out, cudaStream_t st);
// the device view of a closure that has a dataset or a loaded state (false otherwise)
bool closure_device_view(const zsmpm_closure *c, closure_dev *out);
// the network (tcgen05) over rows x[0, min(*n_dev, cap)) of raw features into y; fixed launch
// shape, so that it can be captured in a CUDA graph
// the closure kernels' attributes (the split-BF16 forward's 72 KB of shared memory), per device
cudaError_t prepare_closure_kernels();
cudaError_t launch_closure_rows(const closure_dev &cd, const float *x, float *y, const int *n_dev, long long cap,
                                cudaStream_t st);
// records the calling thread's error message (read back by zsmpm_last_error_string)
int record_error(int status, const char *message);
cudaError_t launch_svd_batch(const float *A, float *U, float *S, float *V, long long count,
                             cudaStream_t st);
// the bht<i32,3,int,16> of keys[n][3] built on the device (zsmpm_bht.cu); returns a zsmpm_status
int bht_build_device(const int32_t *keys, int n, int64_t size, int32_t *tkeys, int32_t *indices, int32_t *status,
                     int32_t *active, int32_t *cnt_success, uint32_t *hashers_out, cudaStream_t st);
int64_t bht_table_size(int64_t n);
// exclusive scan of in[0, *n_ptr) into out[0, *n_ptr] (out[n] = total); part holds
// 2 * kScanCtas + 1 partial sums
cudaError_t launch_exclusive_scan(const int *in, const int *n_ptr, int *part, int *out, cudaStream_t st);
cudaError_t launch_constitutive_batch(const material_dev &mat, float *F, float *plastic,
                                      float *tau, long long count, cudaStream_t st);

}  // namespace zsmpm
