/* zsmpm: B200-native explicit MLS/APIC MPM substep on a sparse grid of 8^3 blocks.
 *
 * C ABI of libzsmpm.so.  It replaces the CUDA launches that zpc's execution policy makes
 * for its legacy MPM operators (a zs::CudaExecutionPolicy applying functors over
 * range(Np) or Collapse{nblocks, cells}) with hand-written sm_100a kernels.  Plain
 * pointers and sizes only; no C++ types cross the boundary; no exceptions escape.
 *
 * Reference interfaces replaced (paths inside the zpc repository, include/zensim/...):
 *   zsmpm_activate_blocks  CleanSparsity + ComputeSparsity + EnlargeSparsity launched over
 *                          range(tableSize)/range(Np)/range(cnt)
 *                          (simulation/sparsity/SparsityOp.hpp:41-112,
 *                           simulation/sparsity/SparsityCompute.tpp:5-26)
 *   zsmpm_bin_particles    SpatiallyCount + exclusive_scan + SpatiallyDistribute
 *                          (SparsityOp.hpp:115-196, simulation/particle/Query.tpp:8-58)
 *   zsmpm_p2g              CleanGridBlocks + P2GTransfer
 *                          (simulation/grid/GridOp.hpp:54-69, simulation/transfer/P2G.hpp:45-127,
 *                           CUDA twin cuda/simulation/transfer/P2G.hpp:35-117)
 *   zsmpm_grid_update      ComputeGridBlockVelocity + ApplyBoundaryConditionOnGridBlocks
 *                          (GridOp.hpp:72-164, geometry/Collider.h:80-110)
 *   zsmpm_g2p              G2PTransfer (simulation/transfer/G2P.hpp:43-84) with the
 *                          constitutive update (physics/ConstitutiveModel_Vol_dP.hpp:10-46,
 *                          :241-325; physics/plasticity_models/SnowPlasticity.hpp:24-32)
 *   zsmpm_get_table_view   HashTableView fields (container/HashTable.hpp:279-293, 509-513)
 *   zsmpm_get_grid_view    GridsView / TileVector<f32,512> blocks (geometry/Structure.hpp:33-130)
 *   zsmpm_scene_*          py_interop handle style: container__tv_* / del_container__tv_*
 *                          (py_interop/TileVectorInstantiations.cpp:5-155)
 *   particle views         TileVectorViewLite<f32,32> element (chn, i) at
 *                          ((i/32)*nchn + chn)*32 + i%32 (py_interop/TileVectorView.hpp:10-60)
 *
 * Ownership: the library allocates and frees all device memory of a scene; views are
 * non-owning.  Threading: a scene is bound to one device; calls on one scene must not
 * overlap (as a zs policy bound to a stream is not re-entrant).  Errors: every entry point
 * returns a zsmpm_status; zsmpm_last_error_string() describes the last failure of the
 * calling thread.  Device-side failures (hash table full, particle outside the block-key
 * range, bounded waits that gave up) are recorded in a per-scene status word that
 * zsmpm_scene_status() reads; kernels never trap.
 */
#ifndef ZSMPM_H
#define ZSMPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define ZSMPM_API __declspec(dllexport)
#else
#define ZSMPM_API __attribute__((visibility("default")))
#endif

typedef enum {
  ZSMPM_OK = 0,
  ZSMPM_ERR_TABLE_FULL = 1,    /* hash table load limit reached (HashTable.hpp:369 "proximity") */
  ZSMPM_ERR_CAPACITY = 2,      /* particle / block / output capacity exceeded */
  ZSMPM_ERR_INVALID_ARG = 3,
  ZSMPM_ERR_CUDA = 4,          /* a CUDA runtime call failed (message has the CUDA error) */
  ZSMPM_ERR_TIMEOUT = 5,       /* a bounded device-side wait gave up */
  ZSMPM_ERR_OUT_OF_DOMAIN = 6, /* a particle position is NaN/Inf or beyond the key range */
  ZSMPM_ERR_NO_DEVICE = 7,
  ZSMPM_ERR_NOT_READY = 8      /* stage called before its inputs exist (e.g. p2g before bin) */
} zsmpm_status;

typedef enum {
  ZSMPM_FIXED_COROTATED = 0, /* FixedCorotatedConfig (ConstitutiveModel.hpp:760) */
  ZSMPM_DRUCKER_PRAGER = 1,  /* DruckerPragerConfig with compute_stress_sand */
  ZSMPM_SNOW = 2             /* fixed corotated + Stomakhin snow projection */
} zsmpm_model;

typedef enum {
  /* Standard ordering: the return map runs at the end of G2P and its projected F is
   * stored; the stress used by the next P2G comes from that F. */
  ZSMPM_PLASTICITY_COMMITTED = 0,
  /* The reference's ordering: the return map acts on a copy of F inside the stress
   * evaluation of P2G and only logJp is kept (P2G.hpp:87-100); stored F is the trial F. */
  ZSMPM_PLASTICITY_REFERENCE = 1
} zsmpm_plasticity_mode;

typedef enum {
  ZSMPM_WALL_STICKY = 0,   /* collider_e::Sticky */
  ZSMPM_WALL_SLIP = 1,     /* collider_e::Slip */
  ZSMPM_WALL_SEPARATE = 2, /* collider_e::Separate */
  ZSMPM_WALL_NONE = 3
} zsmpm_wall;

typedef enum {
  ZSMPM_BLOCK_ORDER_SORTED = 0,   /* active blocks ascending by (bx, by, bz), bz fastest */
  ZSMPM_BLOCK_ORDER_INSERTION = 1 /* the order a sequential ComputeSparsity+EnlargeSparsity
                                     inserts them (first particle, then enlargement) */
} zsmpm_block_order;

/* Particle-grid transfers of a scene's substep (zsmpm_scene_set_transfer). */
typedef enum {
  /* P2GTransfer / G2PTransfer (simulation/transfer/P2G.hpp, G2P.hpp): APIC with the quadratic
   * B-spline; the C attribute is the APIC C */
  ZSMPM_TRANSFER_APIC = 0,
  /* P2C2GTransfer / G2C2PTransfer with PreG2C2PTransfer and PostG2C2PTransfer
   * (simulation/transfer/P2C2G.hpp:27-189, G2C2P.hpp:36-278): through the grid cells, tent
   * weights to the cell centers and 1/8 to the corners; fixed corotated only; the C attribute
   * holds the pair's B matrix (as the reference's "C" attribute does for it) */
  ZSMPM_TRANSFER_CELL = 1
} zsmpm_transfer;

/* Parts of P2C2G (zsmpm_p2c2g). */
typedef enum {
  ZSMPM_P2C2G_ALL = 0,      /* P2C2GTransfer: mass, momentum and the stress term */
  ZSMPM_P2C2G_MOMENTUM = 1, /* P2C2GTransferMomentum: mass and momentum m (v + B Dinv (x_i - x_p)) */
  ZSMPM_P2C2G_FORCE = 2     /* P2C2GTransferForce: the stress term alone, into the momentum
                               channels (the mass channel untouched) */
} zsmpm_p2c2g_part;

typedef enum {
  ZSMPM_CLOSURE_PLAIN = 0,   /* analytic return map */
  ZSMPM_CLOSURE_LEARNED = 1  /* MLP closure (zsmpm_closure_*), falls back per particle */
} zsmpm_closure_kind;

typedef struct {
  int32_t model;            /* zsmpm_model */
  int32_t plasticity_mode;  /* zsmpm_plasticity_mode */
  float E, nu, rho;
  float volume;             /* particle rest volume V0 (MaterialConfig::volume) */
  float friction_deg;       /* Drucker-Prager friction angle (DruckerPragerConfig::fa) */
  float cohesion;           /* Drucker-Prager log-strain shift (DruckerPragerConfig::cohesion) */
  float beta;               /* Drucker-Prager volume-correction factor */
  int32_t volume_correction;
  float hardening;          /* snow xi */
  float theta_c, theta_s;   /* snow critical compression / stretch */
} zsmpm_material;

typedef struct {
  float dx;
  float dt;
  float gravity[3];
  int32_t wall_type;        /* zsmpm_wall */
  int32_t wall_cells;       /* walls are planes wall_cells*dx inside each face of [0,1]^3 */
  zsmpm_material material;
  int64_t max_particles;    /* capacity; 0 = the count of the first upload */
  int32_t table_expected;   /* HashTable expected entries; 0 = max(Np/512, 64)
                               (SparsityCompute.tpp:11-14); capacity next_2pow(n)*16 */
  int32_t block_order;      /* zsmpm_block_order */
  int32_t device;           /* CUDA device ordinal */
  int32_t threads_per_cta;  /* G2P CTA size: 0 = default (256) or the autotuner's pick; 128 or 256 */
} zsmpm_scene_desc;

/* Particle arrays in the reference's zs::Particles<f32,3> layout: one array per attribute,
 * vectors and matrices stored per particle (x: 3n, F and C: 9n column-major).  Any of
 * v, C, F, plastic may be NULL on upload (zero, zero, identity, zero/one).  `plastic` is
 * logJp for Drucker-Prager and Jp for snow. */
typedef struct {
  float *m;
  float *x;
  float *v;
  float *C;
  float *F;
  float *plastic;
} zsmpm_particle_arrays;

/* TileVector<f32,32>-style AoSoA view: element (chn, i) at ((i/32)*nchn + chn)*32 + i%32.
 * Channel offsets of the attributes, -1 when absent. */
typedef struct {
  float *base;
  int32_t num_channels;
  int32_t lane_width;  /* must be 32 */
  int32_t off_m, off_x, off_v, off_C, off_F, off_plastic;
} zsmpm_tilevector_view;

/* HashTableView<cuda, HashTable<i32,3,int>> fields, device pointers. */
typedef struct {
  int32_t *keys;        /* [table_size][3], INT32_MAX when empty */
  int32_t *indices;     /* [table_size], -1 when empty */
  int32_t *status;      /* [table_size], -1 (unlocked) */
  int32_t *active_keys; /* [capacity][3], key of block index b */
  int32_t *cnt;         /* device counter of active blocks */
  int32_t table_size;
} zsmpm_table_view;

/* Grid blocks: TileVector<f32,512> with 4 channels (m, v.x, v.y, v.z); channel c of cell
 * `cell` ((lx<<6)|(ly<<3)|lz) of block b at base[(b*4 + c)*512 + cell]. */
typedef struct {
  float *base;
  int32_t num_channels;
  int32_t num_blocks;   /* host copy, valid after the last activation was synchronised */
  int32_t *keys;        /* device, [num_blocks][3] */
} zsmpm_grid_view;

/* BhtViewLite<i32,3,int,16> fields (py_interop/BhtInstantiations.cpp:63-75; container/Bht.hpp),
 * device pointers: the bucketed three-hash table that zpc's SparseGrid keeps its blocks in. */
typedef struct {
  int32_t *keys;        /* [table_size][4] storage keys (x, y, z, pad); bytes 0x3f when empty */
  int32_t *indices;     /* [table_size] block index of the key, -1 when empty */
  int32_t *status;      /* [table_size] slot lock, -1 (unlocked) */
  int32_t *active_keys; /* [cnt][3] key of block index b */
  int32_t *cnt;         /* number of keys */
  int32_t *success;     /* build success flag, 1 */
  int32_t table_size;
  uint32_t hashers[6];  /* (hashx, hashy) of hf0, hf1, hf2 */
} zsmpm_bht_view;

typedef struct zsmpm_scene zsmpm_scene;

ZSMPM_API const char *zsmpm_last_error_string(void);
ZSMPM_API const char *zsmpm_version(void);
/* number of visible CUDA devices (0 when none); never fails */
ZSMPM_API int zsmpm_device_count(void);

/* ---- scene lifetime -------------------------------------------------------------- */
ZSMPM_API zsmpm_status zsmpm_scene_create(const zsmpm_scene_desc *desc, zsmpm_scene **out);
ZSMPM_API zsmpm_status zsmpm_scene_destroy(zsmpm_scene *scene);
/* Copies n particles into the scene (host or device pointers; `on_device` selects).  The
 * particles are binned and sorted on the device; particle identity is kept so downloads
 * return the upload order.  Also evaluates the stress of the uploaded state. */
ZSMPM_API zsmpm_status zsmpm_scene_upload(zsmpm_scene *scene, const zsmpm_particle_arrays *p,
                                          int64_t n, int32_t on_device, void *stream);
ZSMPM_API zsmpm_status zsmpm_scene_upload_tilevector(zsmpm_scene *scene,
                                                     const zsmpm_tilevector_view *tv,
                                                     int64_t n, void *stream);
/* Copies particles out in upload order (host or device pointers).  C is recovered from
 * the stored affine momentum; in ZSMPM_PLASTICITY_REFERENCE mode logJp is the value the
 * next P2G would use (one projection ahead of the reference's stored logJp). */
ZSMPM_API zsmpm_status zsmpm_scene_download(zsmpm_scene *scene, zsmpm_particle_arrays *p,
                                            int32_t on_device, void *stream);
ZSMPM_API zsmpm_status zsmpm_scene_download_tilevector(zsmpm_scene *scene,
                                                       const zsmpm_tilevector_view *tv,
                                                       void *stream);
ZSMPM_API int64_t zsmpm_scene_num_particles(const zsmpm_scene *scene);
/* Synchronises the scene's last stream and returns its device status word. */
ZSMPM_API zsmpm_status zsmpm_scene_status(zsmpm_scene *scene);

/* ---- stages (each enqueues on `stream`, NULL = legacy default stream) --------------- */
/* The block keys of the particles' current positions.  After a zsmpm_g2p the particle blocks
 * come from the moves G2P recorded per block of the last binning (a particle that left its
 * block's 3x3x3 neighbourhood, and every upload, make it read all particles instead); the keys
 * are the same either way. */
ZSMPM_API zsmpm_status zsmpm_activate_blocks(zsmpm_scene *scene, void *stream);
ZSMPM_API zsmpm_status zsmpm_bin_particles(zsmpm_scene *scene, void *stream);
ZSMPM_API zsmpm_status zsmpm_p2g(zsmpm_scene *scene, void *stream);
ZSMPM_API zsmpm_status zsmpm_grid_update(zsmpm_scene *scene, void *stream);
ZSMPM_API zsmpm_status zsmpm_g2p(zsmpm_scene *scene, void *stream);
/* The scene's transfer pair (zsmpm_transfer; ZSMPM_TRANSFER_APIC by default).
 * ZSMPM_TRANSFER_CELL replaces P2G / G2P in zsmpm_p2g, zsmpm_g2p, zsmpm_substep and zsmpm_run
 * with the cell-centric pair; it needs a single fixed-corotated scene without a learned closure.
 * The stored C attribute keeps its numbers: set the scheme before the upload whose C holds the
 * scheme's matrix.  With particles present, the pair's affine term of the stored state is
 * formed on `stream`. */
ZSMPM_API zsmpm_status zsmpm_scene_set_transfer(zsmpm_scene *scene, int32_t transfer, void *stream);
/* P2C2GTransfer / P2C2GTransferMomentum / P2C2GTransferForce (zsmpm_p2c2g_part) over every
 * cell of the active blocks (simulation/transfer/P2C2G.hpp:27-420), adding into the grid that
 * the binning zeroed; ZSMPM_TRANSFER_CELL scenes only.  zsmpm_p2g runs the ALL part. */
ZSMPM_API zsmpm_status zsmpm_p2c2g(zsmpm_scene *scene, int32_t part, void *stream);
/* PreG2C2PTransfer + G2C2PTransfer + PostG2C2PTransfer (simulation/transfer/G2C2P.hpp:36-278):
 * v and B from the updated grid, F <- (I + dt B Dinv) F, x += v dt; ZSMPM_TRANSFER_CELL scenes
 * only (the same call as zsmpm_g2p there). */
ZSMPM_API zsmpm_status zsmpm_g2c2p(zsmpm_scene *scene, void *stream);
/* One full substep (activate, bin, P2G, grid update + walls, G2P). */
ZSMPM_API zsmpm_status zsmpm_substep(zsmpm_scene *scene, void *stream);
/* nsteps substeps, replayed from a CUDA graph of four substeps (captured on first use per
 * buffer parity; the substeps beyond a multiple of four are launched directly).  With a learned
 * closure attached, the closure's network pass of each graph substep but the last runs on a
 * second stream of the scene beside the next substep's activation and binning; the state is
 * complete when the work enqueued on `stream` is.  nsteps = 0 captures the graph for the
 * current buffer parity, if it is not captured yet, and runs nothing.  Asynchronous: capacity
 * and domain errors collect in the device status word, which zsmpm_scene_status reads. */
ZSMPM_API zsmpm_status zsmpm_run(zsmpm_scene *scene, int32_t nsteps, void *stream);

/* ---- views and diagnostics ------------------------------------------------------- */
ZSMPM_API zsmpm_status zsmpm_get_table_view(zsmpm_scene *scene, zsmpm_table_view *out);
ZSMPM_API zsmpm_status zsmpm_get_grid_view(zsmpm_scene *scene, zsmpm_grid_view *out);
/* The active blocks of the last activation as a bht<i32,3,int,16> (synchronises; rebuilt on
 * every call, on the device from the device's active keys): the table that the reference's
 * host BHTView::insert (container/Bht.hpp:612-665) builds when the keys are inserted in
 * ascending block order into a bht sized for max(blocks, 16) entries, so index == block index.
 * The view stays valid until the next call or the scene's destruction. */
ZSMPM_API zsmpm_status zsmpm_get_bht_view(zsmpm_scene *scene, zsmpm_bht_view *out);
/* The same table built on the host from keys[nkeys][3] in order, sized for `expected` entries
 * (0: nkeys): table_keys [cap_slots][4], indices and status [cap_slots]; *table_size and the
 * hasher parameters hashers[6] are set even when cap_slots is too small (then
 * ZSMPM_ERR_CAPACITY).  No device needed. */
ZSMPM_API zsmpm_status zsmpm_bht_build_host(const int32_t *keys, int32_t nkeys, int32_t expected,
                                            int32_t *table_keys, int32_t *indices, int32_t *status,
                                            int32_t cap_slots, int32_t *table_size, uint32_t *hashers);
/* The same table built on the device (the bht's device insert, container/Bht.hpp:490-610,
 * with the layout of the in-order host insert): keys, table_keys [cap_slots][4], indices and
 * status [cap_slots] are device pointers; *table_size and hashers[6] are host outputs.  All
 * keys are placed at once by an iteration over their bucket choices that settles on the
 * in-order layout (synchronises on `stream`). */
ZSMPM_API zsmpm_status zsmpm_bht_build_device(const int32_t *keys, int32_t nkeys, int32_t expected,
                                              int32_t *table_keys, int32_t *indices, int32_t *status,
                                              int32_t cap_slots, int32_t *table_size, uint32_t *hashers,
                                              void *stream);
/* Copies the block table of the last activation into a zs::HashTable<int, 3, int>'s storage
 * (container/HashTable.hpp:45-60, 195-199) held by the caller, in host or device memory:
 * keys [table_size][3], indices and status [table_size], the active keys [count][3] and the
 * count.  table_size must equal the scene's (a HashTable sized for the same expected entry
 * count, next_2pow(n) * 16 slots); cap_active is the active-key array's capacity.  Synchronises
 * `stream`.  The slots are those the reference's insert would give the same keys in the
 * canonical order, so zpc's own HashTableView::query finds every block at its index. */
ZSMPM_API zsmpm_status zsmpm_download_table(zsmpm_scene *scene, int32_t *keys, int32_t *indices,
                                            int32_t *status, int32_t *active_keys, int32_t cap_active,
                                            int32_t *count, int32_t table_size, void *stream);
/* Number of active blocks of the last activation (synchronises). */
ZSMPM_API zsmpm_status zsmpm_num_blocks(zsmpm_scene *scene, int32_t *out);
/* Copies the active keys [nb][3] and the grid [nb][4][512] to host memory. */
ZSMPM_API zsmpm_status zsmpm_download_grid(zsmpm_scene *scene, int32_t *keys, float *grid,
                                           int32_t cap_blocks, int32_t *out_nblocks);
/* Host copies of the per-slot particle order of the last binning: order[slot] = upload
 * index of the particle in slot, block_start[nb+1]. */
ZSMPM_API zsmpm_status zsmpm_download_binning(zsmpm_scene *scene, int32_t *order,
                                              int32_t *block_start, int32_t cap_blocks);
/* How the last binning ordered the particles (synchronises): *movers_merged = -1 when it
 * counted every particle (SpatiallyCount + exclusive_scan + SpatiallyDistribute,
 * simulation/sparsity/SparsityOp.hpp:115-196), else the number of particles it moved into
 * other cells while keeping the rest of the previous binning's order (the incremental path,
 * taken after a G2P whose particles all stayed within their block's 3x3x3 neighbourhood).
 * Both give the same order.  Valid until the next activation. */
ZSMPM_API zsmpm_status zsmpm_binning_info(zsmpm_scene *scene, int32_t *movers_merged);
/* Per-stage device times (ms) of the last zsmpm_substep when timing is enabled. */
ZSMPM_API zsmpm_status zsmpm_set_stage_timing(zsmpm_scene *scene, int32_t enabled);
ZSMPM_API zsmpm_status zsmpm_stage_times(zsmpm_scene *scene, float *ms, int32_t count);
/* Number of kernels one zsmpm_substep launches. */
ZSMPM_API int32_t zsmpm_kernels_per_substep(const zsmpm_scene *scene);

/* ---- stand-alone kernels (device pointers), for parity tests of single operators ---- */
/* 3x3 SVD of `count` column-major matrices (math/matrix/SVD.hpp:15-1025). */
ZSMPM_API zsmpm_status zsmpm_svd3(const float *A, float *U, float *S, float *V, int64_t count,
                                  void *stream);
/* Constitutive update of `count` particles: F (in/out, projected as the model does),
 * plastic (in/out) and tau = V0 P F^T (out). */
ZSMPM_API zsmpm_status zsmpm_constitutive(const zsmpm_material *mat, float *F, float *plastic,
                                          float *tau, int64_t count, void *stream);

/* ---- colliders (geometry/Collider.h, geometry/AnalyticLevelSet.h) ------------------------- */
typedef enum {
  ZSMPM_SHAPE_PLANE = 0,    /* AnalyticLevelSet<Plane>: a = origin, b = normal (used as given) */
  ZSMPM_SHAPE_CUBOID = 1,   /* AnalyticLevelSet<Cuboid>: a = min corner, b = max corner */
  ZSMPM_SHAPE_SPHERE = 2,   /* AnalyticLevelSet<Sphere>: a = center, b[0] = radius */
  ZSMPM_SHAPE_CYLINDER = 3  /* AnalyticLevelSet<Cylinder>: a = bottom, b[0] = radius,
                               b[1] = length, axis = 0, 1 or 2 */
} zsmpm_collider_shape;

/* Collider<AnalyticLevelSet<shape, f32, 3>> (Collider.h:10-200): a rigid analytic level set
 * placed by scale s, rotation R and translation t, with their rates.  A grid node at x is
 * inside when the level set's signed distance at X = R^T (x - t) / s is negative; its velocity
 * then becomes the collider's, omega x (x - t) + (dsdt / s)(x - t) + dt/dt (sticky), or keeps
 * its tangential part relative to it (slip; separate only when moving into the collider), with
 * the normal R n(X) (resolveCollision, :80-110). */
typedef struct {
  int32_t shape;    /* zsmpm_collider_shape */
  int32_t type;     /* ZSMPM_WALL_STICKY, ZSMPM_WALL_SLIP or ZSMPM_WALL_SEPARATE */
  int32_t axis;     /* cylinder axis */
  int32_t reserved; /* 0 */
  float a[3], b[3]; /* the shape's parameters, see zsmpm_collider_shape */
  float s, dsdt;    /* scale (non-zero) and its rate */
  float R[9];       /* rotation, row-major: R[3*i + j] = R(i, j) */
  float omega[3];   /* angular velocity */
  float t[3];       /* translation b */
  float dtdt[3];    /* its rate db/dt */
} zsmpm_collider;

#define ZSMPM_MAX_COLLIDERS 16

/* The scene's colliders (at most ZSMPM_MAX_COLLIDERS; count 0 removes them).  The grid update
 * (and zsmpm_implicit_project) applies the six walls of the scene description first, then the
 * colliders in list order, each to the nodes with positive mass (ApplyBoundaryConditionOnGridBlocks,
 * simulation/grid/GridOp.hpp:113-158, one launch per boundary in the reference).  The copy is
 * ordered on `stream` and the call returns once it is done; the kernels read the colliders when
 * they run, so moving colliders are updated between substeps without rebuilding the substep
 * graph.  Single scenes only. */
ZSMPM_API zsmpm_status zsmpm_scene_set_colliders(zsmpm_scene *scene, const zsmpm_collider *colliders,
                                                 int32_t count, void *stream);

/* LevelSetBoundary<SparseLevelSet<3>> (geometry/Collider.h:204-236 applied by
 * ApplyBoundaryConditionOnGridBlocks, simulation/grid/GridOp.hpp:32-36, :126-134): a signed
 * distance sampled on 8^3 blocks, read by trilinear interpolation
 * (geometry/SparseLevelSet.hpp:660-690, 803-930), with `background` outside the blocks.  A world
 * position x maps to index space by X = ((x - t) Rinv) Sinv, row vectors times row-major
 * matrices, the SparseLevelSet's _i2wT, _i2wRinv and _i2wSinv (SparseLevelSet.hpp:366-374); the
 * node at integer index coordinate c holds sdf[block][(c & 7) as x*64 + y*8 + z] of the block
 * whose origin (a multiple of 8 per axis) is c - (c & 7).  Nodes with positive grid mass inside
 * (distance < 0) are made still (sticky), or lose the normal part of their velocity (slip; separate
 * only when moving into it), with the normal from central differences (eps 1e-6) of the distance. */
typedef struct {
  int32_t nblocks;
  int32_t type;         /* ZSMPM_WALL_STICKY, ZSMPM_WALL_SLIP or ZSMPM_WALL_SEPARATE */
  const int32_t *keys;  /* host [nblocks][3] block origins, distinct multiples of 8 */
  const float *sdf;     /* host [nblocks][512] */
  float background;     /* the distance outside the blocks (SparseLevelSet::_backgroundValue) */
  float sinv[9], rinv[9], t[3];
} zsmpm_levelset_desc;

#define ZSMPM_MAX_LEVELSETS 4

/* Adds a sparse level-set boundary, applied after the scene's walls and colliders in the order
 * added.  The block map spans the keys' bounding box and holds at most 2^22 blocks.  The call
 * copies the data to the device and synchronises `stream`.  Single scenes only. */
ZSMPM_API zsmpm_status zsmpm_scene_add_levelset(zsmpm_scene *scene, const zsmpm_levelset_desc *desc,
                                                void *stream);
/* Removes every level-set boundary of the scene and frees their device data (synchronises the
 * device). */
ZSMPM_API zsmpm_status zsmpm_scene_clear_levelsets(zsmpm_scene *scene);

/* ---- the implicit system (simulation/mpm/ImplicitMPM.hpp) ---------------------------- */
/* Grid dof vectors are device arrays of `ndofs` floats, node-major over the active blocks in
 * canonical order: entry (block*512 + cell)*3 + d, cell = x*64 + y*8 + z inside the block.
 * This is the layout of a dof_view<space, 3> over a zs::Vector<float> (types/View.h:77-168)
 * that ImplicitMPMSystem's operators take.  ndofs must be at least 1536 * zsmpm_num_blocks;
 * shorter vectors are not touched and leave ZSMPM_ERR_CAPACITY in the scene status.  Vectors
 * must be 16-byte aligned.  All calls are asynchronous on `stream`; they need a binned scene
 * (zsmpm_activate_blocks + zsmpm_bin_particles for the current positions), and all but
 * zsmpm_g2p2g read the grid mass of a zsmpm_p2g of that activation.  Single scenes only. */

/* G2P2GTransfer (simulation/transfer/G2P2G.hpp:49-142; replaces its launch in
 * ImplicitMPM.hpp:51-53).  ADDS to f, per particle and stencil node,
 * W (4/dx^2) (V0 P(F*) F*^T)(x_i - x_p), where F* = (I + dt C) F and C is gathered from the
 * velocity field v; the particle state is not changed.  Fixed corotated, Drucker-Prager and
 * snow. */
ZSMPM_API zsmpm_status zsmpm_g2p2g(zsmpm_scene *scene, const float *v, float *f, int64_t ndofs,
                                   float dt, void *stream);
/* ImplicitMPMSystem::multiply (ImplicitMPM.hpp:34-61): out = 0, out += G2P2G(in), then where
 * the node mass m > 0, out = (out dt^2 + m) in (ForceDtSqrPlusMass, :17-33). */
ZSMPM_API zsmpm_status zsmpm_implicit_multiply(zsmpm_scene *scene, const float *in, float *out,
                                               int64_t ndofs, float dt, void *stream);
/* ImplicitMPMSystem::project (ImplicitMPM.hpp:99-124) with the scene's six walls
 * (Projector, :63-97): nodes with m > 0 get the walls' collision response, others are 0. */
ZSMPM_API zsmpm_status zsmpm_implicit_project(zsmpm_scene *scene, float *inout, int64_t ndofs,
                                              void *stream);
/* ImplicitMPMSystem::precondition (ImplicitMPM.hpp:139-153; DivPernodeMass, :126-137):
 * out = in / m where m > 0; other entries of out are left unchanged. */
ZSMPM_API zsmpm_status zsmpm_implicit_precondition(zsmpm_scene *scene, const float *in, float *out,
                                                   int64_t ndofs, void *stream);

/* ConjugateGradient<T, dim>'s settings (math/linear/ConjugateGradient.hpp:10-38). */
typedef struct {
  int32_t max_iters; /* maxIters (the reference's default: 1000) */
  float tol;         /* tol (1e-6 for float) */
  float rel_tol;     /* relTol (0.5); the loop stops once sqrt(r.q) <= min(rel_tol * its first value, tol) */
} zsmpm_cg_options;

/* ConjugateGradient::solve (ConjugateGradient.hpp:69-172) with the implicit system above as
 * its matrix: x (in: initial guess; out: result) and b are dof vectors.  The iterations run on
 * the device; their scalars stay in device memory, and the host reads the stopping flag once
 * every 8 iterations.  opts may be null (the reference's defaults).  iters_out (host, may be
 * null) receives the iteration count solve returns.  The call synchronises `stream`.  Its
 * four scratch vectors are allocated on the first call and grown when ndofs grows.  Entries of
 * the preconditioned residual that the reference leaves unwritten (nodes without mass) start
 * at zero here. */
ZSMPM_API zsmpm_status zsmpm_implicit_cg(zsmpm_scene *scene, float *x, const float *b, int64_t ndofs,
                                         float dt, const zsmpm_cg_options *opts, int32_t *iters_out,
                                         void *stream);

/* ---- batched scenes ------------------------------------------------------------ */
/* Many independent MPM systems advanced together: every stage is one launch over the blocks
 * of all scenes, and zsmpm_run replays one CUDA graph for the whole batch.  The scenes share
 * dx, dt, gravity and walls (desc; walls in each scene's own [0,1]^3) and have a material
 * each.  Particle positions stay in scene coordinates; scene s's block keys are offset by 32
 * blocks per axis times its slot (s & 7, (s >> 3) & 7, s >> 6), so the scenes never share a
 * block.  Limits: 1/dx <= 176, at most 65,536 scenes, each scene's particles inside
 * [-4 * 8 dx, 27 * 8 dx) per axis (else ZSMPM_ERR_OUT_OF_DOMAIN).  Drucker-Prager scenes run
 * the committed plasticity ordering.  No counterpart in the reference, which advances one
 * system per launch sequence. */
ZSMPM_API zsmpm_status zsmpm_batch_create(const zsmpm_scene_desc *desc, const zsmpm_material *materials,
                                          int32_t nscenes, zsmpm_scene **out);
/* Particles of all scenes concatenated in scene order, counts[nscenes] per scene.  Downloads
 * (zsmpm_scene_download) return them in the same order.  Other scene calls (run, substep,
 * stages, status, download, views, timing, autotune) work on a batch as on one scene. */
ZSMPM_API zsmpm_status zsmpm_batch_upload(zsmpm_scene *s, const zsmpm_particle_arrays *p, const int64_t *counts,
                                          int32_t on_device, void *stream);
ZSMPM_API zsmpm_status zsmpm_batch_num_scenes(const zsmpm_scene *s, int32_t *out);

/* ---- launch-shape autotuner ----------------------------------------------------- */
typedef struct {
  int32_t g2p_threads;      /* G2P CTA size: 128 or 256 (0 = default 256) */
  int32_t g2p_ctas_per_sm;  /* persistent G2P CTAs per SM, 1-6 (0 = default: 3, learned 2) */
  int32_t p2g_ctas_per_sm;  /* persistent P2G CTAs per SM, 1-4 (0 = the staging depth's
                               default: 4 for 8 ranks, 3 for 12, 2 for 16) */
  float g2p_ms, p2g_ms;     /* stage times of the chosen shapes (autotune output) */
  int32_t p2g_ranks;        /* P2G staging depth: particles per cell staged per round, 8, 12 or
                               16 (0 = 12); deeper staging means fewer rounds on dense cells and
                               more shared memory per CTA */
} zsmpm_tuning;

/* Times G2P over CTA size x CTAs per SM, and P2G over staging depth x CTAs per SM, on the
 * uploaded particles (one untimed and `trials` timed substeps per candidate; this advances the
 * simulation by those substeps), keeps the fastest of each and returns them in *out
 * (optional). */
ZSMPM_API zsmpm_status zsmpm_autotune(zsmpm_scene *s, int32_t trials, zsmpm_tuning *out, void *stream);
ZSMPM_API zsmpm_status zsmpm_set_tuning(zsmpm_scene *s, const zsmpm_tuning *t);

/* ---- learned return-mapping closure -------------------------------------------- */
/* An MLP 6 -> 64 -> 64 -> 64 -> 6 (SiLU) that replaces the return-mapping branch of the
 * constitutive update inside G2P (ConstitutiveModel_Vol_dP.hpp:241-325 for Drucker-Prager,
 * SnowPlasticity.hpp:24-32 for snow).  Inputs: the log singular values of the trial F (sorted
 * as the SVD returns them) and three material/state features (Drucker-Prager: friction angle
 * in degrees, cohesion as a log-strain shift, logJp; snow: theta_c, theta_s, log Jp).
 * Outputs: projected minus trial log strain (3) and principal Kirchhoff stress (3).  Trained
 * on the GPU by this library's own forward/backward/Adam kernels on pairs generated by the
 * plain return map; inference inside G2P runs in BF16 on tensor cores with FP32 accumulation,
 * falls back to the plain return map per particle whose inputs leave the training hull
 * (per-feature min/max), and audits a sample of particles against the plain map.  No
 * counterpart in the reference. */
typedef struct zsmpm_closure zsmpm_closure;

typedef struct {
  int32_t model;            /* zsmpm_model: ZSMPM_DRUCKER_PRAGER or ZSMPM_SNOW */
  float params[9158];       /* FP32 weights: W1[64][6] b1 W2[64][64] b2 W3[64][64] b3 W4[6][64] b4 */
  float in_mean[6], in_inv_std[6];  /* input normalisation (x - mean) * inv_std */
  float in_min[6], in_max[6];       /* training hull of the raw inputs */
  float out_scale[6];               /* outputs are network outputs times out_scale */
} zsmpm_closure_state;

typedef struct {
  int64_t audited;          /* network-projected particle updates checked against the plain return map */
  double mean_rel_error;    /* mean of |tau_mlp - tau_plain| / (|tau_plain| + 1e-4 (3 lambda + 2 mu)) */
  double max_rel_error;
  double agg_rel_error;     /* sqrt(sum |dtau|^2 / sum |tau_plain|^2) over the audited particles */
  int64_t fallbacks;        /* projections outside the training hull that used the plain map */
  int64_t network_updates;  /* particle updates whose projection the network gave */
  int64_t updates;          /* all particle updates of G2P with the closure attached */
} zsmpm_closure_audit;

/* Rows of the last dataset: generated (random plus logged) and kept (those the plain return
 * map projects, the training set; G2P decides the branch exactly and runs the network only for
 * projections). */
ZSMPM_API zsmpm_status zsmpm_closure_dataset_size(const zsmpm_closure *c, int64_t *generated, int64_t *kept);
ZSMPM_API zsmpm_status zsmpm_closure_create(const zsmpm_material *mat, int32_t device, zsmpm_closure **out);
ZSMPM_API zsmpm_status zsmpm_closure_destroy(zsmpm_closure *c);
/* Training set: n_random random trial states (log singular values uniform in
 * [log 0.5, log 2]; Drucker-Prager friction 20-45 deg, cohesion 0-100 Pa mapped to a
 * log-strain shift by 1/(3 lambda + 2 mu), zero for a quarter of the samples, logJp zero for
 * half of them and else uniform in [0, 0.2]; snow theta_c 0.015-0.035, theta_s 0.005-0.01,
 * log Jp in [-0.3, 0.3]) plus n_logged raw feature rows (device pointer, 6 floats each, e.g.
 * from zsmpm_scene_set_state_log); targets from the plain return map.  Sets the input
 * normalisation and the training hull (per-feature min/max of the training inputs). */
ZSMPM_API zsmpm_status zsmpm_closure_build_dataset(zsmpm_closure *c, int64_t n_random, uint64_t seed,
                                                   const float *logged, int64_t n_logged, void *stream);
/* Adam on the mean squared error of normalised outputs, batches of `batch` samples;
 * loss_out (host, `epochs` floats, optional) receives each epoch's mean loss. */
ZSMPM_API zsmpm_status zsmpm_closure_train(zsmpm_closure *c, int32_t epochs, int32_t batch, float lr,
                                           uint64_t seed, float *loss_out, void *stream);
/* Loss and its gradient (mean over n samples) by the training kernels, for gradient checks:
 * x, y raw device rows [n][6]; grad device [9158]; loss device [1]. */
ZSMPM_API zsmpm_status zsmpm_closure_loss_grad(zsmpm_closure *c, const float *x, const float *y, int64_t n,
                                               float *grad, float *loss, void *stream);
/* Network outputs (unscaled D and tau) of raw feature rows (device [n][6]).  bf16 selects the
 * path: 0 an FP32 forward of the master weights; 1 the BF16 mma.sync forward that G2P runs
 * (one warp per 32 rows, activations in registers); 2 a BF16 tcgen05 forward (5th-generation
 * tensor cores: 128-row tiles per CTA, operands in shared memory, FP32 accumulators in tensor
 * memory); 3 the tcgen05 forward with split-BF16 operands (weights and activations as hi + lo
 * BF16 pairs, A_hi W_hi + A_hi W_lo + A_lo W_hi per layer into the FP32 accumulator; SiLU in
 * FP32), the path the substep's projections take.  Asynchronous; zsmpm_closure_status reports a
 * tcgen05 wait that gave up. */
ZSMPM_API zsmpm_status zsmpm_closure_infer(zsmpm_closure *c, const float *x, float *y, int64_t n, int32_t bf16,
                                           void *stream);
/* Synchronises the device and reports (then clears) a bounded tensor-core wait that gave up
 * in zsmpm_closure_infer (ZSMPM_ERR_TIMEOUT). */
ZSMPM_API zsmpm_status zsmpm_closure_status(zsmpm_closure *c);
/* The plain return map's (D, tau) for raw feature rows (device [n][6]). */
ZSMPM_API zsmpm_status zsmpm_closure_targets(zsmpm_closure *c, const float *x, float *y, int64_t n, void *stream);
ZSMPM_API zsmpm_status zsmpm_closure_get_state(zsmpm_closure *c, zsmpm_closure_state *out);
ZSMPM_API zsmpm_status zsmpm_closure_set_state(zsmpm_closure *c, const zsmpm_closure_state *in);
/* Attach a trained closure to a scene (NULL detaches; the scene keeps the closure's device
 * pointers, so destroy the closure only after detaching it); audit_period N checks one
 * particle in N per substep against the plain map (0 = no audit).  Needs the committed
 * plasticity ordering.  On a batch the closure serves every scene of its material model and
 * the others keep the plain return map; the network works in units of each scene's
 * 3 lambda + 2 mu, so scenes that share the closure material's Poisson ratio share it. */
ZSMPM_API zsmpm_status zsmpm_scene_set_closure(zsmpm_scene *s, zsmpm_closure *c, int32_t audit_period);
/* Audit totals since the closure was attached or the last reset (synchronises). */
ZSMPM_API zsmpm_status zsmpm_scene_closure_audit(zsmpm_scene *s, zsmpm_closure_audit *out, int32_t reset);
/* Log the raw closure features of the trial state of one particle in `period` per substep into
 * buffer (device, cap x 6) during G2P; period 0 stops logging.  Resets the count. */
ZSMPM_API zsmpm_status zsmpm_scene_set_state_log(zsmpm_scene *s, float *buffer, int64_t cap, int32_t period);
/* Rows logged so far (at most cap; synchronises). */
ZSMPM_API zsmpm_status zsmpm_scene_state_log_count(zsmpm_scene *s, int64_t *count_out);

/* ---- particle output (io/ParticleIO.hpp:11-22) ---------------------------------- */
/* Houdini classic binary geometry (.bgeo), the format zs::write_partio writes through partio:
 * big-endian "Bgeo" V5, one point per particle with its position as P (and w = 1), one
 * particle-system primitive over all points.  Host arrays; the path must end in ".bgeo"
 * (the gzip-compressed ".bgeo.gz" that partio also writes is not built).
 * zsmpm_write_partio replaces write_partio<float,3>(filename, data, tag): with tag
 * "position" (or null) data[n][3] are the positions; with another tag they are stored as a
 * vector point attribute of that name and P is zero.  _with_stress and _with_grid replace
 * write_partio_with_stress (a float attribute "stress") and write_partio_with_grid (a vector
 * attribute "force").  No device needed. */
ZSMPM_API zsmpm_status zsmpm_write_partio(const char *path, const float *data, int64_t n, const char *tag);
ZSMPM_API zsmpm_status zsmpm_write_partio_with_stress(const char *path, const float *pos, const float *stress,
                                                      int64_t n);
ZSMPM_API zsmpm_status zsmpm_write_partio_with_grid(const char *path, const float *pos, const float *force,
                                                    int64_t n);
/* The scene's particle positions, in upload order, written as with zsmpm_write_partio
 * (synchronises). */
ZSMPM_API zsmpm_status zsmpm_scene_write_partio(zsmpm_scene *scene, const char *path);

/* ---- allocation-free variant --------------------------------------------------- */
/* Block activation without any device allocation.  No counterpart in the reference: it is
 * for callers that cannot call cudaMalloc at this point -- hosts whose own memory pool has
 * already reserved the GPU, plug-in or real-time loops that forbid allocation after
 * start-up.  Same result as
 * zsmpm_activate_blocks: the active block keys of the particles at x (device pointer,
 * 3 floats per particle as in zs::Particles "x") after the +{0,1}^3 enlargement, ascending
 * by (bx, by, bz), written to keys_out (device, cap_blocks x 3 int32), and their count to
 * *count_out (device int32), or a negative code: -1 table, block or bounding-box limit
 * reached, -2 more than cap_blocks blocks, -3 a position is NaN/Inf or out of range.
 * Its scratch is one fixed array of about 3 MB in device memory, held on every GPU that
 * loads the library until the process exits; it limits a call to 1,048,576 particles
 * (larger n, or n < 1, is rejected with ZSMPM_ERR_CAPACITY), 32,748 active blocks (a
 * 32,768-slot table on every call, whatever n) and an active-block bounding box of 2^21
 * positions.  The array's device address is looked up once per CUDA context, on the first
 * call made with that context current, so make that first call before any stream capture;
 * a context recreated after cudaDeviceReset gets its own lookup.
 * All calls share the array and each overwrites the last one's contents; calls whose work
 * overlaps on the GPU race and give undefined results. */
ZSMPM_API zsmpm_status zsmpm_activate_blocks_noalloc(const float *x, int64_t n, float dx,
                                                     int32_t *keys_out, int32_t cap_blocks,
                                                     int32_t *count_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* ZSMPM_H */
