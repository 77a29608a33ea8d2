// Host runtime of libzsmpm.so: the C ABI declared in include/zsmpm.h.
//
// A scene owns every device buffer of one MPM system (particles double-buffered in binned
// order, the HashTable<i32,3,int>-layout block table, the sparse grid of 8^3 blocks and
// the binning scratch).  Stages enqueue kernels on the caller's stream; zsmpm_run replays
// a CUDA graph of four substeps (the particle buffers alternate between them).
#include <algorithm>
#include <cstdint>
#include <initializer_list>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "zsmpm.h"
#include "zsmpm_internal.h"

using namespace zsmpm;

struct zsmpm_scene {
  zsmpm_scene_desc desc{};
  int device = 0;
  scene_device dev{};
  particle_buffers bufs[2];
  int cur = 0;
  bool uploaded = false;
  bool binned = false;  // src[] valid for the current particle order
  int bins_since_activation = 0;  // a second binning after one activation recounts every particle
  // the two sets of cell and block starts the binnings alternate between (by particle buffer parity)
  int *cell_start_buf[2] = {nullptr, nullptr};
  int *block_start_buf[2] = {nullptr, nullptr};
  cudaStream_t last_stream = nullptr;
  // graphs of kGraphSubsteps consecutive substeps, one per starting buffer parity
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  cudaStream_t graph_stream = nullptr;
  // the learned closure's pass (network and finish) deferred to a second stream beside the next
  // substep's activation and binning, joined before that substep's P2G
  cudaStream_t side_stream = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  bool join_pending = false;
  // stage timing
  bool timing = false;
  cudaEvent_t ev[6] = {};
  float stage_ms[5] = {};
  std::vector<void *> allocations;
  double *audit = nullptr;                  // closure audit accumulators (device, 8 doubles)
  // batched scenes
  int nscenes = 0;                          // 0: a single scene
  bool any_plastic = false;
  std::vector<int64_t> counts;              // particles of each scene (last upload)
  // bht layout of the active keys (zsmpm_get_bht_view), grown on demand
  int32_t *bht_keys = nullptr, *bht_indices = nullptr, *bht_status = nullptr, *bht_active = nullptr,
          *bht_cnt = nullptr;
  int64_t bht_cap = 0;
  // device staging for host-pointer uploads and downloads (AoS arrays), kept between calls
  float *staging = nullptr;
  size_t staging_floats = 0;
  unsigned long long *log_count = nullptr;  // trial-state log counter (device)
  // implicit solve scratch: four dof vectors and the solver state, grown on demand
  float *cg_buf = nullptr;
  int64_t cg_cap = 0;
  cg_state *cg = nullptr;
  // sparse level-set boundaries: their device maps and distances, freed by clear or destroy
  int nlevelsets = 0;
  std::vector<void *> levelset_buffers;
};

namespace {

thread_local std::string g_error;

zsmpm_status fail(zsmpm_status st, const std::string &msg) {
  g_error = msg;
  return st;
}

zsmpm_status cuda_fail(cudaError_t e, const char *what) {
  return fail(ZSMPM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define ZS_TRY(expr, what)                        \
  do {                                            \
    cudaError_t e__ = (expr);                     \
    if (e__ != cudaSuccess) return cuda_fail(e__, what); \
  } while (0)

template <class T> zsmpm_status dev_alloc(zsmpm_scene *s, T **p, size_t count, const char *what) {
  void *ptr = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&ptr, bytes);
  if (e != cudaSuccess) return cuda_fail(e, what);
  s->allocations.push_back(ptr);
  *p = static_cast<T *>(ptr);
  return ZSMPM_OK;
}

#define ZS_ALLOC(ptr, count, what)                             \
  do {                                                         \
    zsmpm_status st__ = dev_alloc(s, &(ptr), (count), (what)); \
    if (st__ != ZSMPM_OK) return st__;                         \
  } while (0)

int64_t next_2pow(int64_t n) {
  int64_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

material_dev make_material(const zsmpm_material &m) {
  material_dev d{};
  d.model = m.model;
  d.mode = m.model == ZSMPM_SNOW ? 0 : m.plasticity_mode;
  d.volume_correction = m.volume_correction;
  // ConstitutiveModel.hpp:34-38 (mu evaluated through the double literal 0.5)
  d.mu = (float)(0.5 * (double)m.E / (double)(1.f + m.nu));
  d.lambda = m.E * m.nu / ((1.f + m.nu) * (1.f - 2.f * m.nu));
  d.volume = m.volume;
  d.cohesion = m.cohesion;
  d.beta = m.beta;
  const float sin_phi = (float)std::sin((double)m.friction_deg / 180.0 * 3.14159265358979323846);
  d.yield_surface = 0.816496580927726f * 2.f * sin_phi / (3.f - sin_phi);
  d.hardening = m.hardening;
  d.theta_c = m.theta_c;
  d.theta_s = m.theta_s;
  d.friction_deg = m.friction_deg;
  return d;
}

cudaStream_t as_stream(void *st) { return static_cast<cudaStream_t>(st); }

zsmpm_status check_scene(zsmpm_scene *s, bool need_particles) {
  if (!s) return fail(ZSMPM_ERR_INVALID_ARG, "scene is null");
  if (need_particles && !s->uploaded) return fail(ZSMPM_ERR_NOT_READY, "no particles uploaded");
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  return ZSMPM_OK;
}

void bind_buffers(zsmpm_scene *s) {
  s->dev.cur = s->bufs[s->cur];
  s->dev.nxt = s->bufs[s->cur ^ 1];
  // a binning writes the set of its particle buffer parity; the last binning (before the G2P
  // that flipped the parity) wrote the other one
  s->dev.cell_start = s->cell_start_buf[s->cur];
  s->dev.block_start = s->block_start_buf[s->cur];
  s->dev.cell_start_prev = s->cell_start_buf[s->cur ^ 1];
  s->dev.block_start_prev = s->block_start_buf[s->cur ^ 1];
}

zsmpm_status status_from_word(int w) {
  if (w == 0) return ZSMPM_OK;
  std::string msg = "device status:";
  zsmpm_status st = ZSMPM_ERR_CAPACITY;
  if (w & kStatusOutOfDomain) {
    msg += " particle position NaN/Inf or outside the block-key range;";
    st = ZSMPM_ERR_OUT_OF_DOMAIN;
  }
  if (w & kStatusTableFull) {
    msg += " hash table full;";
    st = ZSMPM_ERR_TABLE_FULL;
  }
  if (w & kStatusCapacity) msg += " block capacity exceeded;";
  if (w & kStatusBitmap) msg += " active-block bounding box too large;";
  if (w & kStatusMissingBlock) msg += " particle stencil outside its block neighbourhood;";
  if (w & kStatusTimeout) {
    msg += " bounded wait gave up;";
    st = ZSMPM_ERR_TIMEOUT;
  }
  return fail(st, msg);
}

// the scene's staging buffer with room for `floats` floats (grown, never shrunk)
cudaError_t staging_for(zsmpm_scene *s, size_t floats) {
  if (floats <= s->staging_floats) return cudaSuccess;
  if (s->staging) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return e;
    cudaFree(s->staging);
    s->staging = nullptr;
    s->staging_floats = 0;
  }
  cudaError_t e = cudaMalloc(&s->staging, floats * sizeof(float));
  if (e == cudaSuccess) s->staging_floats = floats;
  return e;
}

zsmpm_status allocate_particles(zsmpm_scene *s, int64_t cap) {
  const bool plastic = s->desc.material.model != ZSMPM_FIXED_COROTATED || s->any_plastic;
  for (int k = 0; k < 2; ++k) {
    particle_buffers &b = s->bufs[k];
    ZS_ALLOC(b.xm, cap, "alloc xm");
    ZS_ALLOC(b.v, cap, "alloc v");
    ZS_ALLOC(b.C, 9 * mat_capacity(cap), "alloc C");
    ZS_ALLOC(b.A, 9 * mat_capacity(cap), "alloc A");
    ZS_ALLOC(b.F, 9 * mat_capacity(cap), "alloc F");
    if (plastic) ZS_ALLOC(b.plastic, cap, "alloc plastic");
    ZS_ALLOC(b.id, cap, "alloc id");
    if (s->nscenes > 0) ZS_ALLOC(b.sid, cap, "alloc scene ids");
  }
  scene_device &d = s->dev;
  ZS_ALLOC(d.key32, cap, "alloc key32");
  ZS_ALLOC(d.rnk, cap, "alloc rnk");
  ZS_ALLOC(d.tmp, cap, "alloc tmp");
  ZS_ALLOC(d.src, cap, "alloc src");
  // incremental binning: a flag per slot and a list of the particles that left their cell (a
  // G2P whose movers overflow the list makes the next binning a full one)
  d.prm.mover_cap = (int)std::min<int64_t>(cap / 4 + 1024, 0x7fffffff);
  ZS_ALLOC(d.moved, cap, "alloc moved flags");
  ZS_ALLOC(d.movers, d.prm.mover_cap, "alloc movers");
  ZS_ALLOC(d.mover_pos, d.prm.mover_cap, "alloc mover positions");
  ZS_ALLOC(d.dirty, d.prm.mover_cap, "alloc dirty cells");
  return ZSMPM_OK;
}

zsmpm_status allocate_blocks(zsmpm_scene *s, int64_t n) {
  scene_device &d = s->dev;
  int64_t expected = s->desc.table_expected > 0 ? s->desc.table_expected : std::max<int64_t>(n / 512, 64);
  const int64_t T = next_2pow(expected) * 16;
  if (T > (int64_t)1 << 30) return fail(ZSMPM_ERR_CAPACITY, "hash table too large");
  d.prm.table_size = (int)T;
  d.prm.nb_cap = (int)std::max<int64_t>(1, std::min<int64_t>(T - 20, std::max<int64_t>(65536, n / 16)));
  d.prm.bitmap_cap = 1 << 23;  // 2^28 dense block positions
  const int64_t nbc = d.prm.nb_cap;
  ZS_ALLOC(d.pk, T, "alloc table pk");
  ZS_ALLOC(d.tkeys, 3 * T, "alloc table keys");
  ZS_ALLOC(d.tidx, T, "alloc table indices");
  ZS_ALLOC(d.tstatus, T, "alloc table status");
  ZS_ALLOC(d.active_keys, 3 * nbc, "alloc active keys");
  ZS_ALLOC(d.view_cnt, 1, "alloc cnt");
  ZS_ALLOC(d.ins_pk, nbc, "alloc ins_pk");
  ZS_ALLOC(d.ins_slot, nbc, "alloc ins_slot");
  ZS_ALLOC(d.blk_pk, nbc, "alloc blk_pk");
  ZS_ALLOC(d.bmask, nbc, "alloc block move masks");
  ZS_ALLOC(d.nbr, 8 * nbc, "alloc nbr");
  ZS_ALLOC(d.bitmap, d.prm.bitmap_cap, "alloc bitmap");
  ZS_ALLOC(d.word_prefix, (int64_t)d.prm.bitmap_cap + 1, "alloc word prefix");
  ZS_ALLOC(d.ctr, kCtrCount, "alloc counters");
  ZS_ALLOC(d.block_count, nbc, "alloc block count");
  ZS_ALLOC(d.work_order, nbc, "alloc work order");
  ZS_ALLOC(s->block_start_buf[0], nbc + 1, "alloc block start");
  ZS_ALLOC(s->block_start_buf[1], nbc + 1, "alloc block start");
  ZS_ALLOC(d.cell_count, 512 * nbc, "alloc cell count");
  ZS_ALLOC(s->cell_start_buf[0], 512 * nbc, "alloc cell start");
  ZS_ALLOC(s->cell_start_buf[1], 512 * nbc, "alloc cell start");
  ZS_ALLOC(d.old_pk, nbc, "alloc previous block keys");
  ZS_ALLOC(d.new_of_old, nbc, "alloc previous block map");
  ZS_ALLOC(d.scan_part, 2 * kScanCtas + 1, "alloc scan partials");
  ZS_ALLOC(d.grid, (size_t)kGridChannels * 512 * nbc, "alloc grid");
  ZS_TRY(cudaMemset(d.bitmap, 0, sizeof(uint32_t) * d.prm.bitmap_cap), "memset bitmap");
  ZS_TRY(cudaMemset(d.ctr, 0, sizeof(int) * kCtrCount), "memset counters");
  ZS_TRY(cudaMemset(d.block_count, 0, sizeof(int) * nbc), "memset block count");
  ZS_TRY(cudaMemset(d.cell_count, 0, sizeof(int) * 512 * nbc), "memset cell count");
  ZS_TRY(cudaMemset(d.view_cnt, 0, sizeof(int)), "memset cnt");
  ZS_TRY(cudaMemset(d.tstatus, 0xff, sizeof(int) * T), "memset table status");
  return ZSMPM_OK;
}

void release_bht(zsmpm_scene *s) {
  for (int32_t **p : {&s->bht_keys, &s->bht_indices, &s->bht_status, &s->bht_active, &s->bht_cnt}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  s->bht_cap = 0;
}

void release(zsmpm_scene *s) {
  release_bht(s);
  if (s->staging) cudaFree(s->staging);
  s->staging = nullptr;
  s->staging_floats = 0;
  for (int k = 0; k < 2; ++k)
    if (s->graph[k]) cudaGraphExecDestroy(s->graph[k]);
  for (auto &e : s->ev)
    if (e) cudaEventDestroy(e);
  if (s->fork_ev) cudaEventDestroy(s->fork_ev);
  if (s->join_ev) cudaEventDestroy(s->join_ev);
  if (s->side_stream) cudaStreamDestroy(s->side_stream);
  if (s->graph_stream) cudaStreamDestroy(s->graph_stream);
  s->fork_ev = s->join_ev = nullptr;
  s->side_stream = s->graph_stream = nullptr;
  for (void *p : s->allocations) cudaFree(p);
  s->allocations.clear();
  for (void *p : s->levelset_buffers) cudaFree(p);
  s->levelset_buffers.clear();
}

void invalidate_graphs(zsmpm_scene *s) {
  for (int k = 0; k < 2; ++k)
    if (s->graph[k]) {
      cudaGraphExecDestroy(s->graph[k]);
      s->graph[k] = nullptr;
    }
}

zsmpm_status read_status(zsmpm_scene *s) {
  int w = 0;
  ZS_TRY(cudaMemcpy(&w, &s->dev.ctr[kCtrStatus], sizeof(int), cudaMemcpyDeviceToHost), "read status");
  if (w) {
    // report once, then clear so that the next call starts clean
    cudaMemset(&s->dev.ctr[kCtrStatus], 0, sizeof(int));
  }
  return status_from_word(w);
}

// Substeps kept in one CUDA graph: the closure pass of every substep but the last runs beside
// the next substep's activation and binning.
constexpr int kGraphSubsteps = 4;

// defer_closure: with a learned closure attached, leave the closure pass (network and finish)
// to the side stream and have the next substep_enqueue join it before its P2G (zsmpm_run's
// graphs only; the side stream and its events must exist)
zsmpm_status substep_enqueue(zsmpm_scene *s, cudaStream_t st, bool defer_closure = false) {
  bind_buffers(s);
  if (s->timing) cudaEventRecord(s->ev[0], st);
  ZS_TRY(launch_activate(s->dev, st), "activate");
  if (s->timing) cudaEventRecord(s->ev[1], st);
  s->dev.prm.bin_full = 0;
  ZS_TRY(launch_bin(s->dev, st), "bin");
  if (s->timing) cudaEventRecord(s->ev[2], st);
  if (s->join_pending) {
    // the last substep's closure pass writes F, the affine momentum and the plastic state that
    // this P2G and G2P read
    ZS_TRY(cudaStreamWaitEvent(st, s->join_ev, 0), "join the closure pass");
    s->join_pending = false;
  }
  ZS_TRY(launch_p2g(s->dev, st), "p2g");
  if (s->timing) cudaEventRecord(s->ev[3], st);
  ZS_TRY(launch_grid_update(s->dev, st), "grid update");
  if (s->timing) cudaEventRecord(s->ev[4], st);
  const bool deferred = defer_closure && s->dev.aux.learned && s->side_stream;
  ZS_TRY(launch_g2p(s->dev, st, !deferred), "g2p");
  if (deferred) {
    ZS_TRY(cudaEventRecord(s->fork_ev, st), "fork the closure pass");
    ZS_TRY(cudaStreamWaitEvent(s->side_stream, s->fork_ev, 0), "fork the closure pass");
    ZS_TRY(launch_closure_pass(s->dev, s->side_stream), "closure pass");
    ZS_TRY(cudaEventRecord(s->join_ev, s->side_stream), "closure pass done");
    s->join_pending = true;
  }
  if (s->timing) cudaEventRecord(s->ev[5], st);
  s->cur ^= 1;
  bind_buffers(s);
  return ZSMPM_OK;
}

}  // namespace

namespace zsmpm {
int record_error(int status, const char *message) {
  return (int)fail((zsmpm_status)status, message ? message : "");
}
}  // namespace zsmpm

extern "C" {

ZSMPM_API const char *zsmpm_last_error_string(void) { return g_error.c_str(); }
ZSMPM_API const char *zsmpm_version(void) { return "zsmpm-b200 0.1 (sm_100a)"; }

ZSMPM_API int zsmpm_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

ZSMPM_API zsmpm_status zsmpm_scene_create(const zsmpm_scene_desc *desc, zsmpm_scene **out) {
  if (!desc || !out) return fail(ZSMPM_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (!(desc->dx > 0.f) || !(desc->dt > 0.f)) return fail(ZSMPM_ERR_INVALID_ARG, "dx and dt must be > 0");
  if (desc->material.model < 0 || desc->material.model > 2)
    return fail(ZSMPM_ERR_INVALID_ARG, "unknown material model");
  if (desc->wall_type < 0 || desc->wall_type > 3) return fail(ZSMPM_ERR_INVALID_ARG, "unknown wall type");
  if (desc->threads_per_cta != 0 && desc->threads_per_cta != 128 && desc->threads_per_cta != 256)
    return fail(ZSMPM_ERR_INVALID_ARG, "threads_per_cta must be 0, 128 or 256");
  if (desc->block_order != ZSMPM_BLOCK_ORDER_SORTED)
    return fail(ZSMPM_ERR_INVALID_ARG, "only ZSMPM_BLOCK_ORDER_SORTED is implemented by the device path");
  if (zsmpm_device_count() <= 0) return fail(ZSMPM_ERR_NO_DEVICE, "no CUDA device visible");
  auto *s = new zsmpm_scene();
  s->desc = *desc;
  s->device = desc->device;
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) {
    delete s;
    return cuda_fail(e, "cudaSetDevice");
  }
  scene_params &p = s->dev.prm;
  p.dx = desc->dx;
  p.inv_dx = 1.f / desc->dx;
  {
    int ex = 0;
    p.dx_pow2 = std::isfinite(desc->dx) && desc->dx > 0.f && std::frexp(desc->dx, &ex) == 0.5f ? 1 : 0;
  }
  p.dt = desc->dt;
  p.kappa = desc->dt * (4.f * p.inv_dx * p.inv_dx);  // dt * D_inv (P2G.hpp:52, :104)
  p.four_over_dx = 4.f * p.inv_dx;
  for (int d = 0; d < 3; ++d) p.gravity[d] = desc->gravity[d];
  p.wall_type = desc->wall_type;
  p.wall_cells = desc->wall_cells;
  p.mat = make_material(desc->material);
  p.g2p_threads = desc->threads_per_cta;
  for (auto &ev : s->ev) cudaEventCreate(&ev);
  e = prepare_kernels();
  if (e != cudaSuccess) {
    release(s);
    delete s;
    return cuda_fail(e, "kernel attributes");
  }
  {
    collider_dev *cols = nullptr;
    int *ncol = nullptr;
    zsmpm_status st = dev_alloc(s, &cols, kMaxColliders, "colliders");
    if (st == ZSMPM_OK) st = dev_alloc(s, &ncol, 1, "collider count");
    if (st == ZSMPM_OK && cudaMemset(ncol, 0, sizeof(int)) != cudaSuccess) st = fail(ZSMPM_ERR_CUDA, "collider count");
    if (st != ZSMPM_OK) {
      release(s);
      delete s;
      return st;
    }
    p.colliders = cols;
    p.ncolliders = ncol;
    levelset_dev *lss = nullptr;
    int *nls = nullptr;
    st = dev_alloc(s, &lss, kMaxLevelsets, "level sets");
    if (st == ZSMPM_OK) st = dev_alloc(s, &nls, 1, "level-set count");
    if (st == ZSMPM_OK && cudaMemset(nls, 0, sizeof(int)) != cudaSuccess) st = fail(ZSMPM_ERR_CUDA, "level-set count");
    if (st != ZSMPM_OK) {
      release(s);
      delete s;
      return st;
    }
    p.levelsets = lss;
    p.nlevelsets = nls;
  }
  *out = s;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_scene_add_levelset(zsmpm_scene *s, const zsmpm_levelset_desc *d, void *stream) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (s->nscenes > 0) return fail(ZSMPM_ERR_INVALID_ARG, "level sets apply to single scenes");
  if (!d) return fail(ZSMPM_ERR_INVALID_ARG, "null level set");
  if (s->nlevelsets >= kMaxLevelsets) return fail(ZSMPM_ERR_CAPACITY, "at most ZSMPM_MAX_LEVELSETS level sets");
  if (d->type < 0 || d->type > 2) return fail(ZSMPM_ERR_INVALID_ARG, "level-set type must be sticky, slip or separate");
  if (d->nblocks < 0 || (d->nblocks > 0 && (!d->keys || !d->sdf)))
    return fail(ZSMPM_ERR_INVALID_ARG, "level-set blocks need keys and distances");
  levelset_dev L{};
  L.type = d->type;
  L.nblocks = d->nblocks;
  L.background = d->background;
  std::memcpy(L.sinv, d->sinv, sizeof(L.sinv));
  std::memcpy(L.rinv, d->rinv, sizeof(L.rinv));
  std::memcpy(L.t, d->t, sizeof(L.t));
  int64_t lo[3] = {0, 0, 0}, hi[3] = {-1, -1, -1};
  for (int b = 0; b < d->nblocks; ++b)
    for (int k = 0; k < 3; ++k) {
      const int32_t v = d->keys[3 * b + k];
      if (v % 8 != 0) return fail(ZSMPM_ERR_INVALID_ARG, "level-set block keys are block origins (multiples of 8)");
      const int64_t bc = v / 8;
      if (b == 0 || bc < lo[k]) lo[k] = bc;
      if (b == 0 || bc > hi[k]) hi[k] = bc;
    }
  int64_t cells = 1;
  for (int k = 0; k < 3; ++k) {
    L.lo[k] = (int)lo[k];
    L.dim[k] = (int)(hi[k] - lo[k] + 1);
    cells *= std::max<int64_t>(L.dim[k], 0);
  }
  if (cells > ((int64_t)1 << 22)) return fail(ZSMPM_ERR_CAPACITY, "level-set bounding box above 2^22 blocks");
  std::vector<int> map((size_t)std::max<int64_t>(cells, 1), -1);
  for (int b = 0; b < d->nblocks; ++b) {
    const int64_t ix = d->keys[3 * b] / 8 - lo[0], iy = d->keys[3 * b + 1] / 8 - lo[1], iz = d->keys[3 * b + 2] / 8 - lo[2];
    int &slot = map[(size_t)((ix * L.dim[1] + iy) * L.dim[2] + iz)];
    if (slot >= 0) return fail(ZSMPM_ERR_INVALID_ARG, "duplicate level-set block key");
    slot = b;
  }
  int *dmap = nullptr;
  float *dsdf = nullptr;
  cudaError_t e = cudaMalloc(&dmap, sizeof(int) * map.size());
  if (e == cudaSuccess) s->levelset_buffers.push_back(dmap);
  if (e == cudaSuccess) e = cudaMalloc(&dsdf, sizeof(float) * 512 * (size_t)std::max(d->nblocks, 1));
  if (e == cudaSuccess) s->levelset_buffers.push_back(dsdf);
  cudaStream_t cs = as_stream(stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dmap, map.data(), sizeof(int) * map.size(), cudaMemcpyHostToDevice, cs);
  if (e == cudaSuccess && d->nblocks > 0)
    e = cudaMemcpyAsync(dsdf, d->sdf, sizeof(float) * 512 * (size_t)d->nblocks, cudaMemcpyHostToDevice, cs);
  L.map = dmap;
  L.sdf = dsdf;
  const int count = s->nlevelsets + 1;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(const_cast<levelset_dev *>(s->dev.prm.levelsets) + s->nlevelsets, &L, sizeof(L),
                        cudaMemcpyHostToDevice, cs);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(const_cast<int *>(s->dev.prm.nlevelsets), &count, sizeof(int), cudaMemcpyHostToDevice, cs);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cs);  // the host sources are local
  if (e != cudaSuccess) return cuda_fail(e, "add level set");
  s->nlevelsets = count;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_scene_clear_levelsets(zsmpm_scene *s) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  ZS_TRY(cudaDeviceSynchronize(), "clear level sets");
  ZS_TRY(cudaMemset(const_cast<int *>(s->dev.prm.nlevelsets), 0, sizeof(int)), "clear level sets");
  for (void *ptr : s->levelset_buffers) cudaFree(ptr);
  s->levelset_buffers.clear();
  s->nlevelsets = 0;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_scene_set_colliders(zsmpm_scene *s, const zsmpm_collider *colliders, int32_t count,
                                                 void *stream) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (s->nscenes > 0) return fail(ZSMPM_ERR_INVALID_ARG, "colliders apply to single scenes");
  if (count < 0 || count > kMaxColliders) return fail(ZSMPM_ERR_INVALID_ARG, "at most ZSMPM_MAX_COLLIDERS colliders");
  if (count > 0 && !colliders) return fail(ZSMPM_ERR_INVALID_ARG, "null colliders");
  static_assert(sizeof(collider_dev) == sizeof(zsmpm_collider), "collider layouts differ");
  std::vector<collider_dev> host(count > 0 ? count : 1);
  for (int k = 0; k < count; ++k) {
    const zsmpm_collider &c = colliders[k];
    if (c.shape < 0 || c.shape > 3) return fail(ZSMPM_ERR_INVALID_ARG, "unknown collider shape");
    if (c.type < 0 || c.type > 2) return fail(ZSMPM_ERR_INVALID_ARG, "collider type must be sticky, slip or separate");
    if (c.shape == ZSMPM_SHAPE_CYLINDER && (c.axis < 0 || c.axis > 2))
      return fail(ZSMPM_ERR_INVALID_ARG, "cylinder axis must be 0, 1 or 2");
    if (!(c.s != 0.f) || !std::isfinite(c.s)) return fail(ZSMPM_ERR_INVALID_ARG, "collider scale must be finite and non-zero");
    std::memcpy(&host[k], &c, sizeof(collider_dev));
  }
  cudaStream_t cs = as_stream(stream);
  if (count > 0)
    ZS_TRY(cudaMemcpyAsync(const_cast<collider_dev *>(s->dev.prm.colliders), host.data(), sizeof(collider_dev) * count,
                           cudaMemcpyHostToDevice, cs),
           "colliders");
  ZS_TRY(cudaMemcpyAsync(const_cast<int *>(s->dev.prm.ncolliders), &count, sizeof(int), cudaMemcpyHostToDevice, cs),
         "collider count");
  // the host copies are local: wait for the copies before they go out of scope
  ZS_TRY(cudaStreamSynchronize(cs), "colliders");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_scene_destroy(zsmpm_scene *s) {
  if (!s) return ZSMPM_OK;
  cudaSetDevice(s->device);
  cudaDeviceSynchronize();
  release(s);
  delete s;
  return ZSMPM_OK;
}

static zsmpm_status prepare_upload(zsmpm_scene *s, int64_t n) {
  if (n <= 0 || n > (int64_t)0x7fffffff) return fail(ZSMPM_ERR_INVALID_ARG, "particle count out of range");
  if (!s->uploaded) {
    int64_t cap = s->desc.max_particles > 0 ? s->desc.max_particles : n;
    if (cap < n) return fail(ZSMPM_ERR_CAPACITY, "more particles than max_particles");
    zsmpm_status st = allocate_particles(s, cap);
    if (st != ZSMPM_OK) return st;
    st = allocate_blocks(s, cap);
    if (st != ZSMPM_OK) return st;
    s->dev.prm.cap = (int)cap;
  } else if (n > s->dev.prm.cap) {
    return fail(ZSMPM_ERR_CAPACITY, "more particles than the scene's capacity");
  }
  s->dev.prm.n = (int)n;
  s->cur = 0;
  bind_buffers(s);
  invalidate_graphs(s);
  return ZSMPM_OK;
}

static zsmpm_status upload_arrays(zsmpm_scene *s, const zsmpm_particle_arrays *p, int64_t n, int32_t on_device,
                                  void *stream);

ZSMPM_API zsmpm_status zsmpm_scene_upload(zsmpm_scene *s, const zsmpm_particle_arrays *p, int64_t n,
                                          int32_t on_device, void *stream) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (s->nscenes > 0) return fail(ZSMPM_ERR_INVALID_ARG, "a batch takes zsmpm_batch_upload");
  return upload_arrays(s, p, n, on_device, stream);
}

static zsmpm_status upload_arrays(zsmpm_scene *s, const zsmpm_particle_arrays *p, int64_t n, int32_t on_device,
                                  void *stream) {
  zsmpm_status st = ZSMPM_OK;
  if (!p || !p->m || !p->x) return fail(ZSMPM_ERR_INVALID_ARG, "m and x are required");
  st = prepare_upload(s, n);
  if (st != ZSMPM_OK) return st;
  cudaStream_t cs = as_stream(stream);
  const float *dm = p->m, *dx = p->x, *dv = p->v, *dC = p->C, *dF = p->F, *dpl = p->plastic;
  if (!on_device) {
    // host arrays go through the scene's staging buffer (26 floats per particle at most)
    ZS_TRY(staging_for(s, 26 * (size_t)n), "upload staging");
    float *base = s->staging;
    auto stage = [&](const float *h, size_t count, const float **d) -> cudaError_t {
      if (!h) {
        *d = nullptr;
        return cudaSuccess;
      }
      float *dst = base;
      base += count;
      *d = dst;
      return cudaMemcpyAsync(dst, h, count * sizeof(float), cudaMemcpyHostToDevice, cs);
    };
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = stage(p->m, n, &dm);
    if (e == cudaSuccess) e = stage(p->x, 3 * n, &dx);
    if (e == cudaSuccess) e = stage(p->v, 3 * n, &dv);
    if (e == cudaSuccess) e = stage(p->C, 9 * n, &dC);
    if (e == cudaSuccess) e = stage(p->F, 9 * n, &dF);
    if (e == cudaSuccess) e = stage(p->plastic, n, &dpl);
    if (e != cudaSuccess) return cuda_fail(e, "upload staging copy");
  }
  cudaError_t e = launch_import(s->dev, dm, dx, dv, dC, dF, dpl, (int)n, cs);
  if (e == cudaSuccess) e = launch_prime(s->dev, cs);
  // host arrays may be reused once the call returns, and the staging buffer is free again
  if (e == cudaSuccess && !on_device) e = cudaStreamSynchronize(cs);
  if (e != cudaSuccess) return cuda_fail(e, "upload");
  s->uploaded = true;
  s->binned = false;
  s->last_stream = cs;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_scene_upload_tilevector(zsmpm_scene *s, const zsmpm_tilevector_view *tv,
                                                     int64_t n, void *stream) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (!tv || !tv->base || tv->lane_width != 32 || tv->off_m < 0 || tv->off_x < 0)
    return fail(ZSMPM_ERR_INVALID_ARG, "tile vector view needs base, lane_width 32, m and x");
  if (s->nscenes > 0) return fail(ZSMPM_ERR_INVALID_ARG, "a batch takes zsmpm_batch_upload");
  st = prepare_upload(s, n);
  if (st != ZSMPM_OK) return st;
  cudaStream_t cs = as_stream(stream);
  cudaError_t e = launch_import_tilevector(s->dev, tv->base, tv->num_channels, tv->off_m, tv->off_x,
                                           tv->off_v, tv->off_C, tv->off_F, tv->off_plastic, (int)n, cs);
  if (e == cudaSuccess) e = launch_prime(s->dev, cs);
  if (e != cudaSuccess) return cuda_fail(e, "upload tilevector");
  s->uploaded = true;
  s->binned = false;
  s->last_stream = cs;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_scene_download(zsmpm_scene *s, zsmpm_particle_arrays *p, int32_t on_device,
                                            void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!p) return fail(ZSMPM_ERR_INVALID_ARG, "null particle arrays");
  cudaStream_t cs = as_stream(stream);
  bind_buffers(s);
  const int64_t n = s->dev.prm.n;
  if (on_device) {
    ZS_TRY(launch_export(s->dev, p->m, p->x, p->v, p->C, p->F, p->plastic, cs), "download");
    return ZSMPM_OK;
  }
  ZS_TRY(staging_for(s, 26 * (size_t)n), "download staging");
  float *dbuf = s->staging;
  float *dm = dbuf, *dx = dm + n, *dv = dx + 3 * n, *dC = dv + 3 * n, *dF = dC + 9 * n, *dpl = dF + 9 * n;
  cudaError_t e = launch_export(s->dev, p->m ? dm : nullptr, p->x ? dx : nullptr, p->v ? dv : nullptr,
                                p->C ? dC : nullptr, p->F ? dF : nullptr, p->plastic ? dpl : nullptr, cs);
  auto get = [&](float *h, const float *d, size_t count) {
    if (h && e == cudaSuccess) e = cudaMemcpyAsync(h, d, count * sizeof(float), cudaMemcpyDeviceToHost, cs);
  };
  get(p->m, dm, n);
  get(p->x, dx, 3 * n);
  get(p->v, dv, 3 * n);
  get(p->C, dC, 9 * n);
  get(p->F, dF, 9 * n);
  get(p->plastic, dpl, n);
  cudaError_t e2 = cudaStreamSynchronize(cs);
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess) return cuda_fail(e, "download");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_scene_write_partio(zsmpm_scene *s, const char *path) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  std::vector<float> x(3 * (size_t)s->dev.prm.n);
  zsmpm_particle_arrays arrs{};
  arrs.x = x.data();
  st = zsmpm_scene_download(s, &arrs, 0, s->last_stream);
  if (st != ZSMPM_OK) return st;
  return zsmpm_write_partio(path, x.data(), s->dev.prm.n, "position");
}

ZSMPM_API zsmpm_status zsmpm_scene_download_tilevector(zsmpm_scene *s, const zsmpm_tilevector_view *tv,
                                                       void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!tv || !tv->base || tv->lane_width != 32) return fail(ZSMPM_ERR_INVALID_ARG, "bad tile vector view");
  bind_buffers(s);
  ZS_TRY(launch_export_tilevector(s->dev, tv->base, tv->num_channels, tv->off_m, tv->off_x, tv->off_v,
                                  tv->off_C, tv->off_F, tv->off_plastic, as_stream(stream)),
         "download tilevector");
  return ZSMPM_OK;
}

ZSMPM_API int64_t zsmpm_scene_num_particles(const zsmpm_scene *s) { return s ? s->dev.prm.n : 0; }

ZSMPM_API zsmpm_status zsmpm_scene_status(zsmpm_scene *s) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (!s->uploaded) return ZSMPM_OK;
  ZS_TRY(cudaStreamSynchronize(s->last_stream), "synchronize");
  return read_status(s);
}

ZSMPM_API zsmpm_status zsmpm_activate_blocks(zsmpm_scene *s, void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  bind_buffers(s);
  ZS_TRY(launch_activate(s->dev, as_stream(stream)), "activate");
  s->binned = false;
  s->bins_since_activation = 0;
  s->last_stream = as_stream(stream);
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_bin_particles(zsmpm_scene *s, void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  bind_buffers(s);
  // only the first binning after an activation may merge the movers of the last G2P
  s->dev.prm.bin_full = s->bins_since_activation > 0 ? 1 : 0;
  cudaError_t e = launch_bin(s->dev, as_stream(stream));
  s->dev.prm.bin_full = 0;
  ZS_TRY(e, "bin");
  s->bins_since_activation += 1;
  s->binned = true;
  s->last_stream = as_stream(stream);
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_p2g(zsmpm_scene *s, void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!s->binned) return fail(ZSMPM_ERR_NOT_READY, "p2g needs zsmpm_activate_blocks and zsmpm_bin_particles first");
  bind_buffers(s);
  ZS_TRY(launch_p2g(s->dev, as_stream(stream)), "p2g");
  s->last_stream = as_stream(stream);
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_grid_update(zsmpm_scene *s, void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!s->binned) return fail(ZSMPM_ERR_NOT_READY, "grid update needs an activated grid");
  bind_buffers(s);
  ZS_TRY(launch_grid_update(s->dev, as_stream(stream)), "grid update");
  s->last_stream = as_stream(stream);
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_g2p(zsmpm_scene *s, void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!s->binned) return fail(ZSMPM_ERR_NOT_READY, "g2p needs a binned, updated grid");
  bind_buffers(s);
  ZS_TRY(launch_g2p(s->dev, as_stream(stream)), "g2p");
  s->cur ^= 1;
  bind_buffers(s);
  s->binned = false;
  s->last_stream = as_stream(stream);
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_scene_set_transfer(zsmpm_scene *s, int32_t transfer, void *stream) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (transfer != ZSMPM_TRANSFER_APIC && transfer != ZSMPM_TRANSFER_CELL)
    return fail(ZSMPM_ERR_INVALID_ARG, "unknown transfer scheme");
  if (transfer == ZSMPM_TRANSFER_CELL) {
    if (s->nscenes > 0) return fail(ZSMPM_ERR_INVALID_ARG, "the cell-centric transfers run on single scenes");
    if (s->desc.material.model != ZSMPM_FIXED_COROTATED)
      return fail(ZSMPM_ERR_INVALID_ARG,
                  "the cell-centric transfers are built for fixed corotated (P2C2G's plasticity branch "
                  "writes the plastic state once per visiting cell)");
    if (s->dev.aux.learned) return fail(ZSMPM_ERR_INVALID_ARG, "detach the learned closure first");
  }
  if (s->dev.prm.transfer == transfer) return ZSMPM_OK;
  invalidate_graphs(s);
  s->dev.prm.transfer = transfer;
  if (s->uploaded) {
    // the affine term the next transfer reads, from the stored state
    cudaStream_t cs = as_stream(stream);
    bind_buffers(s);
    ZS_TRY(launch_prime(s->dev, cs), "transfer affine term");
    s->binned = false;
    s->last_stream = cs;
  }
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_p2c2g(zsmpm_scene *s, int32_t part, void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (s->dev.prm.transfer != kTransferCell)
    return fail(ZSMPM_ERR_INVALID_ARG, "zsmpm_p2c2g needs zsmpm_scene_set_transfer(ZSMPM_TRANSFER_CELL)");
  if (part < ZSMPM_P2C2G_ALL || part > ZSMPM_P2C2G_FORCE) return fail(ZSMPM_ERR_INVALID_ARG, "unknown P2C2G part");
  if (!s->binned) return fail(ZSMPM_ERR_NOT_READY, "p2c2g needs zsmpm_activate_blocks and zsmpm_bin_particles first");
  bind_buffers(s);
  ZS_TRY(launch_p2c2g(s->dev, part, as_stream(stream)), "p2c2g");
  s->last_stream = as_stream(stream);
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_g2c2p(zsmpm_scene *s, void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (s->dev.prm.transfer != kTransferCell)
    return fail(ZSMPM_ERR_INVALID_ARG, "zsmpm_g2c2p needs zsmpm_scene_set_transfer(ZSMPM_TRANSFER_CELL)");
  return zsmpm_g2p(s, stream);
}

ZSMPM_API zsmpm_status zsmpm_substep(zsmpm_scene *s, void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  st = substep_enqueue(s, as_stream(stream));
  if (st != ZSMPM_OK) return st;
  s->binned = false;
  s->last_stream = as_stream(stream);
  if (s->timing) {
    ZS_TRY(cudaEventSynchronize(s->ev[5]), "stage timing");
    for (int k = 0; k < 5; ++k) cudaEventElapsedTime(&s->stage_ms[k], s->ev[k], s->ev[k + 1]);
  }
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_run(zsmpm_scene *s, int32_t nsteps, void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (nsteps < 0) return fail(ZSMPM_ERR_INVALID_ARG, "nsteps < 0");
  cudaStream_t cs = as_stream(stream);
  const bool timing = s->timing;
  s->timing = false;
  // capture kGraphSubsteps substeps starting from the current parity once, on a private
  // stream (capture is not allowed on the legacy default stream); with a learned closure the
  // closure pass of each substep but the last forks to the side stream and joins the next
  // substep before its P2G, so the graph's own end joins every stream it forked
  const int parity = s->cur;
  // (nsteps == 0 only captures: a caller prepares the graph outside a timed region)
  if ((nsteps >= kGraphSubsteps || nsteps == 0) && !s->graph[parity]) {
    if (!s->graph_stream) ZS_TRY(cudaStreamCreateWithFlags(&s->graph_stream, cudaStreamNonBlocking), "graph stream");
    if (!s->side_stream) ZS_TRY(cudaStreamCreateWithFlags(&s->side_stream, cudaStreamNonBlocking), "side stream");
    if (!s->fork_ev) ZS_TRY(cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming), "fork event");
    if (!s->join_ev) ZS_TRY(cudaEventCreateWithFlags(&s->join_ev, cudaEventDisableTiming), "join event");
    ZS_TRY(cudaStreamBeginCapture(s->graph_stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    zsmpm_status a = ZSMPM_OK;
    for (int k = 0; k < kGraphSubsteps && a == ZSMPM_OK; ++k)
      a = substep_enqueue(s, s->graph_stream, k + 1 < kGraphSubsteps);
    s->join_pending = false;  // the last substep joined the pass before it (or capture failed)
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->graph_stream, &g);
    s->cur = parity;  // capture enqueued nothing; restore the parity it advanced
    bind_buffers(s);
    if (a != ZSMPM_OK) {
      if (g) cudaGraphDestroy(g);
      s->timing = timing;
      return a;
    }
    if (e != cudaSuccess) {
      s->timing = timing;
      return cuda_fail(e, "end capture");
    }
    e = cudaGraphInstantiate(&s->graph[parity], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      s->timing = timing;
      return cuda_fail(e, "graph instantiate");
    }
  }
  int done = 0;
  for (; done + kGraphSubsteps <= nsteps; done += kGraphSubsteps) {
    cudaError_t e = cudaGraphLaunch(s->graph[parity], cs);
    if (e != cudaSuccess) {
      s->timing = timing;
      return cuda_fail(e, "graph launch");
    }
  }
  // an even number of substeps leaves the parity unchanged
  for (; done < nsteps; ++done) {
    st = substep_enqueue(s, cs);
    if (st != ZSMPM_OK) {
      s->timing = timing;
      return st;
    }
  }
  s->timing = timing;
  s->binned = false;
  s->last_stream = cs;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_get_table_view(zsmpm_scene *s, zsmpm_table_view *out) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!out) return fail(ZSMPM_ERR_INVALID_ARG, "null view");
  out->keys = s->dev.tkeys;
  out->indices = s->dev.tidx;
  out->status = s->dev.tstatus;
  out->active_keys = s->dev.active_keys;
  out->cnt = s->dev.view_cnt;
  out->table_size = s->dev.prm.table_size;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_download_table(zsmpm_scene *s, int32_t *keys, int32_t *indices, int32_t *status,
                                            int32_t *active_keys, int32_t cap_active, int32_t *count,
                                            int32_t table_size, void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!keys || !indices || !status || !active_keys || !count)
    return fail(ZSMPM_ERR_INVALID_ARG, "null table array");
  if (table_size != s->dev.prm.table_size)
    return fail(ZSMPM_ERR_INVALID_ARG, ("the destination table has " + std::to_string(table_size) +
                                        " slots, the scene's " + std::to_string(s->dev.prm.table_size) +
                                        " (size it for the same expected entry count)")
                                           .c_str());
  cudaStream_t cs = as_stream(stream);
  int nb = 0;
  ZS_TRY(cudaMemcpyAsync(&nb, s->dev.view_cnt, sizeof(int), cudaMemcpyDeviceToHost, cs), "table count");
  ZS_TRY(cudaStreamSynchronize(cs), "table count");
  if (nb > cap_active) return fail(ZSMPM_ERR_CAPACITY, "active-key array too small");
  const size_t T = (size_t)table_size;
  // cudaMemcpyDefault: the destination may be host or device memory (unified addressing)
  ZS_TRY(cudaMemcpyAsync(keys, s->dev.tkeys, T * 3 * sizeof(int), cudaMemcpyDefault, cs), "table keys");
  ZS_TRY(cudaMemcpyAsync(indices, s->dev.tidx, T * sizeof(int), cudaMemcpyDefault, cs), "table indices");
  ZS_TRY(cudaMemcpyAsync(status, s->dev.tstatus, T * sizeof(int), cudaMemcpyDefault, cs), "table status");
  ZS_TRY(cudaMemcpyAsync(active_keys, s->dev.active_keys, (size_t)nb * 3 * sizeof(int), cudaMemcpyDefault, cs),
         "active keys");
  ZS_TRY(cudaMemcpyAsync(count, s->dev.view_cnt, sizeof(int), cudaMemcpyDefault, cs), "table count");
  ZS_TRY(cudaStreamSynchronize(cs), "table copy");
  s->last_stream = cs;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_num_blocks(zsmpm_scene *s, int32_t *out) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!out) return fail(ZSMPM_ERR_INVALID_ARG, "null output");
  ZS_TRY(cudaStreamSynchronize(s->last_stream), "synchronize");
  ZS_TRY(cudaMemcpy(out, s->dev.view_cnt, sizeof(int), cudaMemcpyDeviceToHost), "read block count");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_binning_info(zsmpm_scene *s, int32_t *movers_merged) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!movers_merged) return fail(ZSMPM_ERR_INVALID_ARG, "null output");
  ZS_TRY(cudaStreamSynchronize(s->last_stream), "synchronize");
  ZS_TRY(cudaMemcpy(movers_merged, &s->dev.ctr[kCtrBinInfo], sizeof(int), cudaMemcpyDeviceToHost),
         "read binning info");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_get_grid_view(zsmpm_scene *s, zsmpm_grid_view *out) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!out) return fail(ZSMPM_ERR_INVALID_ARG, "null view");
  int nb = 0;
  st = zsmpm_num_blocks(s, &nb);
  if (st != ZSMPM_OK) return st;
  out->base = s->dev.grid;
  out->num_channels = kGridChannels;
  out->num_blocks = nb;
  out->keys = s->dev.active_keys;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_download_grid(zsmpm_scene *s, int32_t *keys, float *grid, int32_t cap_blocks,
                                           int32_t *out_nblocks) {
  int nb = 0;
  zsmpm_status st = zsmpm_num_blocks(s, &nb);
  if (st != ZSMPM_OK) return st;
  if (out_nblocks) *out_nblocks = nb;
  if (nb > cap_blocks) return fail(ZSMPM_ERR_CAPACITY, "grid output capacity too small");
  if (keys) ZS_TRY(cudaMemcpy(keys, s->dev.active_keys, sizeof(int) * 3 * nb, cudaMemcpyDeviceToHost), "copy keys");
  if (grid)
    ZS_TRY(cudaMemcpy(grid, s->dev.grid, sizeof(float) * kGridChannels * 512 * (size_t)nb, cudaMemcpyDeviceToHost),
           "copy grid");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_download_binning(zsmpm_scene *s, int32_t *order, int32_t *block_start,
                                              int32_t cap_blocks) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!s->binned) return fail(ZSMPM_ERR_NOT_READY, "call zsmpm_bin_particles first");
  int nb = 0;
  st = zsmpm_num_blocks(s, &nb);
  if (st != ZSMPM_OK) return st;
  if (nb > cap_blocks) return fail(ZSMPM_ERR_CAPACITY, "block_start capacity too small");
  const int n = s->dev.prm.n;
  bind_buffers(s);
  if (order) {
    int *d = nullptr;
    ZS_TRY(cudaMalloc(&d, sizeof(int) * n), "binning staging");
    cudaError_t e = launch_export_order(s->dev, d, s->last_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->last_stream);
    if (e == cudaSuccess) e = cudaMemcpy(order, d, sizeof(int) * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "download binning");
  }
  if (block_start)
    ZS_TRY(cudaMemcpy(block_start, s->dev.block_start, sizeof(int) * (nb + 1), cudaMemcpyDeviceToHost),
           "copy block start");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_set_stage_timing(zsmpm_scene *s, int32_t enabled) {
  if (!s) return fail(ZSMPM_ERR_INVALID_ARG, "scene is null");
  s->timing = enabled != 0;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_stage_times(zsmpm_scene *s, float *ms, int32_t count) {
  if (!s || !ms) return fail(ZSMPM_ERR_INVALID_ARG, "null argument");
  for (int k = 0; k < count && k < 5; ++k) ms[k] = s->stage_ms[k];
  return ZSMPM_OK;
}

ZSMPM_API int32_t zsmpm_kernels_per_substep(const zsmpm_scene *) { return kernels_per_substep(); }

ZSMPM_API zsmpm_status zsmpm_scene_set_closure(zsmpm_scene *s, zsmpm_closure *c, int32_t audit_period) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (audit_period < 0) return fail(ZSMPM_ERR_INVALID_ARG, "audit_period < 0");
  if (!c) {
    invalidate_graphs(s);
    s->dev.aux.learned = 0;
    return ZSMPM_OK;
  }
  if (s->dev.prm.transfer != kTransferApic)
    return fail(ZSMPM_ERR_INVALID_ARG, "the learned closure replaces G2P's return map (APIC transfers only)");
  closure_dev cd{};
  if (!closure_device_view(c, &cd)) return fail(ZSMPM_ERR_NOT_READY, "closure has no dataset or state yet");
  // a batch runs the closure on the scenes of its model and the plain return map on the others
  if (s->nscenes == 0 && cd.model != s->desc.material.model)
    return fail(ZSMPM_ERR_INVALID_ARG, "closure was built for another material model");
  if (s->desc.material.plasticity_mode != ZSMPM_PLASTICITY_COMMITTED && s->desc.material.model != ZSMPM_SNOW)
    return fail(ZSMPM_ERR_INVALID_ARG, "the learned closure runs in the committed plasticity ordering");
  ZS_TRY(prepare_closure_kernels(), "closure kernel attributes");
  if (!s->audit) {
    double *a = nullptr;
    ZS_TRY(cudaMalloc(&a, sizeof(double) * 8), "alloc audit");
    s->allocations.push_back(a);
    s->audit = a;
    ZS_TRY(cudaMemset(s->audit, 0, sizeof(double) * 8), "memset audit");
  }
  // the queue of projections for the network: one entry per particle of the capacity
  if (s->uploaded && s->dev.aux.qcap < s->dev.prm.cap) {
    const long long q = s->dev.prm.cap;
    float *feat = nullptr, *outr = nullptr, *uvs = nullptr;
    int2 *slots = nullptr;
    int *ids = nullptr;
    ZS_ALLOC(feat, 6 * q, "alloc closure queue");
    ZS_ALLOC(outr, 6 * q, "alloc closure queue");
    ZS_ALLOC(uvs, (size_t)kQueueFloats * q, "alloc closure queue");
    ZS_ALLOC(slots, q, "alloc closure queue");
    ZS_ALLOC(ids, q, "alloc closure queue");
    s->dev.aux.q_feat = feat;
    s->dev.aux.q_out = outr;
    s->dev.aux.q_uvs = uvs;
    s->dev.aux.q_slot = slots;
    s->dev.aux.q_id = ids;
    s->dev.aux.qcap = q;
  }
  if (s->dev.aux.qcap < 1) return fail(ZSMPM_ERR_NOT_READY, "attach the closure after the particles are uploaded");
  invalidate_graphs(s);
  cd.audit = s->audit;
  cd.audit_period = audit_period;
  s->dev.aux.cd = cd;
  s->dev.aux.learned = 1;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_scene_closure_audit(zsmpm_scene *s, zsmpm_closure_audit *out, int32_t reset) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (!out) return fail(ZSMPM_ERR_INVALID_ARG, "null output");
  std::memset(out, 0, sizeof(*out));
  if (!s->audit) return ZSMPM_OK;
  if (s->last_stream) ZS_TRY(cudaStreamSynchronize(s->last_stream), "synchronize");
  ZS_TRY(cudaDeviceSynchronize(), "synchronize");
  double h[8];
  ZS_TRY(cudaMemcpy(h, s->audit, sizeof(h), cudaMemcpyDeviceToHost), "read audit");
  out->audited = (int64_t)h[0];
  out->mean_rel_error = h[0] > 0 ? h[1] / h[0] : 0.0;
  out->max_rel_error = h[2];
  out->agg_rel_error = h[4] > 0 ? std::sqrt(h[3] / h[4]) : 0.0;
  out->fallbacks = (int64_t)h[5];
  out->network_updates = (int64_t)h[6];
  out->updates = (int64_t)h[7];
  if (reset) ZS_TRY(cudaMemset(s->audit, 0, sizeof(h)), "reset audit");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_scene_set_state_log(zsmpm_scene *s, float *buffer, int64_t cap, int32_t period) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (period < 0 || (period > 0 && (!buffer || cap < 1))) return fail(ZSMPM_ERR_INVALID_ARG, "bad log arguments");
  if (period > 0 && s->nscenes > 0) return fail(ZSMPM_ERR_INVALID_ARG, "the state log runs on single scenes");
  if (!s->log_count) {
    unsigned long long *c = nullptr;
    ZS_TRY(cudaMalloc(&c, sizeof(unsigned long long)), "alloc log counter");
    s->allocations.push_back(c);
    s->log_count = c;
  }
  invalidate_graphs(s);
  ZS_TRY(cudaMemset(s->log_count, 0, sizeof(unsigned long long)), "reset log counter");
  s->dev.aux.log_buf = period > 0 ? buffer : nullptr;
  s->dev.aux.log_cap = period > 0 ? cap : 0;
  s->dev.aux.log_period = period;
  s->dev.aux.log_count = s->log_count;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_scene_state_log_count(zsmpm_scene *s, int64_t *count_out) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (!count_out) return fail(ZSMPM_ERR_INVALID_ARG, "null output");
  *count_out = 0;
  if (!s->log_count) return ZSMPM_OK;
  if (s->last_stream) ZS_TRY(cudaStreamSynchronize(s->last_stream), "synchronize");
  ZS_TRY(cudaDeviceSynchronize(), "synchronize");
  unsigned long long c = 0;
  ZS_TRY(cudaMemcpy(&c, s->log_count, sizeof(c), cudaMemcpyDeviceToHost), "read log counter");
  *count_out = (int64_t)std::min<unsigned long long>(c, (unsigned long long)std::max<int64_t>(s->dev.aux.log_cap, 0));
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_get_bht_view(zsmpm_scene *s, zsmpm_bht_view *out) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (!out) return fail(ZSMPM_ERR_INVALID_ARG, "null output");
  if (s->last_stream) ZS_TRY(cudaStreamSynchronize(s->last_stream), "synchronize");
  ZS_TRY(cudaDeviceSynchronize(), "synchronize");
  int nb = 0;
  ZS_TRY(cudaMemcpy(&nb, &s->dev.ctr[kCtrBlocks], sizeof(int), cudaMemcpyDeviceToHost), "read block count");
  std::vector<int32_t> keys(3 * (size_t)std::max(nb, 1));
  if (nb > 0)
    ZS_TRY(cudaMemcpy(keys.data(), s->dev.active_keys, sizeof(int32_t) * 3 * nb, cudaMemcpyDeviceToHost),
           "read active keys");
  // sized for max(nb, 16) entries: below that the reference's proximity rule (an index at or
  // above size - 20 fails) rejects even a single key
  const int64_t size = bht_table_size(std::max(nb, 16));
  if (nb > 0 && (int64_t)nb - 1 >= size - 20) return fail(ZSMPM_ERR_TABLE_FULL, "bht table too small for the keys");
  if (size > s->bht_cap) {
    release_bht(s);
    ZS_TRY(cudaMalloc(&s->bht_keys, sizeof(int32_t) * 4 * (size_t)size), "alloc bht keys");
    ZS_TRY(cudaMalloc(&s->bht_indices, sizeof(int32_t) * (size_t)size), "alloc bht indices");
    ZS_TRY(cudaMalloc(&s->bht_status, sizeof(int32_t) * (size_t)size), "alloc bht status");
    ZS_TRY(cudaMalloc(&s->bht_active, sizeof(int32_t) * 3 * (size_t)size), "alloc bht active keys");
    ZS_TRY(cudaMalloc(&s->bht_cnt, sizeof(int32_t) * 2), "alloc bht count");
    s->bht_cap = size;
  }
  // built on the device from the active keys in canonical order (zsmpm_bht.cu)
  uint32_t hash[6] = {};
  const int built = bht_build_device(s->dev.active_keys, nb, size, s->bht_keys, s->bht_indices, s->bht_status,
                                     s->bht_active, s->bht_cnt, hash, s->last_stream);
  if (built != ZSMPM_OK) return (zsmpm_status)built;
  out->keys = s->bht_keys;
  out->indices = s->bht_indices;
  out->status = s->bht_status;
  out->active_keys = s->bht_active;
  out->cnt = s->bht_cnt;
  out->success = s->bht_cnt + 1;
  out->table_size = (int32_t)size;
  for (int k = 0; k < 6; ++k) out->hashers[k] = hash[k];
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_batch_create(const zsmpm_scene_desc *desc, const zsmpm_material *materials,
                                          int32_t nscenes, zsmpm_scene **out) {
  if (!desc || !materials || !out) return fail(ZSMPM_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (nscenes < 1 || nscenes > kBatchMaxScenes) return fail(ZSMPM_ERR_INVALID_ARG, "nscenes out of range");
  if (!(desc->dx > 0.f) || 1.f / desc->dx > 8.f * (kBatchSlot - kBatchMargin - 2))
    return fail(ZSMPM_ERR_INVALID_ARG, "batched scenes need 1/dx <= 176 (a scene's [0,1]^3 fits its key slot)");
  bool plastic = false;
  for (int k = 0; k < nscenes; ++k) {
    const zsmpm_material &m = materials[k];
    if (m.model < 0 || m.model > 2) return fail(ZSMPM_ERR_INVALID_ARG, "unknown material model in batch");
    if (m.model == ZSMPM_DRUCKER_PRAGER && m.plasticity_mode != ZSMPM_PLASTICITY_COMMITTED)
      return fail(ZSMPM_ERR_INVALID_ARG, "batched scenes run the committed plasticity ordering");
    plastic = plastic || m.model != ZSMPM_FIXED_COROTATED;
  }
  zsmpm_scene_desc d = *desc;
  d.material = materials[0];
  zsmpm_scene *s = nullptr;
  zsmpm_status st = zsmpm_scene_create(&d, &s);
  if (st != ZSMPM_OK) return st;
  s->nscenes = nscenes;
  s->any_plastic = plastic;
  std::vector<material_dev> mats(nscenes);
  for (int k = 0; k < nscenes; ++k) mats[k] = make_material(materials[k]);
  material_dev *dm = nullptr;
  int *ds = nullptr;
  cudaError_t e = cudaMalloc(&dm, sizeof(material_dev) * nscenes);
  if (e == cudaSuccess) s->allocations.push_back(dm);
  if (e == cudaSuccess) e = cudaMalloc(&ds, sizeof(int) * (nscenes + 1));
  if (e == cudaSuccess) s->allocations.push_back(ds);
  if (e == cudaSuccess) e = cudaMemcpy(dm, mats.data(), sizeof(material_dev) * nscenes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    zsmpm_scene_destroy(s);
    return cuda_fail(e, "batch materials");
  }
  s->dev.prm.batch = 1;
  s->dev.prm.nscenes = nscenes;
  s->dev.prm.mats = dm;
  s->dev.prm.scene_start = ds;
  *out = s;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_batch_upload(zsmpm_scene *s, const zsmpm_particle_arrays *p, const int64_t *counts,
                                          int32_t on_device, void *stream) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (s->nscenes < 1) return fail(ZSMPM_ERR_INVALID_ARG, "not a batch (zsmpm_batch_create)");
  if (!counts) return fail(ZSMPM_ERR_INVALID_ARG, "null counts");
  std::vector<int> start(s->nscenes + 1, 0);
  int64_t n = 0;
  for (int k = 0; k < s->nscenes; ++k) {
    if (counts[k] < 0) return fail(ZSMPM_ERR_INVALID_ARG, "negative scene particle count");
    n += counts[k];
    if (n > (int64_t)0x7fffffff) return fail(ZSMPM_ERR_INVALID_ARG, "particle count out of range");
    start[k + 1] = (int)n;
  }
  ZS_TRY(cudaMemcpy(const_cast<int *>(s->dev.prm.scene_start), start.data(), sizeof(int) * start.size(),
                    cudaMemcpyHostToDevice),
         "scene starts");
  s->counts.assign(counts, counts + s->nscenes);
  return upload_arrays(s, p, n, on_device, stream);
}

ZSMPM_API zsmpm_status zsmpm_batch_num_scenes(const zsmpm_scene *s, int32_t *out) {
  if (!s || !out) return fail(ZSMPM_ERR_INVALID_ARG, "null argument");
  *out = s->nscenes;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_autotune(zsmpm_scene *s, int32_t trials, zsmpm_tuning *out, void *stream) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (trials < 1) return fail(ZSMPM_ERR_INVALID_ARG, "trials < 1");
  cudaStream_t cs = as_stream(stream);
  scene_params &p = s->dev.prm;
  const bool was_timing = s->timing;
  s->timing = true;
  invalidate_graphs(s);
  // time one stage under a launch shape: one untimed substep, then `trials` timed ones
  auto time_stage = [&](int stage, float *ms) -> zsmpm_status {
    float total = 0.f;
    for (int r = 0; r <= trials; ++r) {
      zsmpm_status q = substep_enqueue(s, cs);
      if (q != ZSMPM_OK) return q;
      ZS_TRY(cudaStreamSynchronize(cs), "tune sync");
      float t = 0.f;
      ZS_TRY(cudaEventElapsedTime(&t, s->ev[stage], s->ev[stage + 1]), "tune timing");
      if (r > 0) total += t;
    }
    *ms = total / trials;
    return read_status(s);
  };
  zsmpm_tuning best{};
  // G2P: CTA size x CTAs per SM (each CTA owns one block at a time)
  float best_g2p = 3.4e38f;
  const int g2p_threads[2] = {256, 128};
  const int g2p_per_sm[6] = {1, 2, 3, 4, 5, 6};
  for (int a : g2p_threads)
    for (int b : g2p_per_sm) {
      if (s->dev.aux.learned && a != 256) continue;  // the learned G2P runs 256-thread CTAs
      // beyond what stays resident: 256 threads hold 80 registers and 58 KB of shared memory
      // (3 CTAs per SM), 128 threads 43 KB (5)
      if ((a == 256 && b > 3) || (a == 128 && b > 5)) continue;
      p.g2p_threads = a;
      p.g2p_ctas_per_sm = b;
      float ms = 0.f;
      st = time_stage(4, &ms);
      if (st != ZSMPM_OK) break;
      if (ms < best_g2p) {
        best_g2p = ms;
        best.g2p_threads = a;
        best.g2p_ctas_per_sm = b;
      }
    }
  // P2G: staging depth x CTAs per SM, up to what the depth's shared memory lets stay resident
  // (8 ranks: 55 KB, 4 CTAs; 12: 72 KB, 3; 16: 88 KB, 2)
  float best_p2g = 3.4e38f;
  const int p2g_shapes[6][2] = {{12, 3}, {12, 2}, {8, 4}, {8, 3}, {16, 2}, {16, 1}};
  if (st == ZSMPM_OK)
    for (const auto &shape : p2g_shapes) {
      p.p2g_ranks = shape[0];
      p.p2g_ctas_per_sm = shape[1];
      float ms = 0.f;
      st = time_stage(2, &ms);
      if (st != ZSMPM_OK) break;
      if (ms < best_p2g) {
        best_p2g = ms;
        best.p2g_ranks = shape[0];
        best.p2g_ctas_per_sm = shape[1];
      }
    }
  s->timing = was_timing;
  if (st != ZSMPM_OK) return st;
  p.g2p_threads = best.g2p_threads;
  p.g2p_ctas_per_sm = best.g2p_ctas_per_sm;
  p.p2g_ctas_per_sm = best.p2g_ctas_per_sm;
  p.p2g_ranks = best.p2g_ranks;
  best.g2p_ms = best_g2p;
  best.p2g_ms = best_p2g;
  invalidate_graphs(s);
  s->last_stream = cs;
  if (out) *out = best;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_set_tuning(zsmpm_scene *s, const zsmpm_tuning *t) {
  zsmpm_status st = check_scene(s, false);
  if (st != ZSMPM_OK) return st;
  if (!t) return fail(ZSMPM_ERR_INVALID_ARG, "null tuning");
  if ((t->g2p_threads != 0 && t->g2p_threads != 128 && t->g2p_threads != 256) || t->g2p_ctas_per_sm < 0 ||
      t->g2p_ctas_per_sm > 6 || t->p2g_ctas_per_sm < 0 || t->p2g_ctas_per_sm > 4 ||
      (t->p2g_ranks != 0 && t->p2g_ranks != 8 && t->p2g_ranks != 12 && t->p2g_ranks != 16))
    return fail(ZSMPM_ERR_INVALID_ARG, "tuning out of range");
  // more CTAs than the staging depth's shared memory lets stay resident would queue, not run
  const int ranks = t->p2g_ranks ? t->p2g_ranks : 12;
  const int max_p2g = ranks == 8 ? 4 : ranks == 12 ? 3 : 2;
  if (t->p2g_ctas_per_sm > max_p2g)
    return fail(ZSMPM_ERR_INVALID_ARG, "p2g_ctas_per_sm beyond what the staging depth's shared memory allows");
  if (s->dev.aux.learned && t->g2p_threads == 128)
    return fail(ZSMPM_ERR_INVALID_ARG, "the learned G2P runs 256-thread CTAs");
  s->dev.prm.g2p_threads = t->g2p_threads;
  s->dev.prm.g2p_ctas_per_sm = t->g2p_ctas_per_sm;
  s->dev.prm.p2g_ctas_per_sm = t->p2g_ctas_per_sm;
  s->dev.prm.p2g_ranks = t->p2g_ranks;
  invalidate_graphs(s);
  return ZSMPM_OK;
}

// ---- the implicit system (ImplicitMPM.hpp)
namespace {

zsmpm_status check_implicit(zsmpm_scene *s, std::initializer_list<const void *> vecs, int64_t ndofs) {
  zsmpm_status st = check_scene(s, true);
  if (st != ZSMPM_OK) return st;
  if (s->nscenes > 0) return fail(ZSMPM_ERR_INVALID_ARG, "the implicit system runs on single scenes");
  if (!s->binned) return fail(ZSMPM_ERR_NOT_READY, "needs zsmpm_activate_blocks and zsmpm_bin_particles first");
  if (ndofs < 0) return fail(ZSMPM_ERR_INVALID_ARG, "ndofs < 0");
  for (const void *v : vecs) {
    if (!v) return fail(ZSMPM_ERR_INVALID_ARG, "null dof vector");
    if (reinterpret_cast<uintptr_t>(v) % 16 != 0) return fail(ZSMPM_ERR_INVALID_ARG, "dof vectors must be 16-byte aligned");
  }
  bind_buffers(s);
  return ZSMPM_OK;
}

}  // namespace

ZSMPM_API zsmpm_status zsmpm_g2p2g(zsmpm_scene *s, const float *v, float *f, int64_t ndofs, float dt, void *stream) {
  zsmpm_status st = check_implicit(s, {v, f}, ndofs);
  if (st != ZSMPM_OK) return st;
  if (!std::isfinite(dt)) return fail(ZSMPM_ERR_INVALID_ARG, "dt must be finite");
  ZS_TRY(launch_g2p2g(s->dev, v, f, ndofs, dt, nullptr, as_stream(stream)), "g2p2g");
  s->last_stream = as_stream(stream);
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_implicit_multiply(zsmpm_scene *s, const float *in, float *out, int64_t ndofs, float dt,
                                               void *stream) {
  zsmpm_status st = check_implicit(s, {in, out}, ndofs);
  if (st != ZSMPM_OK) return st;
  if (!std::isfinite(dt)) return fail(ZSMPM_ERR_INVALID_ARG, "dt must be finite");
  if (in == out) return fail(ZSMPM_ERR_INVALID_ARG, "multiply needs distinct in and out vectors");
  cudaStream_t cs = as_stream(stream);
  ZS_TRY(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)ndofs, cs), "multiply: zero");
  ZS_TRY(launch_g2p2g(s->dev, in, out, ndofs, dt, nullptr, cs), "multiply: g2p2g");
  ZS_TRY(launch_implicit_mass(s->dev, in, out, dt, ndofs, nullptr, cs), "multiply: mass");
  s->last_stream = cs;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_implicit_project(zsmpm_scene *s, float *inout, int64_t ndofs, void *stream) {
  zsmpm_status st = check_implicit(s, {inout}, ndofs);
  if (st != ZSMPM_OK) return st;
  ZS_TRY(launch_implicit_project(s->dev, inout, ndofs, nullptr, as_stream(stream)), "project");
  s->last_stream = as_stream(stream);
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_implicit_precondition(zsmpm_scene *s, const float *in, float *out, int64_t ndofs,
                                                   void *stream) {
  zsmpm_status st = check_implicit(s, {in, out}, ndofs);
  if (st != ZSMPM_OK) return st;
  ZS_TRY(launch_implicit_precondition(s->dev, in, out, ndofs, nullptr, as_stream(stream)), "precondition");
  s->last_stream = as_stream(stream);
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_implicit_cg(zsmpm_scene *s, float *x, const float *b, int64_t ndofs, float dt,
                                         const zsmpm_cg_options *opts, int32_t *iters_out, void *stream) {
  zsmpm_status st = check_implicit(s, {x, b}, ndofs);
  if (st != ZSMPM_OK) return st;
  if (!std::isfinite(dt)) return fail(ZSMPM_ERR_INVALID_ARG, "dt must be finite");
  zsmpm_cg_options o{1000, 1e-6f, 0.5f};
  if (opts) o = *opts;
  if (o.max_iters < 0) return fail(ZSMPM_ERR_INVALID_ARG, "max_iters < 0");
  cudaStream_t cs = as_stream(stream);
  if (!s->cg) ZS_ALLOC(s->cg, 1, "cg state");
  // vectors start on 16-byte boundaries (cudaMalloc returns 256-byte aligned memory)
  const int64_t stride = (ndofs + 3) / 4 * 4;
  if (stride > s->cg_cap) {
    ZS_TRY(cudaStreamSynchronize(cs), "cg scratch");
    if (s->cg_buf) {
      s->allocations.erase(std::remove(s->allocations.begin(), s->allocations.end(), (void *)s->cg_buf),
                           s->allocations.end());
      cudaFree(s->cg_buf);
      s->cg_buf = nullptr;
      s->cg_cap = 0;
    }
    ZS_ALLOC(s->cg_buf, 4 * (size_t)stride, "cg scratch");
    s->cg_cap = stride;
  }
  const cg_vectors v{s->cg_buf, s->cg_buf + stride, s->cg_buf + 2 * stride, s->cg_buf + 3 * stride};
  ZS_TRY(launch_cg_begin(s->dev, x, b, v, ndofs, dt, s->cg, o.tol, o.rel_tol, cs), "cg begin");
  constexpr int kChunk = 8;
  cg_state h{};
  for (int it = 0; it < o.max_iters + 1; it += kChunk) {
    for (int k = 0; k < kChunk; ++k) ZS_TRY(launch_cg_iteration(s->dev, x, v, ndofs, dt, s->cg, o.max_iters, cs), "cg iteration");
    ZS_TRY(cudaMemcpyAsync(&h, s->cg, sizeof(cg_state), cudaMemcpyDeviceToHost, cs), "cg state");
    ZS_TRY(cudaStreamSynchronize(cs), "cg iteration");
    if (h.done) break;
  }
  s->last_stream = cs;
  if (iters_out) *iters_out = h.iter;
  return read_status(s);
}

ZSMPM_API zsmpm_status zsmpm_svd3(const float *A, float *U, float *S, float *V, int64_t count, void *stream) {
  if (count < 0 || (count > 0 && (!A || !U || !S || !V))) return fail(ZSMPM_ERR_INVALID_ARG, "bad svd arguments");
  if (count == 0) return ZSMPM_OK;
  ZS_TRY(launch_svd_batch(A, U, S, V, count, as_stream(stream)), "svd");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_constitutive(const zsmpm_material *mat, float *F, float *plastic, float *tau,
                                          int64_t count, void *stream) {
  if (!mat || count < 0 || (count > 0 && (!F || !tau))) return fail(ZSMPM_ERR_INVALID_ARG, "bad arguments");
  if (mat->model != ZSMPM_FIXED_COROTATED && count > 0 && !plastic)
    return fail(ZSMPM_ERR_INVALID_ARG, "plastic state required for this model");
  if (count == 0) return ZSMPM_OK;
  ZS_TRY(launch_constitutive_batch(make_material(*mat), F, plastic, tau, count, as_stream(stream)),
         "constitutive");
  return ZSMPM_OK;
}

}  // extern "C"
