// Test infrastructure: drives the REFERENCE's own MPM operators (zpc, compiled from its
// sources by oracle/build_ref.sh) through its own seq/omp execution policies.  The entry
// points below are called by oracle/ref_cli.cpp, which the Python tests and the CPU
// baseline arm of the benchmark run as a subprocess.  Nothing here is linked into the
// product library.
//
// One substep is the canonical explicit MLS/APIC substep that the reference's operators
// compose into (the reference ships the operators but no driver):
//   1. CleanSparsity + ComputeSparsity + EnlargeSparsity{0..2}^3
//        (simulation/sparsity/SparsityOp.hpp:41-112, driver SparsityCompute.tpp:5-26)
//   2. optional canonical re-ordering of the active keys (ascending (bx,by,bz)) followed by
//      ResetHashTable + ReinsertHashTable (container/HashTable.hpp:215-247), which assigns
//      index == position in the sorted key list
//   3. CleanGridBlocks + P2GTransfer (simulation/grid/GridOp.hpp:54-69,
//      simulation/transfer/P2G.hpp:45-127)
//   4. grid velocity v = (mv + rhs)/m + g dt.  The reference's ComputeGridBlockVelocity
//      (GridOp.hpp:93-99) computes mv/m + g dt and never consumes the rhs channel that P2G
//      fills (P2G.hpp:120-123), so the rhs term is restated here in GridVelocityWithRhs.
//   5. ApplyBoundaryConditionOnGridBlocks with six analytic planes (GridOp.hpp:113-164,
//      geometry/Collider.h:80-110, geometry/AnalyticLevelSet.h:11-43)
//   6. G2PTransfer (simulation/transfer/G2P.hpp:43-84)
// zsref_run_cell composes the cell-centric transfer pair instead of P2G / G2P (below).
// zsref_g2p2g drives the implicit-force operator G2P2GTransfer
// (simulation/transfer/G2P2G.hpp:49-142) over a caller-given grid velocity field, and
// zsref_implicit the implicit system's operators and its conjugate-gradient solve
// (simulation/mpm/ImplicitMPM.hpp:13-159, math/linear/ConjugateGradient.hpp:69-172).
// Stress and plasticity are evaluated inside P2G on a local copy of F exactly as the
// reference does ("ref-verbatim"): the projected F is not written back, logJp is.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <vector>

#include "zensim/omp/execution/ExecutionPolicy.hpp"
#include "zensim/simulation/sparsity/SparsityOp.hpp"
#include "zensim/simulation/transfer/P2G.hpp"
#include "zensim/simulation/transfer/G2P.hpp"
#include "zensim/simulation/transfer/G2P2G.hpp"
#include "zensim/simulation/transfer/P2C2G.hpp"
#include "zensim/simulation/transfer/G2C2P.hpp"
#include "zensim/container/IndexBuckets.hpp"
#include "zensim/simulation/mpm/ImplicitMPM.hpp"
#include "zensim/math/linear/ConjugateGradient.hpp"
#include "zensim/geometry/SparseLevelSet.hpp"
#include "zensim/simulation/grid/GridOp.hpp"
#include "zensim/geometry/AnalyticLevelSet.h"
#include "zensim/geometry/Collider.h"
#include "zensim/container/Bht.hpp"
#include "zensim/types/View.h"

namespace {

  using namespace zs;
  using table_t = HashTable<i32, 3, int>;
  using grids_t = Grids<f32, 3, 8>;
  using particles_t = Particles<f32, 3>;

  // Restated grid update: v = (mv + rhs) * (1/m) + g dt on cells with m != 0.
  template <execspace_e space> struct GridVelocityWithRhs {
    using view_t = GridsView<space, grids_t>;
    GridVelocityWithRhs(wrapv<space>, grids_t &g, float dt, vec<float, 3> grav)
        : grids{proxy<space>(g)}, dt{dt}, grav{grav} {}
    void operator()(typename grids_t::size_type blockid,
                    typename grids_t::cell_index_type cellid) noexcept {
      auto block = grids[blockid];
      float mass = block(0, cellid);
      if (mass != 0.f) {
        mass = 1.f / mass;
        vec<float, 3> vel{};
        for (int d = 0; d != 3; ++d)
          vel[d] = (block(1 + d, cellid) + block(4 + d, cellid)) * mass + grav[d] * dt;
        for (int d = 0; d != 3; ++d) block(1 + d, cellid) = vel[d];
      }
    }
    view_t grids;
    float dt;
    vec<float, 3> grav;
  };

  using plane_t = AnalyticLevelSet<analytic_geometry_e::Plane, float, 3>;

  // zsmpm_collider's layout: shape 0 plane, 1 cuboid, 2 sphere, 3 cylinder; type 0 sticky,
  // 1 slip, 2 separate; rot row-major
  struct ref_collider {
    int shape, type, axis, reserved;
    float a[3], b[3];
    float s, dsdt;
    float rot[9];
    float omega[3], t[3], dtdt[3];
  };

  // A SparseLevelSet<3> boundary: block origins (index space, multiples of 8), 512 "sdf" values
  // per block in cell order x*64 + y*8 + z, the background value and the world-to-index
  // transform X = ((x - t) Rinv) Sinv (row-vector products, matrices row-major).
  struct ref_levelset {
    int nblocks, type;
    float background, sinv[9], rinv[9], t[3];
    const int *keys;
    const float *sdf;
  };

  // One ApplyBoundaryConditionOnGridBlocks launch with LevelSetBoundary<SparseLevelSet<3>>
  // (Collider.h:204-236, GridOp.hpp:32-36, :126-134): the level set is built by the reference's
  // own bht insert and grid storage, then sampled through its SparseLevelSetView.
  template <class Pol, execspace_e space, class Table, class Grids>
  void apply_levelset(Pol &pol, wrapv<space>, const ref_levelset &L, Table &table, Grids &grids, int nb) {
    SparseLevelSet<3> ls{{{"sdf", 1}}, 1.f, (size_t)std::max(L.nblocks, 1), memsrc_e::host, -1};
    {
      auto tv = view<execspace_e::host>(ls._table);
      for (int b = 0; b != L.nblocks; ++b)
        tv.insert(vec<int, 3>{L.keys[3 * b], L.keys[3 * b + 1], L.keys[3 * b + 2]});
      auto gv = proxy<execspace_e::host>({}, ls._grid);
      for (int b = 0; b != L.nblocks; ++b) {
        const auto bno = tv.query(vec<int, 3>{L.keys[3 * b], L.keys[3 * b + 1], L.keys[3 * b + 2]});
        for (int c = 0; c != 512; ++c) gv(0, (size_t)bno, c) = L.sdf[(size_t)b * 512 + c];
      }
    }
    for (int i = 0; i != 3; ++i) {
      ls._i2wT[i] = L.t[i];
      for (int j = 0; j != 3; ++j) {
        ls._i2wSinv(i, j) = L.sinv[3 * i + j];
        ls._i2wRinv(i, j) = L.rinv[3 * i + j];
      }
    }
    ls._backgroundValue = L.background;
    LevelSetBoundary<SparseLevelSet<3>> boundary{ls, L.type == 0   ? collider_e::Sticky
                                                     : L.type == 1 ? collider_e::Slip
                                                                   : collider_e::Separate};
    pol(Collapse{(size_t)nb, (size_t)512},
        ApplyBoundaryConditionOnGridBlocks{wrapv<space>{}, boundary, table, grids});
  }

  // One ApplyBoundaryConditionOnGridBlocks launch (GridOp.hpp:113-158) with a
  // Collider<AnalyticLevelSet<shape, f32, 3>> (Collider.h:10-200) placed as described.
  template <class Pol, execspace_e space, class Table, class Grids>
  void apply_collider(Pol &pol, wrapv<space>, const ref_collider &c, Table &table, Grids &grids, int nb) {
    auto go = [&](auto ls) {
      Collider col{ls, c.type == 0 ? collider_e::Sticky : c.type == 1 ? collider_e::Slip : collider_e::Separate};
      col.s = c.s;
      col.dsdt = c.dsdt;
      for (int i = 0; i != 3; ++i)
        for (int j = 0; j != 3; ++j) col.R(i, j) = c.rot[3 * i + j];
      col.omega.omega = vec<float, 3>{c.omega[0], c.omega[1], c.omega[2]};
      col.b = vec<float, 3>{c.t[0], c.t[1], c.t[2]};
      col.dbdt = vec<float, 3>{c.dtdt[0], c.dtdt[1], c.dtdt[2]};
      pol(Collapse{(size_t)nb, (size_t)512}, ApplyBoundaryConditionOnGridBlocks{wrapv<space>{}, col, table, grids});
    };
    const vec<float, 3> a{c.a[0], c.a[1], c.a[2]}, b{c.b[0], c.b[1], c.b[2]};
    if (c.shape == 0)
      go(AnalyticLevelSet<analytic_geometry_e::Plane, float, 3>{a, b});
    else if (c.shape == 1)
      go(AnalyticLevelSet<analytic_geometry_e::Cuboid, float, 3>{a, b});
    else if (c.shape == 2)
      go(AnalyticLevelSet<analytic_geometry_e::Sphere, float, 3>{a, c.b[0]});
    else
      go(AnalyticLevelSet<analytic_geometry_e::Cylinder, float, 3>{a, c.b[0], c.b[1], c.axis});
  }

  // Block activation of zsref_run (ComputeSparsity + EnlargeSparsity, then the canonical key
  // order and ReinsertHashTable) on the given positions; returns the block count or -1 when the
  // table is full.
  template <class Pol, execspace_e space>
  int activate_canonical(Pol &pol, wrapv<space>, table_t &table, particles_t &pars, float dx) {
    pol(range(table._tableSize), CleanSparsity{wrapv<space>{}, table});
    pol(range(pars.size()), ComputeSparsity{wrapv<space>{}, dx, 8, table, pars.attrVector("x")});
    const int npb = table.size();
    pol(range((size_t)npb),
        EnlargeSparsity{wrapv<space>{}, table, vec<int, 3>{0, 0, 0}, vec<int, 3>{2, 2, 2}});
    const int nb = table.size();
    if (nb >= table._tableSize - 20) return -1;
    auto *keys = table._activeKeys.data();
    std::sort(keys, keys + nb, [](const auto &a, const auto &b) {
      for (int d = 0; d != 3; ++d)
        if (a[d] != b[d]) return a[d] < b[d];
      return false;
    });
    pol(range(table._tableSize), ResetHashTable{proxy<space>(table), false});
    pol(range((size_t)nb), ReinsertHashTable{proxy<space>(table)});
    return nb;
  }


  // ImplicitMPMSystem's multiply / project / precondition (ImplicitMPM.hpp:34-153) for one
  // model, one partition, one particle set and the six walls: the same bodies with the
  // simulator's loops over model groups and boundaries reduced to their single entries, calling
  // the reference's own functors (DofFill, G2P2GTransfer, ForceDtSqrPlusMass, Projector,
  // DivPernodeMass).
  template <class Model> struct RefImplicitSystem {
    Model model;
    table_t &table;
    particles_t &pars;
    grids_t &grids;
    std::vector<Collider<plane_t>> &walls;
    float dt;

    template <class Pol, typename In, typename Out> void multiply(Pol &&policy, In &&in, Out &&out) {
      constexpr execspace_e space = RM_REF_T(policy)::exec_tag::value;
      policy(range(out.numEntries()), DofFill{out, 0});
      policy(range(pars.size()),
             G2P2GTransfer{wrapv<space>{}, wrapv<transfer_scheme_e::apic>{}, dt, model,
                           proxy<space>(grids.grid()), in, out, table, pars});
      auto gridm = dof_view<space, 1>(grids.grid(), "m", 0);
      policy(range(in.numEntries()), ImplicitMPMSystem::ForceDtSqrPlusMass{out, gridm, out, in, dt});
    }
    template <class Pol, typename InOut> void project(Pol &&policy, InOut &&inout) {
      constexpr execspace_e space = RM_REF_T(policy)::exec_tag::value;
      for (auto &w : walls)
        policy(range((size_t)inout.numEntries() / 3),
               ImplicitMPMSystem::Projector{w, proxy<space>(table), proxy<space>(grids.grid()), inout});
    }
    template <class Pol, typename In, typename Out> void precondition(Pol &&policy, In &&in, Out &&out) {
      constexpr execspace_e space = RM_REF_T(policy)::exec_tag::value;
      auto gridm = dof_view<space, 1>(grids.grid(), "m", 0);
      policy(range(out.numEntries()), ImplicitMPMSystem::DivPernodeMass{in, gridm, out});
    }
  };

}  // namespace

extern "C" {

struct zsref_params {
  int model;          // 0 fixed-corotated, 1 Drucker-Prager sand
  int policy;         // 0 seq_exec, 1 omp_exec
  int threads;        // omp threads; <= 0 selects zpc's default (hardware_concurrency - 1)
  int order;          // 0 keep the table's insertion order, 1 canonical ascending (bx,by,bz)
  int wall_type;      // 0 sticky, 1 slip, 2 separate
  int wall_cells;     // wall thickness in cells (planes at wall_cells*dx from each face)
  int table_expected; // expected entry count given to HashTable (capacity next_2pow(n)*16)
  int volume_correction;
  float dx, dt, gx, gy, gz;
  float E, nu, volume;
  float friction_deg, cohesion, beta;
};

// Runs nsteps substeps in place on SoA host arrays (x,v: n*3; C,F: n*9 column-major).
// Grid output (optional, out_keys may be NULL): active block keys (i32*3 each) in table
// index order and per block 512 cells x 4 channels (m, vx, vy, vz) after the boundary
// conditions of the last substep, channel-major inside a block.
// Returns 0 on success, 1 if the grid output capacity is too small, 2 if the table is full.
int zsref_run_colliders(const zsref_params *p, int n, float *m, float *x, float *v, float *C, float *F,
                        float *logJp, int nsteps, int cap_blocks, int *out_nblocks, int *out_keys,
                        float *out_grid, double *out_seconds, int ncolliders, const void *colliders,
                        int nlevelsets = 0, const void *levelsets = nullptr);

int zsref_run(const zsref_params *p, int n, float *m, float *x, float *v, float *C, float *F,
              float *logJp, int nsteps, int cap_blocks, int *out_nblocks, int *out_keys,
              float *out_grid, double *out_seconds) {
  return zsref_run_colliders(p, n, m, x, v, C, F, logJp, nsteps, cap_blocks, out_nblocks, out_keys, out_grid,
                             out_seconds, 0, nullptr);
}

// zsref_run with `ncolliders` colliders (ref_collider records) and then `nlevelsets` sparse
// level-set boundaries (ref_levelset records) applied after the walls, each by its own
// ApplyBoundaryConditionOnGridBlocks launch.
int zsref_run_colliders(const zsref_params *p, int n, float *m, float *x, float *v, float *C, float *F,
                        float *logJp, int nsteps, int cap_blocks, int *out_nblocks, int *out_keys,
                        float *out_grid, double *out_seconds, int ncolliders, const void *colliders,
                        int nlevelsets, const void *levelsets) {
  const ref_collider *cols = static_cast<const ref_collider *>(colliders);
  const ref_levelset *lss = static_cast<const ref_levelset *>(levelsets);
  constexpr auto host = execspace_e::host;
  constexpr auto omp = execspace_e::openmp;
  particles_t pars{(size_t)n, memsrc_e::host, -1};
  pars.addAttr("m", attrib_e::scalar);
  pars.addAttr("v", attrib_e::vector);
  pars.addAttr("C", attrib_e::matrix);
  pars.addAttr("F", attrib_e::matrix);
  pars.addAttr("logJp", attrib_e::scalar);
  std::memcpy((float *)pars.getAttrAddress("m"), m, sizeof(float) * n);
  std::memcpy((float *)pars.getAttrAddress("x"), x, sizeof(float) * 3 * n);
  std::memcpy((float *)pars.getAttrAddress("v"), v, sizeof(float) * 3 * n);
  std::memcpy((float *)pars.getAttrAddress("C"), C, sizeof(float) * 9 * n);
  std::memcpy((float *)pars.getAttrAddress("F"), F, sizeof(float) * 9 * n);
  std::memcpy((float *)pars.getAttrAddress("logJp"), logJp, sizeof(float) * n);

  table_t table{(size_t)std::max(p->table_expected, 1), memsrc_e::host, -1};
  grids_t grids{{{"m", 1}, {"v", 3}, {"rhs", 3}}, p->dx, (size_t)table._tableSize,
                memsrc_e::host, -1};

  FixedCorotatedConfig fc{};
  fc.E = p->E;
  fc.nu = p->nu;
  fc.volume = p->volume;
  DruckerPragerConfig dp{};
  dp.E = p->E;
  dp.nu = p->nu;
  dp.volume = p->volume;
  dp.fa = p->friction_deg;
  dp.cohesion = p->cohesion;
  dp.beta = p->beta;
  dp.volumeCorrection = p->volume_correction != 0;
  {
    // ConstitutiveModel.hpp:752 default: sqrt(2/3) * 2 sin(phi) / (3 - sin(phi))
    float sin_phi = (float)std::sin((double)p->friction_deg / 180.0 * 3.14159265358979323846);
    dp.yieldSurface = 0.816496580927726f * 2.f * sin_phi / (3.f - sin_phi);
  }

  std::vector<Collider<plane_t>> walls;
  {
    const float lo = p->wall_cells * p->dx, hi = 1.f - p->wall_cells * p->dx;
    collider_e ct = p->wall_type == 0 ? collider_e::Sticky
                    : p->wall_type == 1 ? collider_e::Slip
                                        : collider_e::Separate;
    for (int d = 0; d != 3; ++d) {
      vec<float, 3> o{0.f, 0.f, 0.f}, nrm{0.f, 0.f, 0.f};
      o[d] = lo;
      nrm[d] = 1.f;
      walls.emplace_back(plane_t{o, nrm}, ct);
      o[d] = hi;
      nrm[d] = -1.f;
      walls.emplace_back(plane_t{o, nrm}, ct);
    }
  }
  const vec<float, 3> grav{p->gx, p->gy, p->gz};
  int status = 0;

  auto run = [&](auto pol, auto tag) {
    constexpr auto space = decltype(tag)::value;
    auto t0 = std::chrono::steady_clock::now();
    for (int step = 0; step != nsteps; ++step) {
      pol(range(table._tableSize), CleanSparsity{wrapv<space>{}, table});
      pol(range((size_t)n),
          ComputeSparsity{wrapv<space>{}, p->dx, 8, table, pars.attrVector("x")});
      int nparblocks = table.size();
      pol(range((size_t)nparblocks),
          EnlargeSparsity{wrapv<space>{}, table, vec<int, 3>{0, 0, 0}, vec<int, 3>{2, 2, 2}});
      int nb = table.size();
      if (nb >= table._tableSize - 20) {
        status = 2;
        return;
      }
      if (p->order == 1) {
        auto *keys = table._activeKeys.data();
        std::sort(keys, keys + nb, [](const auto &a, const auto &b) {
          for (int d = 0; d != 3; ++d)
            if (a[d] != b[d]) return a[d] < b[d];
          return false;
        });
        pol(range(table._tableSize),
            ResetHashTable{proxy<space>(table), false});
        pol(range((size_t)nb), ReinsertHashTable{proxy<space>(table)});
      }
      pol(Collapse{(size_t)nb, (size_t)512}, CleanGridBlocks{wrapv<space>{}, grids});
      if (p->model == 0)
        pol(range((size_t)n), P2GTransfer{wrapv<space>{}, wrapv<transfer_scheme_e::apic>{},
                                          p->dt, fc, pars, table, grids});
      else
        pol(range((size_t)n), P2GTransfer{wrapv<space>{}, wrapv<transfer_scheme_e::apic>{},
                                          p->dt, dp, pars, table, grids});
      pol(Collapse{(size_t)nb, (size_t)512},
          GridVelocityWithRhs<space>{wrapv<space>{}, grids, p->dt, grav});
      for (auto &w : walls)
        pol(Collapse{(size_t)nb, (size_t)512},
            ApplyBoundaryConditionOnGridBlocks{wrapv<space>{}, w, table, grids});
      for (int k = 0; k < ncolliders; ++k) apply_collider(pol, wrapv<space>{}, cols[k], table, grids, nb);
      for (int k = 0; k < nlevelsets; ++k) apply_levelset(pol, wrapv<space>{}, lss[k], table, grids, nb);
      if (p->model == 0)
        pol(range((size_t)n), G2PTransfer{wrapv<space>{}, wrapv<transfer_scheme_e::apic>{},
                                          p->dt, fc, grids, table, pars});
      else
        pol(range((size_t)n), G2PTransfer{wrapv<space>{}, wrapv<transfer_scheme_e::apic>{},
                                          p->dt, dp, grids, table, pars});
    }
    auto t1 = std::chrono::steady_clock::now();
    if (out_seconds) *out_seconds = std::chrono::duration<double>(t1 - t0).count();
  };

  if (p->policy == 0)
    run(seq_exec(), wrapv<host>{});
  else {
    auto pol = omp_exec();
    if (p->threads > 0) pol = OmpExecutionPolicy{}.threads(p->threads);
    run(pol, wrapv<omp>{});
  }
  if (status) return status;

  std::memcpy(x, (float *)pars.getAttrAddress("x"), sizeof(float) * 3 * n);
  std::memcpy(v, (float *)pars.getAttrAddress("v"), sizeof(float) * 3 * n);
  std::memcpy(C, (float *)pars.getAttrAddress("C"), sizeof(float) * 9 * n);
  std::memcpy(F, (float *)pars.getAttrAddress("F"), sizeof(float) * 9 * n);
  std::memcpy(logJp, (float *)pars.getAttrAddress("logJp"), sizeof(float) * n);

  const int nb = table.size();
  if (out_nblocks) *out_nblocks = nb;
  if (out_keys) {
    if (nb > cap_blocks) return 1;
    auto tv = proxy<host>(grids);
    for (int b = 0; b != nb; ++b) {
      auto key = table._activeKeys[b];
      for (int d = 0; d != 3; ++d) out_keys[b * 3 + d] = key[d];
      auto block = tv[b];
      for (int c = 0; c != 4; ++c)
        for (int cell = 0; cell != 512; ++cell)
          out_grid[((size_t)b * 4 + c) * 512 + cell] = block(c, cell);
    }
  }
  return 0;
}

// The cell-centric transfer pair the reference ships without a caller, P2C2GTransfer
// (simulation/transfer/P2C2G.hpp:27-189) and G2C2PTransfer with PreG2C2PTransfer and
// PostG2C2PTransfer (simulation/transfer/G2C2P.hpp:36-278), composed into nsteps substeps:
//   1. the activation of zsref_run, in canonical order;
//   2. the particles' index buckets, built as index_buckets_for_particles does
//      (simulation/particle/Query.tpp:8-58): one bucket per cell coordinate
//      floor(x / dx + 0.5), the collocated offset of IndexBucketsView::bucketCoord;
//   3. CleanGridBlocks, then P2C2GTransfer over every active (block, cell);
//   4. the grid velocity and the walls of zsref_run;
//   5. PreG2C2PTransfer over the particles, G2C2PTransfer over every (block, cell), then
//      PostG2C2PTransfer over the particles.
// Fixed corotated only (p->model == 0; returns 4 otherwise): P2C2G's Drucker-Prager branch
// writes logJp once per visiting cell.  C carries the pair's B attribute between substeps.
// Returns as zsref_run.
int zsref_run_cell(const zsref_params *p, int n, float *m, float *x, float *v, float *C, float *F,
                   int nsteps, int cap_blocks, int *out_nblocks, int *out_keys, float *out_grid,
                   double *out_seconds) {
  if (p->model != 0 || p->order != 1) return 4;
  constexpr auto host = execspace_e::host;
  constexpr auto omp = execspace_e::openmp;
  particles_t pars{(size_t)n, memsrc_e::host, -1};
  pars.addAttr("m", attrib_e::scalar);
  pars.addAttr("v", attrib_e::vector);
  pars.addAttr("C", attrib_e::matrix);
  pars.addAttr("F", attrib_e::matrix);
  pars.addAttr("logJp", attrib_e::scalar);
  std::memcpy((float *)pars.getAttrAddress("m"), m, sizeof(float) * n);
  std::memcpy((float *)pars.getAttrAddress("x"), x, sizeof(float) * 3 * n);
  std::memcpy((float *)pars.getAttrAddress("v"), v, sizeof(float) * 3 * n);
  std::memcpy((float *)pars.getAttrAddress("C"), C, sizeof(float) * 9 * n);
  std::memcpy((float *)pars.getAttrAddress("F"), F, sizeof(float) * 9 * n);
  std::memset((float *)pars.getAttrAddress("logJp"), 0, sizeof(float) * n);

  table_t table{(size_t)std::max(p->table_expected, 1), memsrc_e::host, -1};
  grids_t grids{{{"m", 1}, {"v", 3}, {"rhs", 3}}, p->dx, (size_t)table._tableSize,
                memsrc_e::host, -1};
  FixedCorotatedConfig fc{};
  fc.E = p->E;
  fc.nu = p->nu;
  fc.volume = p->volume;
  std::vector<Collider<plane_t>> walls;
  {
    const float lo = p->wall_cells * p->dx, hi = 1.f - p->wall_cells * p->dx;
    collider_e ct = p->wall_type == 0 ? collider_e::Sticky
                    : p->wall_type == 1 ? collider_e::Slip
                                        : collider_e::Separate;
    for (int d = 0; d != 3; ++d) {
      vec<float, 3> o{0.f, 0.f, 0.f}, nrm{0.f, 0.f, 0.f};
      o[d] = lo;
      nrm[d] = 1.f;
      walls.emplace_back(plane_t{o, nrm}, ct);
      o[d] = hi;
      nrm[d] = -1.f;
      walls.emplace_back(plane_t{o, nrm}, ct);
    }
  }
  const vec<float, 3> grav{p->gx, p->gy, p->gz};
  using buckets_t = IndexBuckets<3, i32, i32>;
  using bvec_t = typename buckets_t::vector_t;
  int status = 0;

  auto run = [&](auto pol, auto tag) {
    constexpr auto space = decltype(tag)::value;
    auto t0 = std::chrono::steady_clock::now();
    for (int step = 0; step != nsteps; ++step) {
      const int nb = activate_canonical(pol, wrapv<space>{}, table, pars, p->dx);
      if (nb < 0) {
        status = 2;
        return;
      }
      // index buckets (Query.tpp:20-56, displacement 0.5)
      buckets_t ib{};
      ib._dx = p->dx;
      ib._table = typename buckets_t::table_t{pars.get_allocator(), pars.size()};
      auto &bt = ib._table;
      pol(range(bt._tableSize), CleanSparsity{wrapv<space>{}, bt});
      pol(range(pars.size()), ComputeSparsity{wrapv<space>{}, p->dx, 1, bt, pars.attrVector("x"), 0, 0.5f});
      const size_t ncells = (size_t)bt.size() + 1;
      ib._counts = bvec_t{pars.get_allocator(), ncells};
      std::memset(ib._counts.data(), 0, sizeof(i32) * ncells);
      auto tmp = ib._counts;
      pol(range(pars.size()),
          SpatiallyCount{wrapv<space>{}, p->dx, bt, pars.attrVector("x"), ib._counts, 1, 0, 0.5f});
      ib._offsets = bvec_t{pars.get_allocator(), ncells};
      exclusive_scan(pol, ib._counts.begin(), ib._counts.end(), ib._offsets.begin());
      ib._indices = bvec_t{pars.get_allocator(), pars.size()};
      pol(range(pars.size()), SpatiallyDistribute{wrapv<space>{}, p->dx, bt, pars.attrVector("x"), tmp,
                                                  ib._offsets, ib._indices, 1, 0, 0.5f});
      pol(Collapse{(size_t)nb, (size_t)512}, CleanGridBlocks{wrapv<space>{}, grids});
      pol(Collapse{(size_t)nb, (size_t)512},
          P2C2GTransfer{wrapv<space>{}, wrapv<transfer_scheme_e::apic>{}, p->dt, fc, ib, pars, table, grids});
      pol(Collapse{(size_t)nb, (size_t)512}, GridVelocityWithRhs<space>{wrapv<space>{}, grids, p->dt, grav});
      for (auto &w : walls)
        pol(Collapse{(size_t)nb, (size_t)512},
            ApplyBoundaryConditionOnGridBlocks{wrapv<space>{}, w, table, grids});
      pol(range(pars.size()), PreG2C2PTransfer{wrapv<space>{}, pars});
      pol(Collapse{(size_t)nb, (size_t)512},
          G2C2PTransfer{wrapv<space>{}, wrapv<transfer_scheme_e::apic>{}, p->dt, fc, ib, grids, table, pars});
      pol(range(pars.size()),
          PostG2C2PTransfer{wrapv<space>{}, wrapv<transfer_scheme_e::apic>{}, p->dt, p->dx, fc, pars});
    }
    auto t1 = std::chrono::steady_clock::now();
    if (out_seconds) *out_seconds = std::chrono::duration<double>(t1 - t0).count();
  };
  if (p->policy == 0)
    run(seq_exec(), wrapv<host>{});
  else {
    auto pol = omp_exec();
    if (p->threads > 0) pol = OmpExecutionPolicy{}.threads(p->threads);
    run(pol, wrapv<omp>{});
  }
  if (status) return status;
  std::memcpy(x, (float *)pars.getAttrAddress("x"), sizeof(float) * 3 * n);
  std::memcpy(v, (float *)pars.getAttrAddress("v"), sizeof(float) * 3 * n);
  std::memcpy(C, (float *)pars.getAttrAddress("C"), sizeof(float) * 9 * n);
  std::memcpy(F, (float *)pars.getAttrAddress("F"), sizeof(float) * 9 * n);
  const int nb = table.size();
  if (out_nblocks) *out_nblocks = nb;
  if (out_keys) {
    if (nb > cap_blocks) return 1;
    auto tv = proxy<host>(grids);
    for (int b = 0; b != nb; ++b) {
      auto key = table._activeKeys[b];
      for (int d = 0; d != 3; ++d) out_keys[b * 3 + d] = key[d];
      auto block = tv[b];
      for (int c = 0; c != 4; ++c)
        for (int cell = 0; cell != 512; ++cell)
          out_grid[((size_t)b * 4 + c) * 512 + cell] = block(c, cell);
    }
  }
  return 0;
}

// G2P2GTransfer on the given particle state (x: 3n, F: 9n column-major, logJp: n) and grid
// velocity field vin, node-major over the canonical blocks: vin[(block*512 + cell)*3 + d], the
// layout of a dof_view<space, 3> over a Vector<float> (types/View.h:77-168).  fout (same
// layout) is zeroed, then receives the operator's atomic sums.  keys are the canonical block
// keys the caller built vin for.  Returns 0; 2 when the table is full; 3 when the activation
// gives other keys than the caller's.
int zsref_g2p2g(const zsref_params *p, int n, const float *x, const float *F, const float *logJp,
                int nb_expected, const int *keys, const float *vin, float *fout,
                double *out_seconds) {
  constexpr auto host = execspace_e::host;
  constexpr auto omp = execspace_e::openmp;
  particles_t pars{(size_t)n, memsrc_e::host, -1};
  pars.addAttr("m", attrib_e::scalar);
  pars.addAttr("F", attrib_e::matrix);
  pars.addAttr("logJp", attrib_e::scalar);
  std::memcpy((float *)pars.getAttrAddress("x"), x, sizeof(float) * 3 * n);
  std::memcpy((float *)pars.getAttrAddress("F"), F, sizeof(float) * 9 * n);
  std::memcpy((float *)pars.getAttrAddress("logJp"), logJp, sizeof(float) * n);
  table_t table{(size_t)std::max(p->table_expected, 1), memsrc_e::host, -1};
  grids_t grids{{{"m", 1}, {"v", 3}, {"rhs", 3}}, p->dx, (size_t)1, memsrc_e::host, -1};
  FixedCorotatedConfig fc{};
  fc.E = p->E;
  fc.nu = p->nu;
  fc.volume = p->volume;
  DruckerPragerConfig dp{};
  dp.E = p->E;
  dp.nu = p->nu;
  dp.volume = p->volume;
  dp.fa = p->friction_deg;
  dp.cohesion = p->cohesion;
  dp.beta = p->beta;
  dp.volumeCorrection = p->volume_correction != 0;
  {
    float sin_phi = (float)std::sin((double)p->friction_deg / 180.0 * 3.14159265358979323846);
    dp.yieldSurface = 0.816496580927726f * 2.f * sin_phi / (3.f - sin_phi);
  }
  const size_t ndofs = (size_t)std::max(nb_expected, 0) * 512 * 3;
  Vector<float> vin_vec{ndofs, memsrc_e::host, -1}, f_vec{ndofs, memsrc_e::host, -1};
  std::memcpy(vin_vec.data(), vin, sizeof(float) * ndofs);
  std::memset(f_vec.data(), 0, sizeof(float) * ndofs);
  int status = 0;
  auto run = [&](auto pol, auto tag) {
    constexpr auto space = decltype(tag)::value;
    const int nb = activate_canonical(pol, wrapv<space>{}, table, pars, p->dx);
    if (nb < 0) {
      status = 2;
      return;
    }
    if (nb != nb_expected) {
      status = 3;
      return;
    }
    for (int b = 0; b != nb; ++b)
      for (int d = 0; d != 3; ++d)
        if (table._activeKeys[b][d] != keys[3 * b + d]) status = 3;
    if (status) return;
    auto vin_view = dof_view<space, 3>(vin_vec);
    auto f_view = dof_view<space, 3>(f_vec);
    auto t0 = std::chrono::steady_clock::now();
    if (p->model == 0)
      pol(range((size_t)n), G2P2GTransfer{wrapv<space>{}, wrapv<transfer_scheme_e::apic>{}, p->dt, fc,
                                          proxy<space>(grids.grid()), vin_view, f_view, table, pars});
    else
      pol(range((size_t)n), G2P2GTransfer{wrapv<space>{}, wrapv<transfer_scheme_e::apic>{}, p->dt, dp,
                                          proxy<space>(grids.grid()), vin_view, f_view, table, pars});
    auto t1 = std::chrono::steady_clock::now();
    if (out_seconds) *out_seconds = std::chrono::duration<double>(t1 - t0).count();
  };
  if (p->policy == 0)
    run(seq_exec(), wrapv<host>{});
  else {
    auto pol = omp_exec();
    if (p->threads > 0) pol = OmpExecutionPolicy{}.threads(p->threads);
    run(pol, wrapv<omp>{});
  }
  if (status) return status;
  std::memcpy(fout, f_vec.data(), sizeof(float) * ndofs);
  return 0;
}

// The implicit system on the given particle state (m: n, x/v: 3n, C/F: 9n, logJp: n) after the
// activation of zsref_run (canonical order; keys must match) and a P2GTransfer that fills the
// grid mass.  Dof vectors a, b, out hold 1536 floats per block (node-major).  op:
//   0  multiply(a -> out)
//   1  project(a in place) -> out
//   2  precondition(a -> out), out preset to b
//   3  ConjugateGradient<float, 3>::solve(system, x = a, b) with maxIters / tol / relTol -> out,
//      *iters = its return value; the solver's q vector is zeroed before the solve (the
//      reference allocates it uninitialised) and its console output is discarded
// out_mass (nb * 512) receives the grid mass.  Returns 0, 2 (table full) or 3 (other keys).
int zsref_implicit(const zsref_params *p, int op, int n, const float *m, const float *x, const float *v,
                   const float *C, const float *F, const float *logJp, int nb_expected, const int *keys,
                   const float *a, const float *b, int max_iters, float tol, float rel_tol, float *out,
                   float *out_mass, int *iters, double *out_seconds) {
  constexpr auto host = execspace_e::host;
  particles_t pars{(size_t)n, memsrc_e::host, -1};
  pars.addAttr("m", attrib_e::scalar);
  pars.addAttr("v", attrib_e::vector);
  pars.addAttr("C", attrib_e::matrix);
  pars.addAttr("F", attrib_e::matrix);
  pars.addAttr("logJp", attrib_e::scalar);
  std::memcpy((float *)pars.getAttrAddress("m"), m, sizeof(float) * n);
  std::memcpy((float *)pars.getAttrAddress("x"), x, sizeof(float) * 3 * n);
  std::memcpy((float *)pars.getAttrAddress("v"), v, sizeof(float) * 3 * n);
  std::memcpy((float *)pars.getAttrAddress("C"), C, sizeof(float) * 9 * n);
  std::memcpy((float *)pars.getAttrAddress("F"), F, sizeof(float) * 9 * n);
  std::memcpy((float *)pars.getAttrAddress("logJp"), logJp, sizeof(float) * n);
  table_t table{(size_t)std::max(p->table_expected, 1), memsrc_e::host, -1};
  auto pol = seq_exec();
  const int nb = activate_canonical(pol, wrapv<host>{}, table, pars, p->dx);
  if (nb < 0) return 2;
  if (nb != nb_expected) return 3;
  for (int bb = 0; bb != nb; ++bb)
    for (int d = 0; d != 3; ++d)
      if (table._activeKeys[bb][d] != keys[3 * bb + d]) return 3;
  grids_t grids{{{"m", 1}, {"v", 3}, {"rhs", 3}}, p->dx, (size_t)table._tableSize, memsrc_e::host, -1};
  FixedCorotatedConfig fc{};
  fc.E = p->E;
  fc.nu = p->nu;
  fc.volume = p->volume;
  DruckerPragerConfig dp{};
  dp.E = p->E;
  dp.nu = p->nu;
  dp.volume = p->volume;
  dp.fa = p->friction_deg;
  dp.cohesion = p->cohesion;
  dp.beta = p->beta;
  dp.volumeCorrection = p->volume_correction != 0;
  {
    float sin_phi = (float)std::sin((double)p->friction_deg / 180.0 * 3.14159265358979323846);
    dp.yieldSurface = 0.816496580927726f * 2.f * sin_phi / (3.f - sin_phi);
  }
  std::vector<Collider<plane_t>> walls;
  if (p->wall_type != 3) {
    const float lo = p->wall_cells * p->dx, hi = 1.f - p->wall_cells * p->dx;
    collider_e ct = p->wall_type == 0 ? collider_e::Sticky
                    : p->wall_type == 1 ? collider_e::Slip
                                        : collider_e::Separate;
    for (int d = 0; d != 3; ++d) {
      vec<float, 3> o{0.f, 0.f, 0.f}, nrm{0.f, 0.f, 0.f};
      o[d] = lo;
      nrm[d] = 1.f;
      walls.emplace_back(plane_t{o, nrm}, ct);
      o[d] = hi;
      nrm[d] = -1.f;
      walls.emplace_back(plane_t{o, nrm}, ct);
    }
  }
  pol(Collapse{(size_t)nb, (size_t)512}, CleanGridBlocks{wrapv<host>{}, grids});
  // P2G's stress term reads a copy of F and writes logJp; the implicit operators read the
  // uploaded logJp, so it is restored
  if (p->model == 0)
    pol(range((size_t)n), P2GTransfer{wrapv<host>{}, wrapv<transfer_scheme_e::apic>{}, p->dt, fc, pars, table, grids});
  else
    pol(range((size_t)n), P2GTransfer{wrapv<host>{}, wrapv<transfer_scheme_e::apic>{}, p->dt, dp, pars, table, grids});
  std::memcpy((float *)pars.getAttrAddress("logJp"), logJp, sizeof(float) * n);
  {
    auto tv = proxy<host>(grids);
    for (int bb = 0; bb != nb; ++bb)
      for (int cell = 0; cell != 512; ++cell) out_mass[(size_t)bb * 512 + cell] = tv[bb](0, cell);
  }
  const size_t ndofs = (size_t)nb * 1536;
  Vector<float> va{ndofs, memsrc_e::host, -1}, vb{ndofs, memsrc_e::host, -1}, vo{ndofs, memsrc_e::host, -1};
  std::memcpy(va.data(), a, sizeof(float) * ndofs);
  std::memcpy(vb.data(), b, sizeof(float) * ndofs);
  std::memset(vo.data(), 0, sizeof(float) * ndofs);
  auto da = dof_view<host, 3>(va), db = dof_view<host, 3>(vb), dout = dof_view<host, 3>(vo);
  auto t0 = std::chrono::steady_clock::now();
  auto go = [&](auto model) {
    RefImplicitSystem<decltype(model)> sys{model, table, pars, grids, walls, p->dt};
    if (op == 0) {
      sys.multiply(pol, da, dout);
    } else if (op == 1) {
      sys.project(pol, da);
      std::memcpy(vo.data(), va.data(), sizeof(float) * ndofs);
    } else if (op == 2) {
      std::memcpy(vo.data(), vb.data(), sizeof(float) * ndofs);
      sys.precondition(pol, da, dout);
    } else {
      ConjugateGradient<float, 3> cg{ndofs, memsrc_e::host, -1};
      cg.maxIters = max_iters;
      cg.tol = tol;
      cg.relTol = rel_tol;
      cg.resize(ndofs);
      std::memset(cg.q_.data(), 0, sizeof(float) * ndofs);
      std::FILE *null_in = std::freopen("/dev/null", "r", stdin);
      (void)null_in;
      std::streambuf *saved = std::cout.rdbuf(nullptr);
      *iters = cg.solve(pol, sys, da, db);
      std::cout.rdbuf(saved);
      std::cout.clear();
      std::memcpy(vo.data(), va.data(), sizeof(float) * ndofs);
    }
  };
  if (p->model == 0)
    go(fc);
  else
    go(dp);
  auto t1 = std::chrono::steady_clock::now();
  if (out_seconds) *out_seconds = std::chrono::duration<double>(t1 - t0).count();
  std::memcpy(out, vo.data(), sizeof(float) * ndofs);
  return 0;
}

// Reference-verbatim stress of one particle, for unit parity of the constitutive code
// (physics/ConstitutiveModel_Vol_dP.hpp:10-46 and :241-325).  PF and F are column-major.
void zsref_stress(int model, float volume, float E, float nu, float friction_deg,
                  float cohesion, float beta, int volume_correction, float *F, float *logJp,
                  float *PF) {
  auto [mu, lambda] = lame_parameters(E, nu);
  vec<float, 9> f{}, pf{};
  for (int i = 0; i != 9; ++i) f[i] = F[i];
  if (model == 0)
    compute_stress_fixedcorotated(volume, mu, lambda, f, pf);
  else {
    float sin_phi = (float)std::sin((double)friction_deg / 180.0 * 3.14159265358979323846);
    float ys = 0.816496580927726f * 2.f * sin_phi / (3.f - sin_phi);
    compute_stress_sand(volume, mu, lambda, cohesion, beta, ys, volume_correction != 0, *logJp,
                        f, pf);
    for (int i = 0; i != 9; ++i) F[i] = f[i];
  }
  for (int i = 0; i != 9; ++i) PF[i] = pf[i];
}

// The reference's float 3x3 SVD (math/matrix/SVD.hpp:15-1025), A column-major.
void zsref_svd(const float *A, float *U, float *S, float *V) {
  math::svd_3d(A[0], A[3], A[6], A[1], A[4], A[7], A[2], A[5], A[8], U[0], U[3], U[6], U[1],
               U[4], U[7], U[2], U[5], U[8], S[0], S[1], S[2], V[0], V[3], V[6], V[1], V[4],
               V[7], V[2], V[5], V[8]);
}

// Block keys of a HashTable after inserting the given particle positions in order with
// seq_exec (ComputeSparsity + EnlargeSparsity), in the table's own insertion order.
// Also reports, for every key, the table slot it landed in.
int zsref_activate(int n, const float *x, float dx, int table_expected, int cap,
                   int *out_nblocks, int *out_nparblocks, int *out_keys, int *out_slots,
                   int *out_table_size) {
  constexpr auto host = execspace_e::host;
  particles_t pars{(size_t)n, memsrc_e::host, -1};
  std::memcpy((float *)pars.getAttrAddress("x"), x, sizeof(float) * 3 * n);
  table_t table{(size_t)std::max(table_expected, 1), memsrc_e::host, -1};
  auto pol = seq_exec();
  pol(range(table._tableSize), CleanSparsity{wrapv<host>{}, table});
  pol(range((size_t)n), ComputeSparsity{wrapv<host>{}, dx, 8, table, pars.attrVector("x")});
  int npb = table.size();
  pol(range((size_t)npb),
      EnlargeSparsity{wrapv<host>{}, table, vec<int, 3>{0, 0, 0}, vec<int, 3>{2, 2, 2}});
  int nb = table.size();
  *out_nblocks = nb;
  *out_nparblocks = npb;
  *out_table_size = table._tableSize;
  if (nb > cap) return 1;
  auto view = proxy<host>(table);
  for (int b = 0; b != nb; ++b) {
    auto key = table._activeKeys[b];
    for (int d = 0; d != 3; ++d) out_keys[b * 3 + d] = key[d];
    out_slots[b] = view.entry(key);
  }
  return 0;
}

// A bht<i32,3,int,16> (container/Bht.hpp) built by the reference's own host insert
// (BHTView::insert, Bht.hpp:612-665) from the given keys in the given order, default insertion
// indices.  Outputs: table size, the three hashers' (hashx, hashy), and per slot the stored key
// (x, y, z), index and status; cnt.  Returns 1 when cap_slots is too small.
int zsref_bht(int nkeys, const int *keys, int expected, int cap_slots, int *out_table_size,
              unsigned *out_hash, int *out_keys, int *out_indices, int *out_status, int *out_cnt) {
  using bht_t = zs::bht<int, 3, int, 16>;
  bht_t table{(size_t)std::max(expected, 1), memsrc_e::host, -1};
  *out_table_size = (int)table._tableSize;
  out_hash[0] = table._hf0._hashx;
  out_hash[1] = table._hf0._hashy;
  out_hash[2] = table._hf1._hashx;
  out_hash[3] = table._hf1._hashy;
  out_hash[4] = table._hf2._hashx;
  out_hash[5] = table._hf2._hashy;
  if ((int)table._tableSize > cap_slots) return 1;
  auto v = view<execspace_e::host>(table);
  for (int k = 0; k != nkeys; ++k) v.insert(vec<int, 3>{keys[3 * k], keys[3 * k + 1], keys[3 * k + 2]});
  for (int i = 0; i != (int)table._tableSize; ++i) {
    const auto &sk = table.self().keys[i];
    for (int d = 0; d != 3; ++d) out_keys[3 * i + d] = sk.val[d];
    out_indices[i] = table.self().indices[i];
    out_status[i] = table.self().status[i];
  }
  *out_cnt = (int)table.size();
  return 0;
}

}  // extern "C"
