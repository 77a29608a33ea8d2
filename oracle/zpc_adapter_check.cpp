// Test infrastructure: checks include/zsmpm_zpc.hpp against zpc's own container types.  Built by
// oracle/build_ref.sh with the reference's headers and host runtime (the same objects as
// zsref_cli) and linked with libzsmpm.so; tests/test_zpc_adapter.py runs it on a GPU.
//
//   1. a zs::TileVector<float, 32> in host memory with the properties m, x, v, C, F, logJp holds
//      a sand box; zsmpm::zpc::upload puts it into a scene, which runs 5 substeps;
//   2. zsmpm::zpc::download fills the TileVector again; every value equals the scene's own SoA
//      download (zsmpm_scene_download) bit for bit;
//   3. zsmpm::zpc::copy_table fills a zs::HashTable<int, 3, int> sized for the scene's expected
//      entry count; zpc's own HashTableView::query (container/HashTable.hpp:444-456), run on the
//      host through proxy<host>, finds every active key at its index, and keys that are not
//      there come back as -1;
//   4. zsmpm::zpc::table_view gives a device HashTableView whose pointers and size are the
//      scene's table view.
// Prints one line and exits 0 when every check holds; exits 1 with the first failure.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "zensim/container/HashTable.hpp"
#include "zensim/container/TileVector.hpp"
#include "zsmpm_zpc.hpp"

#include "zeroed_new.hpp"  // the reference registry's mutex starts unlocked

namespace {

int fail(const char *what) {
  std::printf("zpc adapter check FAILED: %s (%s)\n", what, zsmpm_last_error_string());
  std::fflush(stdout);
  return 1;
}

// splitmix64 of i, as a float in [0, 1)
float unit(uint64_t i) {
  uint64_t z = i + 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return (float)(z >> 40) / (float)(1ull << 24);
}

}  // namespace

int main() {
  const float dx = 1.f / 128;
  // a sand box [0.44, 0.56]^3 at 8 jittered particles per cell, moving at (0.5, -0.4, 0.3)
  std::vector<float> pos;
  const int c0 = (int)std::lround(0.44 / dx), c1 = (int)std::lround(0.56 / dx);
  uint64_t seq = 0;
  for (int i = c0; i < c1; ++i)
    for (int j = c0; j < c1; ++j)
      for (int k = c0; k < c1; ++k)
        for (int s = 0; s < 8; ++s) {
          const float sub[3] = {0.25f + 0.5f * (s >> 2), 0.25f + 0.5f * ((s >> 1) & 1), 0.25f + 0.5f * (s & 1)};
          const int cell[3] = {i, j, k};
          for (int d = 0; d < 3; ++d) pos.push_back(((float)cell[d] + sub[d] + 0.5f * (unit(seq++) - 0.5f)) * dx);
        }
  const size_t n = pos.size() / 3;
  const float volume = dx * dx * dx / 8;

  zs::TileVector<float, 32> tv{{{"m", 1}, {"x", 3}, {"v", 3}, {"C", 9}, {"F", 9}, {"logJp", 1}}, n,
                               zs::memsrc_e::host, -1};
  {
    const zsmpm_tilevector_view w = zsmpm::zpc::tilevector_view(tv);
    for (size_t p = 0; p < n; ++p) {
      zsmpm::zpc::detail::tile_at(w, w.off_m, p) = 2200.f * volume;
      const float vel[3] = {0.5f, -0.4f, 0.3f};
      for (int d = 0; d < 3; ++d) {
        zsmpm::zpc::detail::tile_at(w, w.off_x + d, p) = pos[3 * p + d];
        zsmpm::zpc::detail::tile_at(w, w.off_v + d, p) = vel[d];
      }
      for (int k = 0; k < 9; ++k) {
        zsmpm::zpc::detail::tile_at(w, w.off_C + k, p) = 0.f;
        zsmpm::zpc::detail::tile_at(w, w.off_F + k, p) = (k % 4 == 0) ? 1.f : 0.f;
      }
      zsmpm::zpc::detail::tile_at(w, w.off_plastic, p) = 0.f;
    }
  }

  zsmpm_scene_desc d{};
  d.dx = dx;
  d.dt = 5e-5f;
  d.gravity[1] = -9.8f;
  d.wall_type = ZSMPM_WALL_SLIP;
  d.wall_cells = 3;
  d.material.model = ZSMPM_DRUCKER_PRAGER;
  d.material.plasticity_mode = ZSMPM_PLASTICITY_COMMITTED;
  d.material.E = 3.5e5f;
  d.material.nu = 0.3f;
  d.material.rho = 2200.f;
  d.material.volume = volume;
  d.material.friction_deg = 30.f;
  d.material.beta = 1.f;
  d.material.volume_correction = 1;
  d.block_order = ZSMPM_BLOCK_ORDER_SORTED;
  const int expected = (int)std::max<size_t>(n / 512, 64);
  d.table_expected = expected;
  zsmpm_scene *s = nullptr;
  if (zsmpm_scene_create(&d, &s) != ZSMPM_OK) return fail("scene_create");
  if (zsmpm::zpc::upload(s, tv) != ZSMPM_OK) return fail("upload from the TileVector");
  if (zsmpm_run(s, 5, nullptr) != ZSMPM_OK || zsmpm_scene_status(s) != ZSMPM_OK) return fail("run");

  // 2. the TileVector download against the SoA download
  if (zsmpm::zpc::download(s, tv) != ZSMPM_OK) return fail("download into the TileVector");
  std::vector<float> m(n), x(3 * n), v(3 * n), C(9 * n), F(9 * n), pl(n);
  zsmpm_particle_arrays a{m.data(), x.data(), v.data(), C.data(), F.data(), pl.data()};
  if (zsmpm_scene_download(s, &a, 0, nullptr) != ZSMPM_OK) return fail("SoA download");
  const zsmpm_tilevector_view w = zsmpm::zpc::tilevector_view(tv);
  double moved = 0;
  for (size_t p = 0; p < n; ++p) {
    const float *soa[] = {&m[p], &x[3 * p], &v[3 * p], &C[9 * p], &F[9 * p], &pl[p]};
    const int off[] = {w.off_m, w.off_x, w.off_v, w.off_C, w.off_F, w.off_plastic};
    const int width[] = {1, 3, 3, 9, 9, 1};
    for (int f = 0; f < 6; ++f)
      for (int k = 0; k < width[f]; ++k) {
        const float t = zsmpm::zpc::detail::tile_at(w, off[f] + k, p);
        if (std::memcmp(&t, &soa[f][k], sizeof(float)) != 0) return fail("TileVector download differs from SoA");
      }
    moved += std::fabs(x[3 * p] - pos[3 * p]);
  }
  if (!(moved > 0)) return fail("particles did not move");

  // 3. the table in a caller's zs::HashTable, queried by zpc's own code
  int32_t nb = 0;
  if (zsmpm_num_blocks(s, &nb) != ZSMPM_OK) return fail("num_blocks");
  zs::HashTable<int, 3, int> table{(size_t)expected, zs::memsrc_e::host, -1};
  if (zsmpm::zpc::copy_table(s, table) != ZSMPM_OK) return fail("copy_table");
  if (table.size() != nb) return fail("table count");
  auto hv = zs::proxy<zs::execspace_e::host>(table);
  for (int b = 0; b < nb; ++b) {
    const auto key = table._activeKeys[b];
    if (hv.query(key) != b) return fail("zpc query does not find an active key at its index");
    if (b > 0) {
      const auto prev = table._activeKeys[b - 1];
      const bool ascending = prev[0] < key[0] || (prev[0] == key[0] && (prev[1] < key[1] ||
                                                  (prev[1] == key[1] && prev[2] < key[2])));
      if (!ascending) return fail("active keys not in ascending order");
    }
  }
  if (hv.query(zs::vec<int, 3>{100000, -100000, 7}) != -1) return fail("query of an absent key");
  zs::HashTable<int, 3, int> small{(size_t)expected / 4, zs::memsrc_e::host, -1};
  if (zsmpm::zpc::copy_table(s, small) != ZSMPM_ERR_INVALID_ARG) return fail("a table of another size was taken");

  // 4. the in-place device view
  zsmpm_status st = ZSMPM_ERR_INVALID_ARG;
  auto dv = zsmpm::zpc::table_view<zs::execspace_e::cuda>(s, &st);
  zsmpm_table_view tvw{};
  if (st != ZSMPM_OK || zsmpm_get_table_view(s, &tvw) != ZSMPM_OK) return fail("table_view");
  if ((void *)dv._table.keys != (void *)tvw.keys || dv._table.indices != tvw.indices ||
      dv._table.status != tvw.status || (void *)dv._activeKeys != (void *)tvw.active_keys || dv._cnt != tvw.cnt ||
      dv._tableSize != tvw.table_size || dv._tableSize != table._tableSize)
    return fail("device view fields");

  zsmpm_scene_destroy(s);
  std::printf("zpc adapter check ok: %zu particles in a TileVector<float, 32>, %d blocks found by zpc's query in "
              "a HashTable<int, 3, int> of %d slots\n",
              n, nb, (int)table._tableSize);
  return 0;
}
