/* zsmpm_zpc.hpp -- libzsmpm over zpc's own containers (C++, header only).
 *
 * For a zpc program whose particles live in a zs::TileVector<float, 32> and whose operators
 * query blocks through a zs::HashTable<int, 3, int>.  Include it after zpc's container headers:
 *
 *   #include "zensim/container/TileVector.hpp"
 *   #include "zensim/container/HashTable.hpp"
 *   #include "zsmpm_zpc.hpp"
 *
 * and link libzsmpm.so.  Everything here goes through the C ABI of zsmpm.h; no CUDA header is
 * needed.
 *
 *   upload / download   particles between a TileVector<float, 32> whose properties carry the
 *                       names zs::Particles gives its attributes ("m", "x", "v", "C", "F",
 *                       "logJp" or "Jp"; py_interop/TileVectorView.hpp:10-60) and a scene.  A
 *                       TileVector in device memory is read and written in place by the
 *                       library's kernels (zsmpm_scene_upload_tilevector / _download_tilevector);
 *                       one in host memory goes through the SoA arrays of zsmpm_particle_arrays.
 *   table_view          a zs::HashTableView<space, HashTable<int, 3, int>> over the scene's own
 *                       block table in device memory, without a copy: keys, indices, status,
 *                       active keys, count and table size (container/HashTable.hpp:313-490)
 *                       point at the library's arrays, which have the HashTable storage layout.
 *                       zpc operators launched with it (a CUDA policy over Collapse{nb, 512},
 *                       queries through unpack_coord_in_grid) see the blocks of the last
 *                       activation; the view is valid until the next activation.
 *   copy_table          the same table copied into a caller's zs::HashTable (host or device
 *                       memory) sized for the same expected entry count.
 *
 * The scene keeps its particles binned and double-buffered in its own SoA layout (the B200
 * transfer kernels stage particles by cell), so particles cross by a copy each way; the block
 * table and its slots are shared as they are.
 */
#pragma once

#include <cstdint>
#include <type_traits>
#include <vector>

#include "zsmpm.h"

namespace zsmpm {
namespace zpc {

/* The library's view of a TileVector<float, 32>: base pointer, channel count and the channel
 * offsets of the attributes, -1 where a property is absent. */
template <typename TileVectorT>
zsmpm_tilevector_view tilevector_view(TileVectorT &tv) {
  static_assert(std::is_same<typename TileVectorT::value_type, float>::value,
                "libzsmpm takes TileVector<float, 32> particle attributes");
  static_assert(TileVectorT::lane_width == 32, "libzsmpm takes TileVector<float, 32> particle attributes");
  zsmpm_tilevector_view v{};
  v.base = tv.data();
  v.num_channels = (int32_t)tv.numChannels();
  v.lane_width = 32;
  auto off = [&](const char *name) { return tv.hasProperty(name) ? (int32_t)tv.getPropertyOffset(name) : -1; };
  v.off_m = off("m");
  v.off_x = off("x");
  v.off_v = off("v");
  v.off_C = off("C");
  v.off_F = off("F");
  v.off_plastic = off("logJp") >= 0 ? off("logJp") : off("Jp");
  return v;
}

namespace detail {
/* SoA host arrays of n particles for a host TileVector, channel by channel */
struct host_soa {
  std::vector<float> m, x, v, C, F, pl;
  zsmpm_particle_arrays arrays(const zsmpm_tilevector_view &tv) {
    zsmpm_particle_arrays a{};
    a.m = tv.off_m >= 0 ? m.data() : nullptr;
    a.x = tv.off_x >= 0 ? x.data() : nullptr;
    a.v = tv.off_v >= 0 ? v.data() : nullptr;
    a.C = tv.off_C >= 0 ? C.data() : nullptr;
    a.F = tv.off_F >= 0 ? F.data() : nullptr;
    a.plastic = tv.off_plastic >= 0 ? pl.data() : nullptr;
    return a;
  }
  explicit host_soa(int64_t n) : m(n), x(3 * n), v(3 * n), C(9 * n), F(9 * n), pl(n) {}
};
/* element (chn, i) of a TileVector<float, 32>: ((i / 32) nchn + chn) 32 + i % 32 */
inline float &tile_at(const zsmpm_tilevector_view &tv, int chn, int64_t i) {
  return tv.base[((i >> 5) * tv.num_channels + chn) * 32 + (i & 31)];
}
/* copies between the SoA arrays (vectors and 3x3 matrices per particle, column-major) and
 * the tiles; to_tiles selects the direction */
inline void move_channels(const zsmpm_tilevector_view &tv, host_soa &a, int64_t n, bool to_tiles) {
  struct field {
    int off, width;
    float *soa;
  } fields[] = {{tv.off_m, 1, a.m.data()}, {tv.off_x, 3, a.x.data()}, {tv.off_v, 3, a.v.data()},
                {tv.off_C, 9, a.C.data()}, {tv.off_F, 9, a.F.data()}, {tv.off_plastic, 1, a.pl.data()}};
  for (const field &f : fields) {
    if (f.off < 0) continue;
    for (int64_t i = 0; i < n; ++i)
      for (int k = 0; k < f.width; ++k) {
        float &t = tile_at(tv, f.off + k, i);
        float &s = f.soa[i * f.width + k];
        if (to_tiles)
          t = s;
        else
          s = t;
      }
  }
}
}  // namespace detail

/* Particles of `tv` (tv.size() of them) into the scene, as zsmpm_scene_upload does. */
template <typename TileVectorT>
zsmpm_status upload(zsmpm_scene *s, TileVectorT &tv, void *stream = nullptr) {
  const int64_t n = (int64_t)tv.size();
  const zsmpm_tilevector_view view = tilevector_view(tv);
  if (tv.memspace() != zs::memsrc_e::host) return zsmpm_scene_upload_tilevector(s, &view, n, stream);
  detail::host_soa a(n);
  detail::move_channels(view, a, n, false);
  zsmpm_particle_arrays arrays = a.arrays(view);
  return zsmpm_scene_upload(s, &arrays, n, 0, stream);
}

/* The scene's particles, in upload order, into the attributes `tv` has (tv.size() must equal
 * the scene's particle count).  A host TileVector is complete when this returns. */
template <typename TileVectorT>
zsmpm_status download(zsmpm_scene *s, TileVectorT &tv, void *stream = nullptr) {
  const int64_t n = zsmpm_scene_num_particles(s);
  if (n != (int64_t)tv.size()) return ZSMPM_ERR_INVALID_ARG;
  const zsmpm_tilevector_view view = tilevector_view(tv);
  if (tv.memspace() != zs::memsrc_e::host) return zsmpm_scene_download_tilevector(s, &view, stream);
  detail::host_soa a(n);
  zsmpm_particle_arrays arrays = a.arrays(view);
  const zsmpm_status st = zsmpm_scene_download(s, &arrays, 0, stream);
  if (st == ZSMPM_OK) detail::move_channels(view, a, n, true);
  return st;
}

/* A zpc HashTableView over the scene's block table in device memory (no copy).  *status
 * (optional) receives the outcome; on failure the view is empty. */
template <zs::execspace_e Space, typename TableT = zs::HashTable<int, 3, int>>
zs::HashTableView<Space, TableT> table_view(zsmpm_scene *s, zsmpm_status *status = nullptr) {
  using key_t = typename TableT::key_t;
  static_assert(TableT::dim == 3 && sizeof(key_t) == 3 * sizeof(int32_t) &&
                    sizeof(typename TableT::value_t) == sizeof(int32_t),
                "the scene's block table is a HashTable<int, 3, int>");
  zs::HashTableView<Space, TableT> v{};
  zsmpm_table_view t{};
  const zsmpm_status st = zsmpm_get_table_view(s, &t);
  if (st == ZSMPM_OK) {
    v._table.keys = reinterpret_cast<key_t *>(t.keys);
    v._table.indices = t.indices;
    v._table.status = t.status;
    v._activeKeys = reinterpret_cast<key_t *>(t.active_keys);
    v._tableSize = t.table_size;
    v._cnt = t.cnt;
  }
  if (status) *status = st;
  return v;
}

/* The scene's block table copied into `out`, a zs::HashTable<int, 3, int> in host or device
 * memory sized for the same expected entry count (the same table size). */
template <typename TableT>
zsmpm_status copy_table(zsmpm_scene *s, TableT &out, void *stream = nullptr) {
  static_assert(TableT::dim == 3 && sizeof(typename TableT::key_t) == 3 * sizeof(int32_t) &&
                    sizeof(typename TableT::value_t) == sizeof(int32_t),
                "the scene's block table is a HashTable<int, 3, int>");
  return zsmpm_download_table(s, reinterpret_cast<int32_t *>(out.self().keys.data()), out.self().indices.data(),
                              out.self().status.data(), reinterpret_cast<int32_t *>(out._activeKeys.data()),
                              (int32_t)out._activeKeys.size(), out._cnt.data(), (int32_t)out._tableSize, stream);
}

}  // namespace zpc
}  // namespace zsmpm
