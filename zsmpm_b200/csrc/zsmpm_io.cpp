// Particle output in Houdini's classic binary geometry format (.bgeo), the file that
// zs::write_partio and its two variants (io/ParticleIO.hpp:11-22, io/ParticleIO.cpp) write
// through the partio library.  The partio library is not part of the reference tree, so this
// is a writer of the published layout, in this library's own code:
//
//   header      int32 magic "Bgeo", char 'V', int32 version 5, then int32 counts: points,
//               primitives (1), point groups (0), primitive groups (0), point attributes,
//               vertex attributes (0), primitive attributes (1), detail attributes (0)
//   attributes  per point attribute other than the position: uint16 name length, the name,
//               uint16 component count, int32 type (0 float, 5 vector), one int32 zero
//               default per component
//   points      per point: float32 x y z and the homogeneous w = 1, then the attribute values
//   primitives  the primitive attribute "generator" (uint16 length, name, uint16 size 1,
//               int32 type 4 = index, int32 one string, uint16 length, "papi"), then one
//               particle-system primitive: int32 0x8000, int32 point count, the point indices
//               (uint16 below 65,536 points, else int32), int32 generator index 0
//   trailer     bytes 0x00 and 0xff
//
// All numbers are big-endian.  The attribute named "position" is written as the points'
// position P, as partio does; a write_partio call with another tag stores the data as a
// vector attribute of that name and P as zeros.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "zsmpm.h"

namespace zsmpm {
int record_error(int status, const char *message);  // zsmpm_api.cu: the calling thread's error text
}

namespace {

struct be_writer {
  std::vector<unsigned char> buf;
  void u8(uint8_t v) { buf.push_back(v); }
  void u16(uint16_t v) {
    buf.push_back((unsigned char)(v >> 8));
    buf.push_back((unsigned char)(v & 0xff));
  }
  void u32(uint32_t v) {
    for (int s = 24; s >= 0; s -= 8) buf.push_back((unsigned char)((v >> s) & 0xff));
  }
  void i32(int32_t v) { u32((uint32_t)v); }
  void f32(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    u32(u);
  }
  void str(const std::string &s) {
    u16((uint16_t)s.size());
    buf.insert(buf.end(), s.begin(), s.end());
  }
};

struct point_attribute {
  std::string name;
  int components;   // 1 (float) or 3 (vector)
  const float *data;  // [n][components]
};

int write_bgeo(const char *path, const float *pos, int64_t n, const std::vector<point_attribute> &attrs) {
  using zsmpm::record_error;
  if (!path || !*path) return record_error(ZSMPM_ERR_INVALID_ARG, "write_partio: empty path");
  const std::string p(path);
  if (p.size() < 5 || p.compare(p.size() - 5, 5, ".bgeo") != 0)
    return record_error(ZSMPM_ERR_INVALID_ARG,
                        "write_partio: only uncompressed Houdini .bgeo output is built (the path must end in .bgeo)");
  if (n < 0 || n > 0x7fffffff) return record_error(ZSMPM_ERR_INVALID_ARG, "write_partio: particle count out of range");
  for (const auto &a : attrs)
    if (n > 0 && !a.data) return record_error(ZSMPM_ERR_INVALID_ARG, "write_partio: null attribute data");
  be_writer w;
  w.buf.reserve(64 + (size_t)n * (16 + 12 * attrs.size() + 4));
  w.u32(((uint32_t)'B' << 24) | ((uint32_t)'g' << 16) | ((uint32_t)'e' << 8) | (uint32_t)'o');
  w.u8('V');
  w.i32(5);
  w.i32((int32_t)n);  // points
  w.i32(1);           // primitives: one particle system
  w.i32(0);           // point groups
  w.i32(0);           // primitive groups
  w.i32((int32_t)attrs.size());
  w.i32(0);  // vertex attributes
  w.i32(1);  // primitive attributes: "generator"
  w.i32(0);  // detail attributes
  for (const auto &a : attrs) {
    w.str(a.name);
    w.u16((uint16_t)a.components);
    w.i32(a.components == 3 ? 5 : 0);
    for (int k = 0; k < a.components; ++k) w.i32(0);
  }
  for (int64_t i = 0; i < n; ++i) {
    for (int d = 0; d < 3; ++d) w.f32(pos ? pos[3 * i + d] : 0.f);
    w.f32(1.f);
    for (const auto &a : attrs)
      for (int k = 0; k < a.components; ++k) w.f32(a.data[(size_t)i * a.components + k]);
  }
  w.str("generator");
  w.u16(1);
  w.i32(4);
  w.i32(1);
  w.str("papi");
  w.i32(0x8000);
  w.i32((int32_t)n);
  for (int64_t i = 0; i < n; ++i) {
    if (n < 65536)
      w.u16((uint16_t)i);
    else
      w.i32((int32_t)i);
  }
  w.i32(0);
  w.u8(0x00);
  w.u8(0xff);
  FILE *f = std::fopen(path, "wb");
  if (!f) return record_error(ZSMPM_ERR_INVALID_ARG, (std::string("write_partio: cannot open ") + p).c_str());
  const size_t put = std::fwrite(w.buf.data(), 1, w.buf.size(), f);
  const int closed = std::fclose(f);
  if (put != w.buf.size() || closed != 0)
    return record_error(ZSMPM_ERR_INVALID_ARG, (std::string("write_partio: short write to ") + p).c_str());
  return ZSMPM_OK;
}

}  // namespace

extern "C" {

ZSMPM_API zsmpm_status zsmpm_write_partio(const char *path, const float *data, int64_t n, const char *tag) {
  const std::string name = tag && *tag ? tag : "position";
  if (n > 0 && !data) return (zsmpm_status)zsmpm::record_error(ZSMPM_ERR_INVALID_ARG, "write_partio: null data");
  if (name == "position") return (zsmpm_status)write_bgeo(path, data, n, {});
  return (zsmpm_status)write_bgeo(path, nullptr, n, {point_attribute{name, 3, data}});
}

ZSMPM_API zsmpm_status zsmpm_write_partio_with_stress(const char *path, const float *pos, const float *stress,
                                                      int64_t n) {
  if (n > 0 && (!pos || !stress))
    return (zsmpm_status)zsmpm::record_error(ZSMPM_ERR_INVALID_ARG, "write_partio_with_stress: null data");
  return (zsmpm_status)write_bgeo(path, pos, n, {point_attribute{"stress", 1, stress}});
}

ZSMPM_API zsmpm_status zsmpm_write_partio_with_grid(const char *path, const float *pos, const float *force,
                                                    int64_t n) {
  if (n > 0 && (!pos || !force))
    return (zsmpm_status)zsmpm::record_error(ZSMPM_ERR_INVALID_ARG, "write_partio_with_grid: null data");
  return (zsmpm_status)write_bgeo(path, pos, n, {point_attribute{"force", 3, force}});
}

}  // extern "C"
