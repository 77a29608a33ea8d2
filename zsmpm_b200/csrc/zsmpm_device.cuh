// Device-side math of the MPM substep: packed block keys, the reference's hash, the 3x3
// SVD, the constitutive updates and warp/CTA helpers.  Everything here is __device__ code
// for sm_100a; host code sees only the constants.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace zsmpm {

// ---------------------------------------------------------------- constants / layout
constexpr int kSide = 8;                 // block side (cells)
constexpr int kBlockCells = 512;         // 8^3
constexpr int kGridChannels = 4;         // m, p.x/v.x, p.y/v.y, p.z/v.z
constexpr int kHalo = 12;                // halo side, cells [8b, 8b+12) per axis
constexpr int kHaloCells = kHalo * kHalo * kHalo;
constexpr uint64_t kEmptyKey = ~0ull;
constexpr int kKeyBias = 1 << 20;        // packed block coordinate bias (21 bits each)
constexpr int kKeyLimit = (1 << 20) - 4; // |block coordinate| must stay below this

// device status word bits (OR-ed), surfaced as zsmpm_status by the host
enum : int {
  kStatusTableFull = 1 << 0,
  kStatusCapacity = 1 << 1,
  kStatusOutOfDomain = 1 << 2,
  kStatusMissingBlock = 1 << 3,
  kStatusTimeout = 1 << 4,
  kStatusBitmap = 1 << 5,
};

// Block keys travel packed into 63 bits: (bx+2^20)<<42 | (by+2^20)<<21 | (bz+2^20).
// Packed order equals lexicographic (bx, by, bz) order.
__host__ __device__ __forceinline__ uint64_t pack_key(int bx, int by, int bz) {
  return ((uint64_t)(uint32_t)(bx + kKeyBias) << 42) | ((uint64_t)(uint32_t)(by + kKeyBias) << 21) |
         (uint64_t)(uint32_t)(bz + kKeyBias);
}
__host__ __device__ __forceinline__ int3 unpack_key(uint64_t k) {
  return make_int3((int)((k >> 42) & 0x1fffff) - kKeyBias, (int)((k >> 21) & 0x1fffff) - kKeyBias,
                   (int)(k & 0x1fffff) - kKeyBias);
}

// The reference's HashTable home slot (container/HashTable.hpp:493-500 with
// math/Hash.hpp:17-27): 64-bit hash_combine over the three coordinates, truncated to i32,
// then (h % T + T) % T.
__host__ __device__ __forceinline__ int home_slot(int bx, int by, int bz, int table_size) {
  uint64_t seed = (uint64_t)(int64_t)bx;
  seed ^= ((uint64_t)(int64_t)by + 0x9e3779b97f4a7c15ull + (seed << 12) + (seed >> 4));
  seed ^= ((uint64_t)(int64_t)bz + 0x9e3779b97f4a7c15ull + (seed << 12) + (seed >> 4));
  const int h = (int)(uint32_t)seed;
  return (h % table_size + table_size) % table_size;
}

// floor division by the block side for the stencil-origin cell, written as the reference
// does in ComputeSparsity (SparsityOp.hpp:75-77)
__host__ __device__ __forceinline__ int block_of_cell(int c) { return (c + (c < 0 ? -7 : 0)) / 8; }

// ---------------------------------------------------------------- small matrix helpers
struct mat3 {
  float m[9];  // column-major, m[3*c + r]
};

// ---------------------------------------------------------------- 3x3 SVD
// McAdams et al. 2011 ("Computing the singular value decomposition of 3x3 matrices with
// minimal branching and elementary floating point operations"), the algorithm of the
// reference's math::svd_3d (math/matrix/SVD.hpp:15-1025): four sweeps of approximate
// Givens Jacobi conjugations of A^T A accumulated as a quaternion, column sort with sign
// fix, Givens QR.  Same steps and constants; the reciprocal square roots use the SFU
// (rsqrtf), as the reference's CUDA build does with __frsqrt_rn.
namespace svd_detail {
constexpr float kTiny = 1.e-20f;
constexpr float kSmall = 1.e-12f;
constexpr float kFourGammaSq = 5.8284273147583007813f;
__device__ __forceinline__ float sin_pi8() { return __int_as_float(1053028117); }
__device__ __forceinline__ float cos_pi8() { return __int_as_float(1064076127); }

__device__ __forceinline__ void conjugate(float &pp, float &qq, float &rr, float &pq, float &rp,
                                          float &rq, float &qs, float &qk, float &qi,
                                          float &qj) {
  float sh = pq * 0.5f;
  float t5 = pp - qq;
  const bool big = sh * sh >= kTiny;
  sh = big ? sh : 0.f;
  float ch = big ? t5 : 1.f;
  float sh2 = sh * sh, ch2 = ch * ch;
  const float r = rsqrtf(sh2 + ch2);
  sh *= r;
  ch *= r;
  if (ch2 <= kFourGammaSq * sh2) {
    sh = sin_pi8();
    ch = cos_pi8();
  }
  sh2 = sh * sh;
  ch2 = ch * ch;
  const float c = ch2 - sh2;
  const float s = 2.f * ch * sh;
  const float scale = sh2 + ch2;
  rr = rr * scale * scale;
  rp *= scale;
  rq *= scale;
  const float rp0 = rp, rq0 = rq;
  rp = c * rp0 + s * rq0;
  rq = c * rq0 - s * rp0;
  const float s2 = s * s, c2 = c * c;
  const float pp0 = pp, qq0 = qq, pq0 = pq;
  const float cs = c * s;
  const float two_pq_cs = 2.f * pq0 * cs;
  pp = pp0 * c2 + qq0 * s2 + two_pq_cs;
  qq = qq0 * c2 + pp0 * s2 - two_pq_cs;
  pq = pq0 * (c2 - s2) - t5 * cs;
  const float a = sh * qi, b = sh * qj, k = sh * qk, w = sh * qs;
  qs = ch * qs - k;
  qk = ch * qk + w;
  qi = ch * qi + b;
  qj = ch * qj - a;
}

__device__ __forceinline__ float refined_rsqrt(float x) {
  const float y = rsqrtf(x);
  return y + 0.5f * y - x * (0.5f * y * y * y);
}

__device__ __forceinline__ void givens_qr(float a[3][3], float u[3][3], int p, int q, int col) {
  const float apc = a[p][col], aqc = a[q][col];
  float sh = (aqc * aqc >= kSmall) ? aqc : 0.f;
  float ch = fmaxf(fmaxf(-apc, apc), kSmall);
  const bool pos = apc >= 0.f;
  {
    const float n2 = ch * ch + sh * sh;
    ch = ch + refined_rsqrt(n2) * n2;
  }
  if (!pos) {
    const float t = ch;
    ch = sh;
    sh = t;
  }
  {
    const float r = refined_rsqrt(ch * ch + sh * sh);
    ch *= r;
    sh *= r;
  }
  const float c = ch * ch - sh * sh;
  const float s = 2.f * sh * ch;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float x1 = a[p][k], x2 = a[q][k];
    a[p][k] = c * x1 + s * x2;
    a[q][k] = c * x2 - s * x1;
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const float x1 = u[r][p], x2 = u[r][q];
    u[r][p] = c * x1 + s * x2;
    u[r][q] = c * x2 - s * x1;
  }
}

__device__ __forceinline__ void swap_cols(float a[3][3], float v[3][3], float rho[3], int i, int j,
                                          int neg) {
  if (rho[i] < rho[j]) {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      float t = a[r][i];
      a[r][i] = a[r][j];
      a[r][j] = t;
      t = v[r][i];
      v[r][i] = v[r][j];
      v[r][j] = t;
    }
    const float t = rho[i];
    rho[i] = rho[j];
    rho[j] = t;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      a[r][neg] = -a[r][neg];
      v[r][neg] = -v[r][neg];
    }
  }
}
}  // namespace svd_detail

// A (column-major) = U diag(S) V^T; U, V rotations; S sorted by magnitude, S[2] may be < 0.
// kWarpEarlyExit: stop the Jacobi sweeps after the second or third once, for every lane of the
// warp, the off-diagonal of A^T A is below 1e-7 of its diagonal (squared: 1e-14), where the
// remaining sweeps only move the result by rounding.  Every lane of the warp must call it then.
// The default runs the reference's four sweeps.
template <bool kWarpEarlyExit = false>
__device__ __forceinline__ void svd3(const float *A, float *U, float *S, float *V) {
  using namespace svd_detail;
  float a[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) a[r][c] = A[3 * c + r];
  float s11 = a[0][0] * a[0][0] + a[1][0] * a[1][0] + a[2][0] * a[2][0];
  float s21 = a[0][1] * a[0][0] + a[1][1] * a[1][0] + a[2][1] * a[2][0];
  float s31 = a[0][2] * a[0][0] + a[1][2] * a[1][0] + a[2][2] * a[2][0];
  float s22 = a[0][1] * a[0][1] + a[1][1] * a[1][1] + a[2][1] * a[2][1];
  float s32 = a[0][2] * a[0][1] + a[1][2] * a[1][1] + a[2][2] * a[2][1];
  float s33 = a[0][2] * a[0][2] + a[1][2] * a[1][2] + a[2][2] * a[2][2];
  float qs = 1.f, qx = 0.f, qy = 0.f, qz = 0.f;
#pragma unroll
  for (int sweep = 0; sweep < 4; ++sweep) {
    if (kWarpEarlyExit && sweep >= 2) {
      const float off = s21 * s21 + s31 * s31 + s32 * s32;
      const float diag = s11 * s11 + s22 * s22 + s33 * s33;
      if (__all_sync(0xffffffffu, off <= 1e-14f * diag)) break;
    }
    conjugate(s11, s22, s33, s21, s31, s32, qs, qz, qx, qy);
    conjugate(s22, s33, s11, s32, s21, s31, qs, qx, qy, qz);
    conjugate(s33, s11, s22, s31, s32, s21, qs, qy, qz, qx);
  }
  {
    const float r = refined_rsqrt(qs * qs + qx * qx + qy * qy + qz * qz);
    qs *= r;
    qx *= r;
    qy *= r;
    qz *= r;
  }
  float v[3][3];
  {
    const float xx = qx * qx, yy = qy * qy, zz = qz * qz, ww = qs * qs;
    v[0][0] = ww + xx - yy - zz;
    v[1][1] = ww - xx + yy - zz;
    v[2][2] = ww - xx - yy + zz;
    const float x2 = qx + qx, y2 = qy + qy, z2 = qz + qz;
    const float wx = qs * x2, wy = qs * y2, wz = qs * z2;
    const float xy = qy * x2, yz = qz * y2, zx = qx * z2;
    v[0][1] = xy - wz;
    v[1][2] = yz - wx;
    v[2][0] = zx - wy;
    v[1][0] = xy + wz;
    v[2][1] = yz + wx;
    v[0][2] = zx + wy;
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const float a0 = a[r][0], a1 = a[r][1], a2 = a[r][2];
    a[r][0] = v[0][0] * a0 + v[1][0] * a1 + v[2][0] * a2;
    a[r][1] = v[0][1] * a0 + v[1][1] * a1 + v[2][1] * a2;
    a[r][2] = v[0][2] * a0 + v[1][2] * a1 + v[2][2] * a2;
  }
  float rho[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) rho[c] = a[0][c] * a[0][c] + a[1][c] * a[1][c] + a[2][c] * a[2][c];
  swap_cols(a, v, rho, 0, 1, 1);
  swap_cols(a, v, rho, 0, 2, 0);
  swap_cols(a, v, rho, 1, 2, 2);
  float u[3][3] = {{1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f}};
  givens_qr(a, u, 0, 1, 0);
  givens_qr(a, u, 0, 2, 0);
  givens_qr(a, u, 1, 2, 1);
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      U[3 * c + r] = u[r][c];
      V[3 * c + r] = v[r][c];
    }
  S[0] = a[0][0];
  S[1] = a[1][1];
  S[2] = a[2][2];
}

// ---------------------------------------------------------------- constitutive models
struct material_dev {
  int model;            // 0 FC, 1 DP, 2 snow
  int mode;             // 0 committed, 1 reference ordering
  int volume_correction;
  float mu, lambda, volume;
  float cohesion, beta, yield_surface;
  float hardening, theta_c, theta_s;
  float friction_deg;   // Drucker-Prager friction angle (a feature of the learned closure)
};

// Collider<AnalyticLevelSet<shape, f32, 3>> (geometry/Collider.h:10-200); the same layout as
// zsmpm_collider
struct collider_dev {
  int shape, type, axis, reserved;
  float a[3], b[3];
  float s, dsdt;
  float R[9];  // row-major
  float omega[3], t[3], dtdt[3];
};
constexpr int kMaxColliders = 16;

// The boundary code below spells every float operation with a round-to-nearest intrinsic, in
// the reference's order of operations: the finite-difference normals divide differences of
// nearby distances by 2e-6, which amplifies any change of rounding (such as a contraction to
// FMA) about a thousandfold, so the device keeps the reference's rounding exactly.
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rn_div(float a, float b) { return __fdiv_rn(a, b); }
// sum_i a[i] b[i] accumulated from 0 in index order (VecInterface dot / l2NormSqr)
__device__ __forceinline__ float rn_dot3(float a0, float b0, float a1, float b1, float a2, float b2) {
  return rn_add(rn_add(rn_add(0.f, rn_mul(a0, b0)), rn_mul(a1, b1)), rn_mul(a2, b2));
}

// signed distance of the analytic level sets (geometry/AnalyticLevelSet.h)
__device__ __forceinline__ float collider_sdf(const collider_dev &c, const float X[3]) {
  if (c.shape == 0)  // Plane: n . (x - origin)
    return rn_dot3(c.b[0], rn_sub(X[0], c.a[0]), c.b[1], rn_sub(X[1], c.a[1]), c.b[2], rn_sub(X[2], c.a[2]));
  if (c.shape == 1) {  // Cuboid
    float p[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const float center = rn_div(rn_add(c.a[i], c.b[i]), 2.f);
      const float d = rn_sub(X[i], center);
      p[i] = rn_sub(d > 0.f ? d : -d, rn_div(rn_sub(c.b[i], c.a[i]), 2.f));
    }
    float mx = p[0];
    if (p[1] > mx) mx = p[1];
    if (p[2] > mx) mx = p[2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
      if (p[i] < 0.f) p[i] = 0.f;
    return rn_add(mx < 0.f ? mx : 0.f, __fsqrt_rn(rn_dot3(p[0], p[0], p[1], p[1], p[2], p[2])));
  }
  if (c.shape == 2) {  // Sphere: |x - c| - r
    const float d0 = rn_sub(X[0], c.a[0]), d1 = rn_sub(X[1], c.a[1]), d2 = rn_sub(X[2], c.a[2]);
    return rn_sub(__fsqrt_rn(rn_dot3(d0, d0, d1, d1, d2, d2)), c.b[0]);
  }
  // Cylinder along axis d from a, radius b[0], length b[1]
  const int d = c.axis;
  float dr[2];
#pragma unroll
  for (int k = 0, i = 0; k < 3; ++k)
    if (k != d) dr[i++] = rn_sub(X[k], c.a[k]);
  const float dis_r = __fsqrt_rn(rn_add(rn_add(0.f, rn_mul(dr[0], dr[0])), rn_mul(dr[1], dr[1])));
  const float radius = c.b[0], length = c.b[1];
  const bool outside = dis_r > radius;
  const float xd = X[d], bd = c.a[d];
  const float top = rn_add(bd, length);
  if (xd < bd || xd > top) {
    const float dis_l = xd < bd ? rn_sub(bd, xd) : rn_sub(xd, top);
    if (!outside) return dis_l;
    const float e = rn_sub(dis_r, radius);
    return __fsqrt_rn(rn_add(rn_mul(e, e), rn_mul(dis_l, dis_l)));
  }
  if (outside) return rn_sub(dis_r, radius);
  const float up = rn_sub(top, xd), down = rn_sub(xd, bd);
  const float dis_l = up < down ? up : down;
  const float rr = rn_sub(radius, dis_r);
  return -(dis_l < rr ? dis_l : rr);
}

// n / |n| (VecInterface::normalized)
__device__ __forceinline__ void rn_normalize(float n[3]) {
  const float len = __fsqrt_rn(rn_dot3(n[0], n[0], n[1], n[1], n[2], n[2]));
#pragma unroll
  for (int i = 0; i < 3; ++i) n[i] = rn_div(n[i], len);
}

// material-space normal: the plane's normal as given, the sphere's outward direction (zero
// within 1e-7 of the center), a central difference with eps = 1e-6 for cuboid and cylinder
__device__ __forceinline__ void collider_normal(const collider_dev &c, const float X[3], float n[3]) {
  if (c.shape == 0) {
#pragma unroll
    for (int i = 0; i < 3; ++i) n[i] = c.b[i];
    return;
  }
  if (c.shape == 2) {
#pragma unroll
    for (int i = 0; i < 3; ++i) n[i] = rn_sub(X[i], c.a[i]);
    if (rn_dot3(n[0], n[0], n[1], n[1], n[2], n[2]) < 1e-7f) {
      n[0] = n[1] = n[2] = 0.f;
      return;
    }
    rn_normalize(n);
    return;
  }
  const float eps = 1e-6f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float v1[3] = {X[0], X[1], X[2]}, v2[3] = {X[0], X[1], X[2]};
    v1[i] = rn_add(X[i], eps);
    v2[i] = rn_sub(X[i], eps);
    n[i] = rn_div(rn_sub(collider_sdf(c, v1), collider_sdf(c, v2)), rn_add(eps, eps));
  }
  rn_normalize(n);
}

// the velocity response shared by the colliders and the level sets (Collider.h:95-108): v_object
// for sticky, otherwise the relative velocity loses its normal part (slip, or separate when
// moving into the boundary)
__device__ __forceinline__ void boundary_respond(int type, const float n[3], const float vo[3], float v[3]) {
  if (type == 0) {
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = vo[i];
    return;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) v[i] = rn_sub(v[i], vo[i]);
  const float proj = rn_dot3(n[0], v[0], n[1], v[1], n[2], v[2]);
  if ((type == 2 && proj < 0.f) || type == 1)
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = rn_sub(v[i], rn_mul(proj, n[i]));
#pragma unroll
  for (int i = 0; i < 3; ++i) v[i] = rn_add(v[i], vo[i]);
}

// Collider::resolveCollision (Collider.h:80-110) with erosion 0
__device__ __forceinline__ void collider_resolve(const collider_dev &c, const float x[3], float v[3]) {
  const float xb[3] = {rn_sub(x[0], c.t[0]), rn_sub(x[1], c.t[1]), rn_sub(x[2], c.t[2])};
  const float inv_s = rn_div(1.f, c.s);
  float X[3];
#pragma unroll
  for (int i = 0; i < 3; ++i)  // R^T (x - b) / s
    X[i] = rn_mul(rn_dot3(c.R[i], xb[0], c.R[3 + i], xb[1], c.R[6 + i], xb[2]), inv_s);
  if (!(collider_sdf(c, X) < -0.f)) return;
  const float ds = rn_mul(c.dsdt, inv_s);
  // omega x (x - b) + (dsdt / s)(x - b) + R s V(X) + db/dt, V = 0 for an analytic level set
  const float cr[3] = {rn_sub(rn_mul(c.omega[1], xb[2]), rn_mul(c.omega[2], xb[1])),
                       rn_sub(rn_mul(c.omega[2], xb[0]), rn_mul(c.omega[0], xb[2])),
                       rn_sub(rn_mul(c.omega[0], xb[1]), rn_mul(c.omega[1], xb[0]))};
  float vo[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) vo[i] = rn_add(rn_add(rn_add(cr[i], rn_mul(ds, xb[i])), 0.f), c.dtdt[i]);
  float nX[3] = {0.f, 0.f, 0.f}, n[3] = {0.f, 0.f, 0.f};
  if (c.type != 0) {
    collider_normal(c, X, nX);
#pragma unroll
    for (int i = 0; i < 3; ++i) n[i] = rn_dot3(c.R[3 * i], nX[0], c.R[3 * i + 1], nX[1], c.R[3 * i + 2], nX[2]);
  }
  boundary_respond(c.type, n, vo, v);
}

// LevelSetBoundary<SparseLevelSet<3>>: 8^3 blocks of signed distance found through a dense map
// over the keys' bounding box (block coordinates lo .. lo + dim - 1)
struct levelset_dev {
  int type, nblocks;
  int lo[3], dim[3];
  const int *map;    // dim[0] * dim[1] * dim[2]: block index or -1
  const float *sdf;  // nblocks * 512
  float background;
  float sinv[9], rinv[9], t[3];  // row-major
};
constexpr int kMaxLevelsets = 4;

// SparseLevelSetView::value_or (SparseLevelSet.hpp:477-484) at an integer index coordinate
__device__ __forceinline__ float levelset_node(const levelset_dev &L, int cx, int cy, int cz) {
  const int lx = cx & 7, ly = cy & 7, lz = cz & 7;
  const int ix = ((cx - lx) >> 3) - L.lo[0], iy = ((cy - ly) >> 3) - L.lo[1], iz = ((cz - lz) >> 3) - L.lo[2];
  if (ix < 0 || iy < 0 || iz < 0 || ix >= L.dim[0] || iy >= L.dim[1] || iz >= L.dim[2]) return L.background;
  const int b = L.map[((size_t)ix * L.dim[1] + iy) * L.dim[2] + iz];
  return b < 0 ? L.background : L.sdf[(size_t)b * 512 + ((lx << 6) | (ly << 3) | lz)];
}

// linear_interop(t, a, b) = a + (b - a) t (ZpcMathUtils.hpp:1779-1781)
__device__ __forceinline__ float lerp_ref(float t, float a, float b) { return rn_add(a, rn_mul(rn_sub(b, a), t)); }

// getSignedDistance: worldToIndex (SparseLevelSet.hpp:366-374), then the linear LevelSetArena
// (:862-875, base_node<0> = floor) and xlerp (math/VecInterface.hpp:1043-1049)
__device__ __forceinline__ float levelset_sdf(const levelset_dev &L, const float x[3]) {
  const float a[3] = {rn_sub(x[0], L.t[0]), rn_sub(x[1], L.t[1]), rn_sub(x[2], L.t[2])};
  float b[3], X[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) b[j] = rn_dot3(L.rinv[j], a[0], L.rinv[3 + j], a[1], L.rinv[6 + j], a[2]);
#pragma unroll
  for (int j = 0; j < 3; ++j) X[j] = rn_dot3(L.sinv[j], b[0], L.sinv[3 + j], b[1], L.sinv[6 + j], b[2]);
  int c[3];
  float d[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    c[k] = (int)floorf(X[k]);
    d[k] = rn_sub(X[k], (float)c[k]);
  }
  float p[2][2][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < 2; ++k) p[i][j][k] = levelset_node(L, c[0] + i, c[1] + j, c[2] + k);
  return lerp_ref(d[0], lerp_ref(d[1], lerp_ref(d[2], p[0][0][0], p[0][0][1]), lerp_ref(d[2], p[0][1][0], p[0][1][1])),
                  lerp_ref(d[1], lerp_ref(d[2], p[1][0][0], p[1][0][1]), lerp_ref(d[2], p[1][1][0], p[1][1][1])));
}

// Collider{levelset view, type}.resolveCollision with the identity placement (Collider.h:80-110):
// the level set carries no material velocity here, so the collider's velocity is zero
__device__ __forceinline__ void levelset_resolve(const levelset_dev &L, const float x[3], float v[3]) {
  if (!(levelset_sdf(L, x) < -0.f)) return;
  const float vo[3] = {0.f, 0.f, 0.f};
  float n[3] = {0.f, 0.f, 0.f};
  if (L.type != 0) {
    const float eps = 1e-6f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float v1[3] = {x[0], x[1], x[2]}, v2[3] = {x[0], x[1], x[2]};
      v1[i] = rn_add(x[i], eps);
      v2[i] = rn_sub(x[i], eps);
      n[i] = rn_div(rn_sub(levelset_sdf(L, v1), levelset_sdf(L, v2)), rn_add(eps, eps));
    }
    rn_normalize(n);
  }
  boundary_respond(L.type, n, vo, v);
}

// out[3c+r] = sum_k M[3k+r] d[k] N[3k+c]
__device__ __forceinline__ void mul_diag_t(float *out, const float *M, const float *d,
                                           const float *N) {
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r)
      out[3 * c + r] = M[r] * d[0] * N[c] + M[3 + r] * d[1] * N[3 + c] + M[6 + r] * d[2] * N[6 + c];
}

// Kirchhoff stress tau = V0 P F^T for an isotropic model with F = U diag(S) V^T and
// principal first Piola stress Ph: P F^T = U diag(Ph * S) U^T.
__device__ __forceinline__ void kirchhoff(float *tau, const float *U, const float *Ph,
                                          const float *S, float volume) {
  const float d[3] = {Ph[0] * S[0] * volume, Ph[1] * S[1] * volume, Ph[2] * S[2] * volume};
  mul_diag_t(tau, U, d, U);
}

// Fixed corotated principal stress (ConstitutiveModel_Vol_dP.hpp:17-23)
__device__ __forceinline__ void fc_principal(float mu, float lambda, const float *S, float *Ph) {
  const float J = S[0] * S[1] * S[2];
  const float smu = 2.f * mu, sl = lambda * (J - 1.f);
  Ph[0] = smu * (S[0] - 1.f) + sl * (S[1] * S[2]);
  Ph[1] = smu * (S[1] - 1.f) + sl * (S[0] * S[2]);
  Ph[2] = smu * (S[2] - 1.f) + sl * (S[0] * S[1]);
}

// Return map + stress.  F: trial deformation in, F after the model's projection out
// (the projected F is what the reference's stress functions leave in their F argument);
// plastic: logJp (DP) or Jp (snow); tau out.  Reference ordering keeps F unchanged.
template <bool kWarpEarlyExit = false>
__device__ __forceinline__ void constitutive(const material_dev &mat, float *F, float &plastic,
                                             float *tau) {
  float U[9], S[3], V[9];
  svd3<kWarpEarlyExit>(F, U, S, V);
  if (mat.model == 0) {
    float Ph[3];
    fc_principal(mat.mu, mat.lambda, S, Ph);
    kirchhoff(tau, U, Ph, S, mat.volume);
    return;
  }
  float Ns[3], logNs[3];
  if (mat.model == 1) {
    // compute_stress_sand (ConstitutiveModel_Vol_dP.hpp:241-325)
    float eps[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) eps[i] = logf(fmaxf(fabsf(S[i]), 1e-4f)) - mat.cohesion;
    const float sum_eps = eps[0] + eps[1] + eps[2];
    const float tr = sum_eps + plastic;
    float eh[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) eh[i] = eps[i] - tr / 3.f;
    const float ehn = sqrtf(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2]);
    const float smu = 2.f * mat.mu;
    // the projected log-strain is the exponent itself; the reference takes log(exp(H)),
    // which differs from H only by the rounding of expf and logf
    if (tr >= 0.f) {
      const float e = expf(mat.cohesion);
      Ns[0] = Ns[1] = Ns[2] = e;
      logNs[0] = logNs[1] = logNs[2] = mat.cohesion;
      if (mat.volume_correction) plastic = mat.beta * sum_eps + plastic;
    } else if (mat.mu != 0.f) {
      plastic = 0.f;
      const float dg = ehn + (3.f * mat.lambda + smu) / smu * tr * mat.yield_surface;
      const float f = dg <= 0.f ? 0.f : dg / ehn;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        logNs[i] = eps[i] - f * eh[i] + mat.cohesion;
        Ns[i] = expf(logNs[i]);
      }
    } else {
      Ns[0] = Ns[1] = Ns[2] = 0.f;
      logNs[0] = logNs[1] = logNs[2] = 0.f;
    }
    const float trl = logNs[0] + logNs[1] + logNs[2];
    // P F_new^T = U diag(Ph * Ns) U^T with Ph = (2 mu log Ns + lambda tr log Ns) / Ns
    float PhNs[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) PhNs[i] = (smu * logNs[i] + mat.lambda * trl) * mat.volume;
    mul_diag_t(tau, U, PhNs, U);
  } else {
    // snow: SnowPlasticity::do_project_sigma (SnowPlasticity.hpp:24-32) committed to F,
    // Jp accumulated, then fixed corotated with hardened Lame parameters
    const float J = S[0] * S[1] * S[2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
      Ns[i] = fmaxf(fminf(S[i], 1.f + mat.theta_s), 1.f - mat.theta_c);
    const float Jc = Ns[0] * Ns[1] * Ns[2];
    plastic = plastic * (J / fmaxf(Jc, 1e-6f));
    const float e = expf(mat.hardening * (1.f - plastic));
    float Ph[3];
    fc_principal(mat.mu * e, mat.lambda * e, Ns, Ph);
    kirchhoff(tau, U, Ph, Ns, mat.volume);
  }
  if (mat.mode == 0) mul_diag_t(F, U, Ns, V);
}

// ---------------------------------------------------------------- warp helpers
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// vectorised global reduction of four consecutive floats (16-byte aligned address)
__device__ __forceinline__ void red_add_v4(float *addr, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b),
               "f"(c), "f"(d)
               : "memory");
}

}  // namespace zsmpm
