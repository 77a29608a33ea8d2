/* Test infrastructure (oracle): 3x3 SVDs used by the CPU restatement.
 *
 * oracle_svd_f32 restates math/matrix/SVD.hpp:15-1025 of the reference (the McAdams,
 * Selle, Tamstorf, Teran, Sifakis 2011 algorithm: 4 sweeps of approximate-Givens Jacobi
 * conjugation of A^T A accumulated as a quaternion, column sort with sign fix, Givens QR),
 * keeping every float operation in the reference's order so that it agrees bit for bit
 * with the reference's svd_3d on the host (whose rsqrt is 1/sqrtf, ZpcMathUtils.hpp:842).
 * The three Jacobi conjugations of a sweep are one routine here, parameterised by which
 * entries play the (p, q, r) roles; the reference writes them out three times.
 *
 * oracle_svd_f64 is an independent accurate SVD for the FP64 oracle (cyclic Jacobi with
 * exact rotations to convergence), returning the same conventions: S sorted by
 * decreasing magnitude, U and V proper rotations, the sign carried by S[2].
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

typedef union {
  float f;
  uint32_t u;
} fbits;

static const uint32_t k_one_bits = 1065353216u;     /* 1.0f */
static const uint32_t k_sin_pi8_bits = 1053028117u; /* sin(pi/8) */
static const uint32_t k_cos_pi8_bits = 1064076127u; /* cos(pi/8) */
static const float k_small = 1.e-12f;
static const float k_tiny = 1.e-20f;
static const float k_four_gamma_sq = 5.8284273147583007813f;

static float host_rsqrt(float x) { return 1.f / sqrtf(x); }
static float fmaxf_ref(float a, float b) { return a > b ? a : b; }

/* One approximate-Givens Jacobi conjugation of the symmetric matrix S in the (p,q) plane,
 * r being the remaining index; the rotation is accumulated into quaternion (qs, q[k]),
 * with (qi, qj) the other two vector components in cyclic order after k. */
static void jacobi_conjugate(float *pp, float *qq, float *rr, float *pq, float *rp, float *rq,
                             float *qs, float *qk, float *qi, float *qj) {
  fbits sh, ch, t1, t2, t3, t4, t5, mask;
  float c, s;
  sh.f = *pq * 0.5f;
  t5.f = *pp - *qq;
  t2.f = sh.f * sh.f;
  mask.u = (t2.f >= k_tiny) ? 0xffffffffu : 0u;
  sh.u = mask.u & sh.u;
  ch.u = mask.u & t5.u;
  t2.u = ~mask.u & k_one_bits;
  ch.u = ch.u | t2.u;

  t1.f = sh.f * sh.f;
  t2.f = ch.f * ch.f;
  t3.f = t1.f + t2.f;
  t4.f = host_rsqrt(t3.f);
  sh.f = t4.f * sh.f;
  ch.f = t4.f * ch.f;
  t1.f = k_four_gamma_sq * t1.f;
  mask.u = (t2.f <= t1.f) ? 0xffffffffu : 0u;
  t2.u = k_sin_pi8_bits & mask.u;
  sh.u = ~mask.u & sh.u;
  sh.u = sh.u | t2.u;
  t2.u = k_cos_pi8_bits & mask.u;
  ch.u = ~mask.u & ch.u;
  ch.u = ch.u | t2.u;

  t1.f = sh.f * sh.f;
  t2.f = ch.f * ch.f;
  c = t2.f - t1.f;
  s = ch.f * sh.f;
  s = s + s;

  /* conjugation */
  t3.f = t1.f + t2.f;
  *rr = *rr * t3.f;
  *rp = *rp * t3.f;
  *rq = *rq * t3.f;
  *rr = *rr * t3.f;

  t1.f = s * *rp;
  t2.f = s * *rq;
  *rp = c * *rp;
  *rq = c * *rq;
  *rp = t2.f + *rp;
  *rq = *rq - t1.f;

  t2.f = s * s;
  t1.f = *qq * t2.f;
  t3.f = *pp * t2.f;
  t4.f = c * c;
  *pp = *pp * t4.f;
  *qq = *qq * t4.f;
  *pp = *pp + t1.f;
  *qq = *qq + t3.f;
  t4.f = t4.f - t2.f;
  t2.f = *pq + *pq;
  *pq = *pq * t4.f;
  t4.f = c * s;
  t2.f = t2.f * t4.f;
  t5.f = t5.f * t4.f;
  *pp = *pp + t2.f;
  *pq = *pq - t5.f;
  *qq = *qq - t2.f;

  /* quaternion accumulation */
  {
    float a = sh.f * *qi, b = sh.f * *qj, k = sh.f * *qk, w = sh.f * *qs;
    *qs = ch.f * *qs;
    *qi = ch.f * *qi;
    *qj = ch.f * *qj;
    *qk = ch.f * *qk;
    *qk = *qk + w;
    *qs = *qs - k;
    *qi = *qi + b;
    *qj = *qj - a;
  }
}

/* rsqrt refined by one Newton step, as the reference writes it. */
static float refined_rsqrt(float x) {
  float t1 = host_rsqrt(x), t3, t4;
  t4 = t1 * 0.5f;
  t3 = t1 * t4;
  t3 = t1 * t3;
  t3 = x * t3;
  t1 = t1 + t4;
  t1 = t1 - t3;
  return t1;
}

/* Conditionally swap columns i and j of both A and V (row-major a[r][c], v[r][c]) and the
 * column norms, then negate column `neg` of A and V when swapped. */
static void sort_swap(float a[3][3], float v[3][3], float rho[3], int i, int j, int neg) {
  fbits mask, t5, x, y, f4;
  mask.u = (rho[i] < rho[j]) ? 0xffffffffu : 0u;
  for (int r = 0; r != 3; ++r) {
    x.f = a[r][i];
    y.f = a[r][j];
    t5.u = (x.u ^ y.u) & mask.u;
    x.u ^= t5.u;
    y.u ^= t5.u;
    a[r][i] = x.f;
    a[r][j] = y.f;
  }
  for (int r = 0; r != 3; ++r) {
    x.f = v[r][i];
    y.f = v[r][j];
    t5.u = (x.u ^ y.u) & mask.u;
    x.u ^= t5.u;
    y.u ^= t5.u;
    v[r][i] = x.f;
    v[r][j] = y.f;
  }
  x.f = rho[i];
  y.f = rho[j];
  t5.u = (x.u ^ y.u) & mask.u;
  x.u ^= t5.u;
  y.u ^= t5.u;
  rho[i] = x.f;
  rho[j] = y.f;
  t5.f = -2.f;
  t5.u = t5.u & mask.u;
  f4.f = 1.f;
  f4.f = f4.f + t5.f;
  for (int r = 0; r != 3; ++r) a[r][neg] = a[r][neg] * f4.f;
  for (int r = 0; r != 3; ++r) v[r][neg] = v[r][neg] * f4.f;
}

/* Givens rotation zeroing a[i][col] against a[col][col]... applied to rows (p, q) of A and
 * columns (p, q) of U, with (ch, sh) from the pivot a[p][col] and the entry a[q][col]. */
static void qr_givens(float a[3][3], float u[3][3], int p, int q, int col) {
  fbits sh, ch, t1, t2, t5;
  float c, s, tmp;
  sh.f = a[q][col] * a[q][col];
  sh.u = (sh.f >= k_small) ? 0xffffffffu : 0u;
  {
    fbits aq;
    aq.f = a[q][col];
    sh.u = sh.u & aq.u;
  }
  t5.f = 0.f;
  ch.f = t5.f - a[p][col];
  ch.f = fmaxf_ref(ch.f, a[p][col]);
  ch.f = fmaxf_ref(ch.f, k_small);
  t5.u = (a[p][col] >= t5.f) ? 0xffffffffu : 0u;

  t1.f = ch.f * ch.f;
  t2.f = sh.f * sh.f;
  t2.f = t1.f + t2.f;
  tmp = refined_rsqrt(t2.f);
  t1.f = tmp * t2.f;
  ch.f = ch.f + t1.f;

  t1.u = ~t5.u & sh.u;
  t2.u = ~t5.u & ch.u;
  ch.u = t5.u & ch.u;
  sh.u = t5.u & sh.u;
  ch.u = ch.u | t1.u;
  sh.u = sh.u | t2.u;

  t1.f = ch.f * ch.f;
  t2.f = sh.f * sh.f;
  t2.f = t1.f + t2.f;
  tmp = refined_rsqrt(t2.f);
  ch.f = ch.f * tmp;
  sh.f = sh.f * tmp;
  c = ch.f * ch.f;
  s = sh.f * sh.f;
  c = c - s;
  s = sh.f * ch.f;
  s = s + s;

  for (int k = 0; k != 3; ++k) {
    float x1 = s * a[p][k], x2 = s * a[q][k];
    a[p][k] = c * a[p][k];
    a[q][k] = c * a[q][k];
    a[p][k] = a[p][k] + x2;
    a[q][k] = a[q][k] - x1;
  }
  for (int r = 0; r != 3; ++r) {
    float x1 = s * u[r][p], x2 = s * u[r][q];
    u[r][p] = c * u[r][p];
    u[r][q] = c * u[r][q];
    u[r][p] = u[r][p] + x2;
    u[r][q] = u[r][q] - x1;
  }
}

void oracle_svd_f32(const float *A, float *U, float *S, float *V) {
  float a[3][3], u[3][3], v[3][3];
  for (int r = 0; r != 3; ++r)
    for (int c = 0; c != 3; ++c) a[r][c] = A[3 * c + r];

  /* normal equations S = A^T A (lower triangle), each entry summed over rows 1,2,3 */
  float s11, s21, s31, s22, s32, s33, t;
  s11 = a[0][0] * a[0][0];
  t = a[1][0] * a[1][0];
  s11 = t + s11;
  t = a[2][0] * a[2][0];
  s11 = t + s11;
  s21 = a[0][1] * a[0][0];
  t = a[1][1] * a[1][0];
  s21 = t + s21;
  t = a[2][1] * a[2][0];
  s21 = t + s21;
  s31 = a[0][2] * a[0][0];
  t = a[1][2] * a[1][0];
  s31 = t + s31;
  t = a[2][2] * a[2][0];
  s31 = t + s31;
  s22 = a[0][1] * a[0][1];
  t = a[1][1] * a[1][1];
  s22 = t + s22;
  t = a[2][1] * a[2][1];
  s22 = t + s22;
  s32 = a[0][2] * a[0][1];
  t = a[1][2] * a[1][1];
  s32 = t + s32;
  t = a[2][2] * a[2][1];
  s32 = t + s32;
  s33 = a[0][2] * a[0][2];
  t = a[1][2] * a[1][2];
  s33 = t + s33;
  t = a[2][2] * a[2][2];
  s33 = t + s33;

  float qs = 1.f, qx = 0.f, qy = 0.f, qz = 0.f;
  for (int sweep = 0; sweep != 4; ++sweep) {
    jacobi_conjugate(&s11, &s22, &s33, &s21, &s31, &s32, &qs, &qz, &qx, &qy);
    jacobi_conjugate(&s22, &s33, &s11, &s32, &s21, &s31, &qs, &qx, &qy, &qz);
    jacobi_conjugate(&s33, &s11, &s22, &s31, &s32, &s21, &qs, &qy, &qz, &qx);
  }

  /* normalise quaternion */
  {
    float n2 = qs * qs, t1;
    t1 = qx * qx;
    n2 = t1 + n2;
    t1 = qy * qy;
    n2 = t1 + n2;
    t1 = qz * qz;
    n2 = t1 + n2;
    t1 = refined_rsqrt(n2);
    qs = qs * t1;
    qx = qx * t1;
    qy = qy * t1;
    qz = qz * t1;
  }
  /* quaternion -> V */
  {
    float t1 = qx * qx, t2 = qy * qy, t3 = qz * qz;
    float v11 = qs * qs, v22, v33, v12, v13, v21, v23, v31, v32;
    v22 = v11 - t1;
    v33 = v22 - t2;
    v33 = v33 + t3;
    v22 = v22 + t2;
    v22 = v22 - t3;
    v11 = v11 + t1;
    v11 = v11 - t2;
    v11 = v11 - t3;
    t1 = qx + qx;
    t2 = qy + qy;
    t3 = qz + qz;
    v32 = qs * t1;
    v13 = qs * t2;
    v21 = qs * t3;
    t1 = qy * t1;
    t2 = qz * t2;
    t3 = qx * t3;
    v12 = t1 - v21;
    v23 = t2 - v32;
    v31 = t3 - v13;
    v21 = t1 + v21;
    v32 = t2 + v32;
    v13 = t3 + v13;
    v[0][0] = v11; v[0][1] = v12; v[0][2] = v13;
    v[1][0] = v21; v[1][1] = v22; v[1][2] = v23;
    v[2][0] = v31; v[2][1] = v32; v[2][2] = v33;
  }
  /* A <- A V, row by row */
  for (int r = 0; r != 3; ++r) {
    float t1, t2 = a[r][1], t3 = a[r][2];
    a[r][1] = v[0][1] * a[r][0];
    a[r][2] = v[0][2] * a[r][0];
    a[r][0] = v[0][0] * a[r][0];
    t1 = v[1][0] * t2;
    a[r][0] = a[r][0] + t1;
    t1 = v[2][0] * t3;
    a[r][0] = a[r][0] + t1;
    t1 = v[1][1] * t2;
    a[r][1] = a[r][1] + t1;
    t1 = v[2][1] * t3;
    a[r][1] = a[r][1] + t1;
    t1 = v[1][2] * t2;
    a[r][2] = a[r][2] + t1;
    t1 = v[2][2] * t3;
    a[r][2] = a[r][2] + t1;
  }
  /* sort columns by norm */
  {
    float rho[3];
    for (int c = 0; c != 3; ++c) {
      float r2 = a[0][c] * a[0][c], t4;
      t4 = a[1][c] * a[1][c];
      r2 = r2 + t4;
      t4 = a[2][c] * a[2][c];
      r2 = r2 + t4;
      rho[c] = r2;
    }
    sort_swap(a, v, rho, 0, 1, 1);
    sort_swap(a, v, rho, 0, 2, 0);
    sort_swap(a, v, rho, 1, 2, 2);
  }
  /* QR by three Givens rotations */
  for (int r = 0; r != 3; ++r)
    for (int c = 0; c != 3; ++c) u[r][c] = (r == c) ? 1.f : 0.f;
  qr_givens(a, u, 0, 1, 0);
  qr_givens(a, u, 0, 2, 0);
  qr_givens(a, u, 1, 2, 1);

  for (int r = 0; r != 3; ++r)
    for (int c = 0; c != 3; ++c) {
      U[3 * c + r] = u[r][c];
      V[3 * c + r] = v[r][c];
    }
  S[0] = a[0][0];
  S[1] = a[1][1];
  S[2] = a[2][2];
}

/* ------------------------------------------------- the reference's float square root */
/* zs::math::sqrt(float) (math/MathUtils.h:258-326): a bit-trick reciprocal square root
 * (Lomont's constant 0x5f375a86, two Newton steps), two more Newton steps on the scaled
 * argument, one correction step, then rescaling.  compute_stress_sand uses it for the norm
 * of the deviatoric log strain (ConstitutiveModel_Vol_dP.hpp:263-265). */
static float ref_q_rsqrt(float number) {
  fbits b;
  float x2 = number * 0.5f, y;
  b.f = number;
  b.u = 0x5f375a86u - (b.u >> 1);
  y = b.f;
  y = y * (1.5f - (x2 * y * y));
  y = y * (1.5f - (x2 * y * y));
  return y;
}

float oracle_ref_sqrtf(float arg) {
  const float scale_in = 0x1.0p+26f, scale_out = 0x1.0p-13f;
  fbits inf;
  inf.u = 0x7f800000u;
  if (arg < 0.0f) {
    fbits q;
    q.u = 0x7fffffffu;
    return q.f;
  } else if (arg == 0.0f || !(fabsf(arg) < inf.f)) {
    return arg + arg;
  }
  arg = arg * scale_in;
  float rsq = ref_q_rsqrt(arg);
  rsq = ((-0.5f * arg * rsq) * rsq + 0.5f) * rsq + rsq;
  rsq = ((-0.5f * arg * rsq) * rsq + 0.5f) * rsq + rsq;
  float sqt = rsq * arg;
  float err = sqt * -sqt + arg;
  sqt = (0.5f * rsq * err + sqt);
  return sqt * scale_out;
}

/* ---------------------------------------------------------------- FP64 SVD */

static double det3d(const double m[3][3]) {
  return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
         m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
         m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

void oracle_svd_f64(const double *A, double *U, double *S, double *V) {
  double a[3][3], s[3][3], v[3][3];
  for (int r = 0; r != 3; ++r)
    for (int c = 0; c != 3; ++c) a[r][c] = A[3 * c + r];
  for (int i = 0; i != 3; ++i)
    for (int j = 0; j != 3; ++j) {
      double acc = 0;
      for (int k = 0; k != 3; ++k) acc += a[k][i] * a[k][j];
      s[i][j] = acc;
      v[i][j] = i == j;
    }
  /* cyclic Jacobi eigen-decomposition of s with exact rotations */
  for (int sweep = 0; sweep != 50; ++sweep) {
    double off = fabs(s[0][1]) + fabs(s[0][2]) + fabs(s[1][2]);
    double scale = fabs(s[0][0]) + fabs(s[1][1]) + fabs(s[2][2]);
    if (off <= 1e-300 || off <= 1e-17 * scale) break;
    for (int p = 0; p != 2; ++p)
      for (int q = p + 1; q != 3; ++q) {
        if (s[p][q] == 0.0) continue;
        double theta = (s[q][q] - s[p][p]) / (2 * s[p][q]);
        double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
        double c = 1 / sqrt(tt * tt + 1), sn = tt * c;
        for (int k = 0; k != 3; ++k) {
          double skp = s[k][p], skq = s[k][q];
          s[k][p] = c * skp - sn * skq;
          s[k][q] = sn * skp + c * skq;
        }
        for (int k = 0; k != 3; ++k) {
          double spk = s[p][k], sqk = s[q][k];
          s[p][k] = c * spk - sn * sqk;
          s[q][k] = sn * spk + c * sqk;
        }
        for (int k = 0; k != 3; ++k) {
          double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - sn * vkq;
          v[k][q] = sn * vkp + c * vkq;
        }
      }
  }
  /* sort eigenpairs by decreasing eigenvalue */
  double ev[3] = {s[0][0], s[1][1], s[2][2]};
  int idx[3] = {0, 1, 2};
  for (int i = 0; i != 3; ++i)
    for (int j = i + 1; j != 3; ++j)
      if (ev[idx[j]] > ev[idx[i]]) {
        int t = idx[i];
        idx[i] = idx[j];
        idx[j] = t;
      }
  double vs[3][3];
  for (int r = 0; r != 3; ++r)
    for (int c = 0; c != 3; ++c) vs[r][c] = v[r][idx[c]];
  if (det3d(vs) < 0)
    for (int r = 0; r != 3; ++r) vs[r][2] = -vs[r][2];
  /* B = A V; U columns from normalised B columns, third by cross product */
  double b[3][3], u[3][3], sig[3];
  for (int r = 0; r != 3; ++r)
    for (int c = 0; c != 3; ++c) {
      double acc = 0;
      for (int k = 0; k != 3; ++k) acc += a[r][k] * vs[k][c];
      b[r][c] = acc;
    }
  for (int c = 0; c != 2; ++c) {
    double nrm = sqrt(b[0][c] * b[0][c] + b[1][c] * b[1][c] + b[2][c] * b[2][c]);
    sig[c] = nrm;
    for (int r = 0; r != 3; ++r) u[r][c] = nrm > 0 ? b[r][c] / nrm : (r == c);
  }
  /* re-orthogonalise the second column against the first */
  {
    double d = u[0][0] * u[0][1] + u[1][0] * u[1][1] + u[2][0] * u[2][1];
    for (int r = 0; r != 3; ++r) u[r][1] -= d * u[r][0];
    double nrm = sqrt(u[0][1] * u[0][1] + u[1][1] * u[1][1] + u[2][1] * u[2][1]);
    for (int r = 0; r != 3; ++r) u[r][1] /= nrm;
  }
  u[0][2] = u[1][0] * u[2][1] - u[2][0] * u[1][1];
  u[1][2] = u[2][0] * u[0][1] - u[0][0] * u[2][1];
  u[2][2] = u[0][0] * u[1][1] - u[1][0] * u[0][1];
  sig[2] = b[0][2] * u[0][2] + b[1][2] * u[1][2] + b[2][2] * u[2][2];
  for (int r = 0; r != 3; ++r)
    for (int c = 0; c != 3; ++c) {
      U[3 * c + r] = u[r][c];
      V[3 * c + r] = vs[r][c];
    }
  S[0] = sig[0];
  S[1] = sig[1];
  S[2] = sig[2];
}
