// Learned return-mapping closure: the principal-space return maps it learns, its parameter
// layout, and its BF16 tensor-core inference for one warp of 32 particles.
//
// The network maps (l1, l2, l3, a, b, s) -- the three log singular values of the trial F
// (|S| clamped at 1e-4, sorted descending as the SVD returns them) and three material/state
// features -- to (D1, D2, D3, t1, t2, t3): D = projected log strain minus the trial log
// strain (zero in the elastic region) and t = principal Kirchhoff stress, both scaled.
//   Drucker-Prager: a = friction angle (deg), b = cohesion (log-strain shift), s = logJp
//   snow:           a = theta_c, b = theta_s, s = log Jp
// Layers 6 -> 64 -> 64 -> 64 -> 6 with SiLU on the hidden layers.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "zsmpm_device.cuh"

namespace zsmpm {

constexpr int kMlpIn = 6, kMlpHidden = 64, kMlpOut = 6;
// FP32 master parameter offsets (row-major W[out][in], then bias)
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kMlpHidden * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHidden, kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden, kOffB3 = kOffW3 + kMlpHidden * kMlpHidden;
constexpr int kOffW4 = kOffB3 + kMlpHidden, kOffB4 = kOffW4 + kMlpOut * kMlpHidden;
constexpr int kMlpParams = kOffB4 + kMlpOut;  // 9158

// BF16 B-operand fragments of mma.m16n8k16 (one uint2 per lane per (k-slice, n-tile)):
// layer 1 K=16 (6 padded) N=64, layers 2-3 K=64 N=64, layer 4 K=64 N=8 (6 padded)
constexpr int kFragL1 = 1 * 8 * 32, kFragL2 = 4 * 8 * 32, kFragL3 = 4 * 8 * 32, kFragL4 = 4 * 1 * 32;
constexpr int kFragOff1 = 0, kFragOff2 = kFragOff1 + kFragL1, kFragOff3 = kFragOff2 + kFragL2,
              kFragOff4 = kFragOff3 + kFragL3, kFragTotal = kFragOff4 + kFragL4;  // 2432 uint2
constexpr int kBiasTotal = 64 + 64 + 64 + 8;                                          // padded biases

// Normalisation and hull of the trained network, passed by value to kernels.
struct closure_dev {
  int model;                 // 1 Drucker-Prager, 2 snow
  int audit_period;          // audit one particle in audit_period (0 = no audit)
  float kappa;               // 3 lambda + 2 mu of the material (the stress unit)
  float hardening;           // snow hardening coefficient xi
  float in_mean[kMlpIn], in_inv_std[kMlpIn];  // of the network inputs (closure_inputs)
  float in_min[kMlpIn], in_max[kMlpIn];  // axis-aligned training hull (raw features)
  float out_scale[kMlpOut];  // of the network targets (closure_net_targets)
  const uint2 *frag;         // kFragTotal BF16 weight fragments
  const float *bias;         // kBiasTotal
  const uint4 *umma_w;       // the weights in the tcgen05 shared-memory layout
  int *tc_status;            // bounded-wait failures of the tcgen05 inference
  double *audit;             // [audited, sum rel err, max rel err, sum |dtau|^2, sum |tau|^2, fallbacks,
                             //  network updates, all updates]
};

// ---------------------------------------------------------------- principal return maps
struct principal_result {
  float H[3];      // projected log strain
  float tau[3];    // principal Kirchhoff stress (without the particle volume)
  float plastic;   // updated plastic state (logJp or Jp)
  float Ns[3];     // projected singular values
};

// Drucker-Prager (compute_stress_sand, ConstitutiveModel_Vol_dP.hpp:241-325) in principal
// space from l = log(max(|S|, 1e-4)); the same arithmetic as the plain constitutive update.
__device__ __forceinline__ principal_result dp_principal(float mu, float lambda, float cohesion,
                                                         float beta, int vc, float ys,
                                                         const float l[3], float logJp) {
  principal_result r;
  float eps[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) eps[i] = l[i] - cohesion;
  const float sum_eps = eps[0] + eps[1] + eps[2];
  const float tr = sum_eps + logJp;
  float eh[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) eh[i] = eps[i] - tr / 3.f;
  const float ehn = sqrtf(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2]);
  const float smu = 2.f * mu;
  r.plastic = logJp;
  if (tr >= 0.f) {
#pragma unroll
    for (int i = 0; i < 3; ++i) r.H[i] = cohesion;
    if (vc) r.plastic = beta * sum_eps + logJp;
  } else {
    r.plastic = 0.f;
    const float dg = ehn + (3.f * lambda + smu) / smu * tr * ys;
    const float f = dg <= 0.f ? 0.f : dg / ehn;
#pragma unroll
    for (int i = 0; i < 3; ++i) r.H[i] = eps[i] - f * eh[i] + cohesion;
  }
  const float trl = r.H[0] + r.H[1] + r.H[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r.tau[i] = smu * r.H[i] + lambda * trl;
    r.Ns[i] = expf(r.H[i]);
  }
  return r;
}

// Snow (SnowPlasticity.hpp:24-32 with Jp accumulated, fixed corotated hardened stress) in
// principal space from the signed singular values S of the trial F.
__device__ __forceinline__ principal_result snow_principal(float mu, float lambda, float hardening,
                                                           float theta_c, float theta_s,
                                                           const float S[3], float Jp) {
  principal_result r;
  const float J = S[0] * S[1] * S[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) r.Ns[i] = fmaxf(fminf(S[i], 1.f + theta_s), 1.f - theta_c);
  const float Jc = r.Ns[0] * r.Ns[1] * r.Ns[2];
  r.plastic = Jp * (J / fmaxf(Jc, 1e-6f));
  const float e = expf(hardening * (1.f - r.plastic));
  float Ph[3];
  fc_principal(mu * e, lambda * e, r.Ns, Ph);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r.tau[i] = Ph[i] * r.Ns[i];
    r.H[i] = logf(r.Ns[i]);
  }
  return r;
}

// ---------------------------------------------------------------- network inputs/outputs
// Raw feature rows (what the hull, the training set and the state log hold) are mapped to the
// network's inputs, and its outputs o back to D = sD o[0..2], tau = off + sT o[3..5].
//
// Drucker-Prager: with eps = l - c and s = |(eps, logJp)|, the return map is positively
// homogeneous of degree one in (eps, logJp): H - c and tau - kappa c scale with s (the cone's
// apex is at the origin and the branch tests tr >= 0 and dg <= 0 are scale-free).  So the
// network sees the direction (eps / s, logJp / s), tr / s and the friction angle, and predicts
// D / s and (tau - kappa c) / (kappa s) (sD = s, sT = kappa s, off = kappa c): its error
// vanishes with the strain instead of leaving a stress floor on particles at rest.
// Snow: the log strains are mapped into the clamp box [log(1 - theta_c), log(1 + theta_s)] as
// u = (l - mid) / half, where the clamp sits at u = +-1 for every theta, and the network
// predicts D / half and tau / (kappa exp(xi (1 - Jp))) (the hardened modulus of the trial state).
struct net_scale {
  float sD, sT, off;
};

__device__ __forceinline__ void closure_inputs(int model, float kappa, float hardening, const float *raw, float *in,
                                               net_scale &ns) {
  if (model == 1) {
    const float e0 = raw[0] - raw[4], e1 = raw[1] - raw[4], e2 = raw[2] - raw[4];
    const float s = sqrtf(e0 * e0 + e1 * e1 + e2 * e2 + raw[5] * raw[5]) + 1e-12f;
    const float inv = 1.f / s;
    in[0] = e0 * inv;
    in[1] = e1 * inv;
    in[2] = e2 * inv;
    in[3] = raw[5] * inv;
    in[4] = raw[3];
    in[5] = in[0] + in[1] + in[2] + in[3];
    ns.sD = s;
    ns.sT = kappa * s;
    ns.off = kappa * raw[4];
  } else {
    const float lo = log1pf(-raw[3]), hi = log1pf(raw[4]);
    const float mid = 0.5f * (lo + hi), half = 0.5f * (hi - lo);
    const float ih = 1.f / half;
    in[0] = (raw[0] - mid) * ih;
    in[1] = (raw[1] - mid) * ih;
    in[2] = (raw[2] - mid) * ih;
    in[3] = raw[3];
    in[4] = raw[4];
    in[5] = raw[5];
    ns.sD = half;
    ns.sT = kappa * expf(hardening * (1.f - expf(raw[5])));
    ns.off = 0.f;
  }
}

// (D, tau) of a raw row -> the network's targets
__device__ __forceinline__ void closure_net_targets(const net_scale &ns, const float *y, float *t) {
  const float iD = 1.f / ns.sD, iT = 1.f / ns.sT;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    t[i] = y[i] * iD;
    t[3 + i] = (y[3 + i] - ns.off) * iT;
  }
}

// the network's outputs -> (D, tau)
__device__ __forceinline__ void closure_from_net(const net_scale &ns, const float *o, float *y) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    y[i] = o[i] * ns.sD;
    y[3 + i] = ns.off + ns.sT * o[3 + i];
  }
}

// ---------------------------------------------------------------- BF16 tensor-core MLP
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

// D += A B for one 16x8x16 tile: A row-major BF16 (4 regs), B column-major BF16 (2 regs)
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint2 b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// SiLU on a packed pair in BF16: x * sigmoid(x) = h + h tanh(h), h = x / 2
__device__ __forceinline__ uint32_t silu_bf16x2(uint32_t x) {
  uint32_t h, t, y;
  const uint32_t half = 0x3f003f00u;  // (0.5, 0.5) in bf16
  asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(h) : "r"(x), "r"(half));
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(h));
  asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(y) : "r"(h), "r"(t));
  return y;
}

// One hidden layer of N=64 outputs for one 16-row tile: acc = X W^T + b.
template <int KS>
__device__ __forceinline__ void mlp_layer64(const uint32_t (&a)[KS][4], const uint2 *frag, const float *bias,
                                            float (&acc)[8][4], int lane) {
  const int t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = bias[nt * 8 + 2 * t], b1 = bias[nt * 8 + 2 * t + 1];
    acc[nt][0] = b0;
    acc[nt][1] = b1;
    acc[nt][2] = b0;
    acc[nt][3] = b1;
  }
#pragma unroll
  for (int ks = 0; ks < KS; ++ks)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) mma_bf16_16816(acc[nt], a[ks], frag[(ks * 8 + nt) * 32 + lane]);
}

// Accumulator tile of a 64-wide layer -> SiLU -> A fragments (K = 64, 4 slices) of the next.
// The C fragment of n-tiles (2ks, 2ks+1) holds exactly the A fragment of k-slice ks, so the
// activations never leave registers.
__device__ __forceinline__ void mlp_activate(const float (&acc)[8][4], uint32_t (&a)[4][4]) {
#pragma unroll
  for (int ks = 0; ks < 4; ++ks) {
    a[ks][0] = silu_bf16x2(pack_bf16x2(acc[2 * ks][0], acc[2 * ks][1]));
    a[ks][1] = silu_bf16x2(pack_bf16x2(acc[2 * ks][2], acc[2 * ks][3]));
    a[ks][2] = silu_bf16x2(pack_bf16x2(acc[2 * ks + 1][0], acc[2 * ks + 1][1]));
    a[ks][3] = silu_bf16x2(pack_bf16x2(acc[2 * ks + 1][2], acc[2 * ks + 1][3]));
  }
}

// Forward pass for the 32 particles of a warp.  in[6] are this lane's normalised features,
// out[6] receives this lane's outputs (normalised units).  xs (32 x 16 bf16) and ys
// (32 x 8 float) are per-warp shared scratch.  Every lane of the warp must call this together.
// The two 16-row tiles run one after the other, so that one tile's accumulators (32 floats)
// and activations (16 words) are live at a time.
__device__ __forceinline__ void mlp_forward_warp(const float (&in)[kMlpIn], float (&out)[kMlpOut],
                                                 const uint2 *frag, const float *bias,
                                                 __nv_bfloat16 *xs, float *ys) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int k = 0; k < 16; ++k) xs[lane * 16 + k] = __float2bfloat16_rn(k < kMlpIn ? in[k] : 0.f);
  __syncwarp();
  const uint32_t *xw = reinterpret_cast<const uint32_t *>(xs);  // 8 words per row
#pragma unroll 1
  for (int mt = 0; mt < 2; ++mt) {
    const int r0 = mt * 16 + g, r1 = r0 + 8;
    uint32_t a1[1][4];
    a1[0][0] = xw[r0 * 8 + t];
    a1[0][1] = xw[r1 * 8 + t];
    a1[0][2] = xw[r0 * 8 + 4 + t];
    a1[0][3] = xw[r1 * 8 + 4 + t];
    float acc[8][4];
    uint32_t ah[4][4];
    mlp_layer64<1>(a1, frag + kFragOff1, bias, acc, lane);
    mlp_activate(acc, ah);
    mlp_layer64<4>(ah, frag + kFragOff2, bias + 64, acc, lane);
    mlp_activate(acc, ah);
    mlp_layer64<4>(ah, frag + kFragOff3, bias + 128, acc, lane);
    mlp_activate(acc, ah);
    // output layer, N = 8 (6 used)
    float o[4];
    const float b0 = bias[192 + 2 * t], b1 = bias[192 + 2 * t + 1];
    o[0] = b0;
    o[1] = b1;
    o[2] = b0;
    o[3] = b1;
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) mma_bf16_16816(o, ah[ks], frag[kFragOff4 + ks * 32 + lane]);
    ys[r0 * 8 + 2 * t] = o[0];
    ys[r0 * 8 + 2 * t + 1] = o[1];
    ys[r1 * 8 + 2 * t] = o[2];
    ys[r1 * 8 + 2 * t + 1] = o[3];
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < kMlpOut; ++k) out[k] = ys[lane * 8 + k];
  __syncwarp();
}

}  // namespace zsmpm
