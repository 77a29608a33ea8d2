// Learned return-mapping closure: training set generation from the plain return map,
// FP32 training (hand-written forward/backward/Adam kernels), BF16 fragment packing for
// the tensor-core inference that runs inside G2P, and the zsmpm_closure_* C ABI.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "zsmpm.h"
#include "zsmpm_internal.h"
#include "zsmpm_mlp.cuh"

using namespace zsmpm;

struct zsmpm_closure {
  int device = 0;
  zsmpm_material mat{};
  material_dev md{};
  closure_dev cd{};
  float *params = nullptr;  // FP32 master weights
  float *grad = nullptr;
  float *adam_m = nullptr, *adam_v = nullptr;
  uint2 *frag = nullptr;
  float *bias = nullptr;
  double *audit = nullptr;    // audit accumulators until the closure is attached to a scene
  float *data_x = nullptr;    // raw features [n][6]
  float *data_y = nullptr;    // raw targets [n][6] (D, tau)
  float *data_xt = nullptr;   // network inputs [n][6] (closure_inputs of data_x)
  float *data_yt = nullptr;   // network targets [n][6] (closure_net_targets of data_y)
  int64_t data_n = 0, data_cap = 0;
  float *stats = nullptr;     // reduction scratch
  float *loss = nullptr;
  int adam_t = 0;
  bool normalized = false;
};

namespace {

constexpr int kThreads = 256;
constexpr int kTile = 32;  // samples per CTA in training

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// uniform in [0, 1) from (seed, sample, draw)
__device__ __forceinline__ float urand(uint64_t seed, uint64_t i, int k) {
  return (float)(mix64(seed ^ (i * 16 + k) * 0x9E3779B97F4A7C15ull) >> 40) * (1.f / 16777216.f);
}

// floats as ints whose signed order is the float order (an involution)
__host__ __device__ __forceinline__ int ordered_bits(int i) { return i >= 0 ? i : i ^ 0x7fffffff; }

__device__ __forceinline__ float yield_surface_of(float friction_deg) {
  const float s = sinf(friction_deg * 0.017453292519943295f);
  return 0.816496580927726f * 2.f * s / (3.f - s);
}

// targets of one raw feature row: D = H - l and principal Kirchhoff stress
__device__ __forceinline__ void closure_target(const material_dev &md, int model, const float *x,
                                               float *y) {
  const float l[3] = {x[0], x[1], x[2]};
  principal_result r;
  if (model == 1) {
    r = dp_principal(md.mu, md.lambda, x[4], md.beta, md.volume_correction, yield_surface_of(x[3]), l, x[5]);
  } else {
    const float S[3] = {expf(l[0]), expf(l[1]), expf(l[2])};
    r = snow_principal(md.mu, md.lambda, md.hardening, x[3], x[4], S, expf(x[5]));
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    y[i] = r.H[i] - l[i];
    y[3 + i] = r.tau[i];
  }
}

// random trial states: log singular values (sorted descending) plus the material / state
// features of the model
__global__ void k_closure_random(material_dev md, int model, float coh_scale, uint64_t seed,
                                 float *x, float *y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    // log singular values: [log 0.5, log 2] for Drucker-Prager; [-0.1, 0.05] for snow, around
    // its clamp box [log(1 - theta_c), log(1 + theta_s)]
    const float lo = model == 1 ? -0.69314718f : -0.1f, width = model == 1 ? 1.38629436f : 0.15f;
    float l[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) l[k] = lo + width * urand(seed, i, k);
    // sort descending
    if (l[0] < l[1]) { const float t = l[0]; l[0] = l[1]; l[1] = t; }
    if (l[1] < l[2]) { const float t = l[1]; l[1] = l[2]; l[2] = t; }
    if (l[0] < l[1]) { const float t = l[0]; l[0] = l[1]; l[1] = t; }
    float *xr = x + 6 * i;
    xr[0] = l[0];
    xr[1] = l[1];
    xr[2] = l[2];
    if (model == 1) {
      xr[3] = 20.f + 25.f * urand(seed, i, 3);  // friction angle (deg)
      // cohesion 0..100 Pa as a log-strain shift, exactly 0 for a quarter of the samples
      xr[4] = urand(seed, i, 7) < 0.25f ? 0.f : 100.f * urand(seed, i, 4) * coh_scale;
      xr[5] = urand(seed, i, 5) < 0.5f ? 0.f : 0.2f * urand(seed, i, 6);  // logJp
    } else {
      xr[3] = 0.015f + 0.02f * urand(seed, i, 3);   // theta_c
      xr[4] = 0.005f + 0.005f * urand(seed, i, 4);  // theta_s
      xr[5] = -0.15f + 0.3f * urand(seed, i, 5);    // log Jp
    }
    closure_target(md, model, xr, y + 6 * i);
  }
}

__global__ void k_closure_targets(material_dev md, int model, const float *x, float *y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    closure_target(md, model, x + 6 * i, y + 6 * i);
}

// raw rows (x, y) -> network inputs and targets (xt, yt)
__global__ void k_closure_transform(closure_dev cd, const float *x, const float *y, float *xt, float *yt,
                                    int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float raw[6], in[6], yr[6], t[6];
    net_scale ns;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      raw[k] = x[6 * i + k];
      yr[k] = y[6 * i + k];
    }
    closure_inputs(cd.model, cd.kappa, cd.hardening, raw, in, ns);
    closure_net_targets(ns, yr, t);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      xt[6 * i + k] = in[k];
      yt[6 * i + k] = t[k];
    }
  }
}

// per-feature sum and sum of squares of the network inputs x [n][6], min and max of the raw
// rows r [n][6], sum of squares of the network targets y [n][6]:
// stats[0..5] sum x, [6..11] sumsq x, [12..17] min r, [18..23] max r, [24..29] sumsq y
__global__ void k_closure_stats(const float *x, const float *r, const float *y, int64_t n, float *stats) {
  float sx[6] = {}, qx[6] = {}, mn[6], mx[6], qy[6] = {};
  for (int k = 0; k < 6; ++k) {
    mn[k] = 3.4e38f;
    mx[k] = -3.4e38f;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int k = 0; k < 6; ++k) {
      const float a = x[6 * i + k], b = y[6 * i + k], c = r[6 * i + k];
      sx[k] += a;
      qx[k] += a * a;
      mn[k] = fminf(mn[k], c);
      mx[k] = fmaxf(mx[k], c);
      qy[k] += b * b;
    }
  for (int k = 0; k < 6; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      sx[k] += __shfl_xor_sync(0xffffffffu, sx[k], o);
      qx[k] += __shfl_xor_sync(0xffffffffu, qx[k], o);
      qy[k] += __shfl_xor_sync(0xffffffffu, qy[k], o);
      mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
      mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
    }
  }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 6; ++k) {
      atomicAdd(&stats[k], sx[k]);
      atomicAdd(&stats[6 + k], qx[k]);
      atomicAdd(&stats[24 + k], qy[k]);
      // float min/max through ordered ints (values of either sign)
      atomicMin(reinterpret_cast<int *>(&stats[12 + k]), ordered_bits(__float_as_int(mn[k])));
      atomicMax(reinterpret_cast<int *>(&stats[18 + k]), ordered_bits(__float_as_int(mx[k])));
    }
}

__device__ __forceinline__ float silu(float z) { return z / (1.f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.f / (1.f + expf(-z));
  return s * (1.f + z * (1.f - s));
}

struct norm_dev {
  float in_mean[6], in_inv_std[6], out_inv_scale[6];
};

// Shared-memory copy of the weights with each row padded by one float (row stride kin + 1), so
// that threads of a warp reading W[j][k] for consecutive j hit distinct banks.
constexpr int kSW1 = 0, kSB1 = kSW1 + 64 * 7, kSW2 = kSB1 + 64, kSB2 = kSW2 + 64 * 65, kSW3 = kSB2 + 64,
              kSB3 = kSW3 + 64 * 65, kSW4 = kSB3 + 64, kSB4 = kSW4 + 6 * 65, kSParams = kSB4 + 8;

__device__ __forceinline__ void load_padded(const float *p, float *W) {
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) {
    int dst;
    if (i < kOffB1) dst = kSW1 + (i / 6) * 7 + i % 6;
    else if (i < kOffW2) dst = kSB1 + (i - kOffB1);
    else if (i < kOffB2) dst = kSW2 + ((i - kOffW2) / 64) * 65 + (i - kOffW2) % 64;
    else if (i < kOffW3) dst = kSB2 + (i - kOffB2);
    else if (i < kOffB3) dst = kSW3 + ((i - kOffW3) / 64) * 65 + (i - kOffW3) % 64;
    else if (i < kOffW4) dst = kSB3 + (i - kOffB3);
    else if (i < kOffB4) dst = kSW4 + ((i - kOffW4) / 64) * 65 + (i - kOffW4) % 64;
    else dst = kSB4 + (i - kOffB4);
    W[dst] = p[i];
  }
}

// Forward + backward of the MSE loss on normalised data for one tile of 32 samples per CTA;
// gradients (mean over `total` samples) are accumulated with atomics into grad, and the loss
// into *loss.  Sample k of the batch (k < count) is data row ((first + k) * stride) % n_data.
__global__ void __launch_bounds__(kThreads) k_mlp_train_tile(const float *params, const float *x, const float *y,
                                                             int64_t n_data, int64_t first, int64_t count,
                                                             int64_t stride, int64_t total, norm_dev nd,
                                                             float *grad, float *loss) {
  extern __shared__ float smem[];
  float *W = smem;                                  // kSParams (padded rows)
  float *A0 = W + kSParams;                         // [32][6]
  float *Z1 = A0 + kTile * 6, *A1 = Z1 + kTile * 64;
  float *Z2 = A1 + kTile * 64, *A2 = Z2 + kTile * 64;
  float *Z3 = A2 + kTile * 64, *A3 = Z3 + kTile * 64;
  float *OUT = A3 + kTile * 64;                     // [32][6]
  float *Y = OUT + kTile * 6;                       // [32][6]
  float *dA = Y + kTile * 6;                        // [32][64]
  float *dZ = dA + kTile * 64;                      // [32][64]
  const int t = threadIdx.x;
  const int64_t base = (int64_t)blockIdx.x * kTile;
  load_padded(params, W);
  for (int i = t; i < kTile * 6; i += blockDim.x) {
    const int s = i / 6, k = i % 6;
    const int64_t row = base + s;
    float xv = 0.f, yv = 0.f;
    if (row < count) {
      const int64_t r = (int64_t)(((unsigned long long)(first + row) * (unsigned long long)stride) %
                                  (unsigned long long)n_data);
      xv = (x[6 * r + k] - nd.in_mean[k]) * nd.in_inv_std[k];
      yv = y[6 * r + k] * nd.out_inv_scale[k];
    }
    A0[i] = xv;
    Y[i] = yv;
  }
  __syncthreads();
  const int valid = (int)(count - base < kTile ? count - base : kTile);
  auto dense = [&](const float *in, int kin, const float *Wl, const float *bl, float *z, float *a, int nout,
                   bool act) {
    for (int i = t; i < kTile * nout; i += blockDim.x) {
      const int s = i / nout, j = i % nout;
      float acc = bl[j];
      for (int k = 0; k < kin; ++k) acc += in[s * kin + k] * Wl[j * (kin + 1) + k];
      z[i] = acc;
      if (a) a[i] = act ? silu(acc) : acc;
    }
    __syncthreads();
  };
  dense(A0, 6, W + kSW1, W + kSB1, Z1, A1, 64, true);
  dense(A1, 64, W + kSW2, W + kSB2, Z2, A2, 64, true);
  dense(A2, 64, W + kSW3, W + kSB3, Z3, A3, 64, true);
  dense(A3, 64, W + kSW4, W + kSB4, OUT, nullptr, 6, false);
  // dL/dOUT for L = mean over samples and outputs of (OUT - Y)^2
  const float inv = 1.f / ((float)total * 6.f);
  float lsum = 0.f;
  for (int i = t; i < kTile * 6; i += blockDim.x) {
    const int s = i / 6;
    const float e = s < valid ? OUT[i] - Y[i] : 0.f;
    dZ[i] = 2.f * e * inv;  // dOUT stored in dZ[32][6]
    lsum += e * e * inv;
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((t & 31) == 0) atomicAdd(loss, lsum);
  __syncthreads();
  // back through a dense layer: gW[j][k] += sum_s dz[s][j] in[s][k]; gb[j] += sum_s dz[s][j];
  // din[s][k] = sum_j dz[s][j] W[j][k]
  auto back = [&](const float *dz, int nout, const float *in, int kin, const float *Wl, float *gW, float *gb,
                  float *din) {
    for (int i = t; i < nout * kin; i += blockDim.x) {
      const int j = i / kin, k = i % kin;
      float acc = 0.f;
      for (int s = 0; s < kTile; ++s) acc += dz[s * nout + j] * in[s * kin + k];
      atomicAdd(&gW[i], acc);
    }
    for (int j = t; j < nout; j += blockDim.x) {
      float acc = 0.f;
      for (int s = 0; s < kTile; ++s) acc += dz[s * nout + j];
      atomicAdd(&gb[j], acc);
    }
    if (din)
      for (int i = t; i < kTile * kin; i += blockDim.x) {
        const int s = i / kin, k = i % kin;
        float acc = 0.f;
        for (int j = 0; j < nout; ++j) acc += dz[s * nout + j] * Wl[j * (kin + 1) + k];
        din[i] = acc;
      }
    __syncthreads();
  };
  auto through_silu = [&](const float *da, const float *z, float *dz) {
    for (int i = t; i < kTile * 64; i += blockDim.x) dz[i] = da[i] * silu_grad(z[i]);
    __syncthreads();
  };
  back(dZ, 6, A3, 64, W + kSW4, grad + kOffW4, grad + kOffB4, dA);
  through_silu(dA, Z3, dZ);
  back(dZ, 64, A2, 64, W + kSW3, grad + kOffW3, grad + kOffB3, dA);
  through_silu(dA, Z2, dZ);
  back(dZ, 64, A1, 64, W + kSW2, grad + kOffW2, grad + kOffB2, dA);
  through_silu(dA, Z1, dZ);
  back(dZ, 64, A0, 6, W + kOffW1, grad + kOffW1, grad + kOffB1, nullptr);
}

constexpr size_t kTrainSmem =
    sizeof(float) * (kSParams + kTile * 6 + 6 * kTile * 64 + kTile * 6 * 2 + 2 * kTile * 64);

__global__ void k_adam(float *p, float *g, float *m, float *v, int n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    g[i] = 0.f;
  }
}

// FP32 master weights -> BF16 mma B fragments and padded biases
__global__ void k_pack_fragments(const float *p, uint2 *frag, float *bias) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  auto W = [&](int layer, int n, int k) -> float {
    if (layer == 0) return (n < 64 && k < 6) ? p[kOffW1 + n * 6 + k] : 0.f;
    if (layer == 1) return p[kOffW2 + n * 64 + k];
    if (layer == 2) return p[kOffW3 + n * 64 + k];
    return (n < 6) ? p[kOffW4 + n * 64 + k] : 0.f;
  };
  if (tid < kFragTotal) {
    int layer, local, NT;
    if (tid < kFragOff2) { layer = 0; local = tid - kFragOff1; NT = 8; }
    else if (tid < kFragOff3) { layer = 1; local = tid - kFragOff2; NT = 8; }
    else if (tid < kFragOff4) { layer = 2; local = tid - kFragOff3; NT = 8; }
    else { layer = 3; local = tid - kFragOff4; NT = 1; }
    const int lane = local & 31, pair = local >> 5;
    const int ks = pair / NT, nt = pair % NT;
    const int n = nt * 8 + (lane >> 2), k0 = ks * 16 + 2 * (lane & 3);
    uint2 f;
    f.x = pack_bf16x2(W(layer, n, k0), W(layer, n, k0 + 1));
    f.y = pack_bf16x2(W(layer, n, k0 + 8), W(layer, n, k0 + 9));
    frag[tid] = f;
  }
  if (tid < kBiasTotal) {
    float b = 0.f;
    if (tid < 64) b = p[kOffB1 + tid];
    else if (tid < 128) b = p[kOffB2 + tid - 64];
    else if (tid < 192) b = p[kOffB3 + tid - 128];
    else if (tid - 192 < 6) b = p[kOffB4 + tid - 192];
    bias[tid] = b;
  }
}

// Inference of raw feature rows on BF16 tensor cores (one warp per 32 rows, the code G2P
// runs); outputs are unscaled (D, tau).
__global__ void __launch_bounds__(kThreads) k_closure_infer_bf16(closure_dev cd, const float *x, float *y, int64_t n) {
  __shared__ __align__(16) __nv_bfloat16 xs[kThreads / 32][32 * 16];
  __shared__ float ys[kThreads / 32][32 * 8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t base = ((int64_t)blockIdx.x * (kThreads / 32) + warp) * 32; base < n;
       base += (int64_t)gridDim.x * kThreads) {
    const int64_t i = base + lane;
    float raw[6], in[kMlpIn], out[kMlpOut];
    net_scale ns;
#pragma unroll
    for (int k = 0; k < 6; ++k) raw[k] = i < n ? x[6 * i + k] : (k == 3 ? 0.02f : k == 4 ? 0.0075f : 0.f);
    closure_inputs(cd.model, cd.kappa, cd.hardening, raw, in, ns);
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) in[k] = (in[k] - cd.in_mean[k]) * cd.in_inv_std[k];
    mlp_forward_warp(in, out, cd.frag, cd.bias, xs[warp], ys[warp]);
#pragma unroll
    for (int k = 0; k < kMlpOut; ++k) out[k] *= cd.out_scale[k];
    float yr[6];
    closure_from_net(ns, out, yr);
    if (i < n)
#pragma unroll
      for (int k = 0; k < 6; ++k) y[6 * i + k] = yr[k];
  }
}

// FP32 forward of the master weights (a reference for the BF16 path)
__global__ void k_closure_infer_fp32(closure_dev cd, const float *p, const float *x, float *y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float raw[6], a0[6], h1[64], h2[64], o[6];
    net_scale ns;
    for (int k = 0; k < 6; ++k) raw[k] = x[6 * i + k];
    closure_inputs(cd.model, cd.kappa, cd.hardening, raw, a0, ns);
    for (int k = 0; k < 6; ++k) a0[k] = (a0[k] - cd.in_mean[k]) * cd.in_inv_std[k];
    for (int j = 0; j < 64; ++j) {
      float acc = p[kOffB1 + j];
      for (int k = 0; k < 6; ++k) acc += p[kOffW1 + j * 6 + k] * a0[k];
      h1[j] = silu(acc);
    }
    for (int j = 0; j < 64; ++j) {
      float acc = p[kOffB2 + j];
      for (int k = 0; k < 64; ++k) acc += p[kOffW2 + j * 64 + k] * h1[k];
      h2[j] = silu(acc);
    }
    for (int j = 0; j < 64; ++j) {
      float acc = p[kOffB3 + j];
      for (int k = 0; k < 64; ++k) acc += p[kOffW3 + j * 64 + k] * h2[k];
      h1[j] = silu(acc);
    }
    for (int j = 0; j < 6; ++j) {
      float acc = p[kOffB4 + j];
      for (int k = 0; k < 64; ++k) acc += p[kOffW4 + j * 64 + k] * h1[k];
      o[j] = acc * cd.out_scale[j];
    }
    float yr[6];
    closure_from_net(ns, o, yr);
    for (int k = 0; k < 6; ++k) y[6 * i + k] = yr[k];
  }
}

zsmpm_status cerr(zsmpm_status st, const std::string &m) { return (zsmpm_status)record_error(st, m.c_str()); }
zsmpm_status ccuda(cudaError_t e, const char *what) {
  return cerr(ZSMPM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CZ_TRY(expr, what)                             \
  do {                                                 \
    cudaError_t e__ = (expr);                          \
    if (e__ != cudaSuccess) return ccuda(e__, what);   \
  } while (0)

int sms() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

// the training kernel's shared-memory size (above the 48 KB default), once per device
cudaError_t prepare_train_kernel(int device) {
  static std::mutex mu;
  static std::vector<char> done;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)done.size() <= device) done.resize(device + 1, 0);
  if (done[device]) return cudaSuccess;
  const cudaError_t e =
      cudaFuncSetAttribute(k_mlp_train_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem);
  if (e == cudaSuccess) done[device] = 1;
  return e;
}

// deterministic Xavier-uniform initial weights, zero biases
void init_params(std::vector<float> &h, uint64_t seed) {
  h.assign(kMlpParams, 0.f);
  uint64_t s = seed * 0x9E3779B97F4A7C15ull + 1;
  auto rnd = [&]() {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return (double)(s >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int nout, int nin) {
    const double a = std::sqrt(6.0 / (nin + nout));
    for (int i = 0; i < nout * nin; ++i) h[off + i] = (float)((2 * rnd() - 1) * a);
  };
  fill(kOffW1, 64, 6);
  fill(kOffW2, 64, 64);
  fill(kOffW3, 64, 64);
  fill(kOffW4, 6, 64);
}

norm_dev norm_of(const closure_dev &cd) {
  norm_dev nd{};
  for (int k = 0; k < 6; ++k) {
    nd.in_mean[k] = cd.in_mean[k];
    nd.in_inv_std[k] = cd.in_inv_std[k];
    nd.out_inv_scale[k] = 1.f / cd.out_scale[k];
  }
  return nd;
}

zsmpm_status pack(zsmpm_closure *c, cudaStream_t st) {
  k_pack_fragments<<<(kFragTotal + 255) / 256, 256, 0, st>>>(c->params, c->frag, c->bias);
  CZ_TRY(cudaGetLastError(), "pack fragments");
  return ZSMPM_OK;
}

}  // namespace

namespace zsmpm {
bool closure_device_view(const zsmpm_closure *c, closure_dev *out) {
  if (!c || !c->normalized) return false;
  *out = c->cd;
  return true;
}
}  // namespace zsmpm

extern "C" {

ZSMPM_API zsmpm_status zsmpm_closure_create(const zsmpm_material *mat, int32_t device, zsmpm_closure **out) {
  if (!mat || !out) return cerr(ZSMPM_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (mat->model != ZSMPM_DRUCKER_PRAGER && mat->model != ZSMPM_SNOW)
    return cerr(ZSMPM_ERR_INVALID_ARG, "the learned closure replaces a return map: Drucker-Prager or snow");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return cerr(ZSMPM_ERR_NO_DEVICE, "no CUDA device");
  }
  CZ_TRY(cudaSetDevice(device), "cudaSetDevice");
  auto *c = new zsmpm_closure();
  c->device = device;
  c->mat = *mat;
  c->md.model = mat->model;
  c->md.mode = 0;
  c->md.volume_correction = mat->volume_correction;
  c->md.mu = (float)(0.5 * (double)mat->E / (double)(1.f + mat->nu));
  c->md.lambda = mat->E * mat->nu / ((1.f + mat->nu) * (1.f - 2.f * mat->nu));
  c->md.volume = mat->volume;
  c->md.cohesion = mat->cohesion;
  c->md.beta = mat->beta;
  c->md.friction_deg = mat->friction_deg;
  c->md.hardening = mat->hardening;
  c->md.theta_c = mat->theta_c;
  c->md.theta_s = mat->theta_s;
  c->cd.model = mat->model;
  c->cd.kappa = 3.f * c->md.lambda + 2.f * c->md.mu;
  c->cd.hardening = mat->hardening;
  cudaError_t e = cudaMalloc(&c->params, sizeof(float) * kMlpParams);
  if (e == cudaSuccess) e = cudaMalloc(&c->grad, sizeof(float) * kMlpParams);
  if (e == cudaSuccess) e = cudaMalloc(&c->adam_m, sizeof(float) * kMlpParams);
  if (e == cudaSuccess) e = cudaMalloc(&c->adam_v, sizeof(float) * kMlpParams);
  if (e == cudaSuccess) e = cudaMalloc(&c->frag, sizeof(uint2) * kFragTotal);
  if (e == cudaSuccess) e = cudaMalloc(&c->bias, sizeof(float) * kBiasTotal);
  if (e == cudaSuccess) e = cudaMalloc(&c->stats, sizeof(float) * 32);
  if (e == cudaSuccess) e = cudaMalloc(&c->loss, sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&c->audit, sizeof(double) * 8);
  std::vector<float> h;
  init_params(h, 12345);
  if (e == cudaSuccess) e = cudaMemcpy(c->params, h.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(c->grad, 0, sizeof(float) * kMlpParams);
  if (e == cudaSuccess) e = cudaMemset(c->adam_m, 0, sizeof(float) * kMlpParams);
  if (e == cudaSuccess) e = cudaMemset(c->adam_v, 0, sizeof(float) * kMlpParams);
  if (e == cudaSuccess) e = cudaMemset(c->audit, 0, sizeof(double) * 8);
  if (e != cudaSuccess) {
    zsmpm_closure_destroy(c);
    return ccuda(e, "closure allocation");
  }
  for (int k = 0; k < 6; ++k) {
    c->cd.in_mean[k] = 0.f;
    c->cd.in_inv_std[k] = 1.f;
    c->cd.in_min[k] = -3.4e38f;
    c->cd.in_max[k] = 3.4e38f;
    c->cd.out_scale[k] = 1.f;
  }
  c->cd.frag = c->frag;
  c->cd.bias = c->bias;
  c->cd.audit = c->audit;
  *out = c;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_closure_destroy(zsmpm_closure *c) {
  if (!c) return ZSMPM_OK;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  for (void *p : {(void *)c->params, (void *)c->grad, (void *)c->adam_m, (void *)c->adam_v, (void *)c->frag,
                  (void *)c->bias, (void *)c->stats, (void *)c->loss, (void *)c->audit, (void *)c->data_x,
                  (void *)c->data_y, (void *)c->data_xt, (void *)c->data_yt})
    if (p) cudaFree(p);
  delete c;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_closure_build_dataset(zsmpm_closure *c, int64_t n_random, uint64_t seed,
                                                   const float *logged, int64_t n_logged, void *stream) {
  if (!c || n_random < 0 || n_logged < 0 || (n_logged > 0 && !logged) || n_random + n_logged < 1)
    return cerr(ZSMPM_ERR_INVALID_ARG, "bad dataset arguments");
  CZ_TRY(cudaSetDevice(c->device), "cudaSetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = n_random + n_logged;
  if (n > c->data_cap) {
    CZ_TRY(cudaStreamSynchronize(st), "dataset sync");
    for (float **b : {&c->data_x, &c->data_y, &c->data_xt, &c->data_yt}) {
      if (*b) cudaFree(*b);
      *b = nullptr;
    }
    c->data_cap = 0;
    for (float **b : {&c->data_x, &c->data_y, &c->data_xt, &c->data_yt})
      CZ_TRY(cudaMalloc(b, sizeof(float) * 6 * n), "dataset");
    c->data_cap = n;
  }
  c->data_n = n;
  const float coh_scale = 1.f / (3.f * c->md.lambda + 2.f * c->md.mu);  // Pa -> log-strain shift
  if (n_random)
    k_closure_random<<<sms() * 8, kThreads, 0, st>>>(c->md, c->cd.model, coh_scale, seed, c->data_x, c->data_y,
                                                     n_random);
  if (n_logged) {
    CZ_TRY(cudaMemcpyAsync(c->data_x + 6 * n_random, logged, sizeof(float) * 6 * n_logged, cudaMemcpyDeviceToDevice,
                           st),
           "copy logged states");
    k_closure_targets<<<sms() * 8, kThreads, 0, st>>>(c->md, c->cd.model, c->data_x + 6 * n_random,
                                                      c->data_y + 6 * n_random, n_logged);
  }
  k_closure_transform<<<sms() * 8, kThreads, 0, st>>>(c->cd, c->data_x, c->data_y, c->data_xt, c->data_yt, n);
  CZ_TRY(cudaGetLastError(), "dataset kernels");
  // normalisation of the network's inputs and targets; hull of the raw training rows
  float init[32];
  for (int k = 0; k < 32; ++k) init[k] = 0.f;
  for (int k = 0; k < 6; ++k) {
    const int lo = ordered_bits(0x7f7fffff), hi = ordered_bits((int)0xff7fffffu);  // +FLT_MAX, -FLT_MAX
    std::memcpy(&init[12 + k], &lo, 4);
    std::memcpy(&init[18 + k], &hi, 4);
  }
  CZ_TRY(cudaMemcpyAsync(c->stats, init, sizeof(init), cudaMemcpyHostToDevice, st), "stats init");
  k_closure_stats<<<sms() * 4, kThreads, 0, st>>>(c->data_xt, c->data_x, c->data_yt, n, c->stats);
  float h[32];
  CZ_TRY(cudaMemcpyAsync(h, c->stats, sizeof(h), cudaMemcpyDeviceToHost, st), "stats read");
  CZ_TRY(cudaStreamSynchronize(st), "stats sync");
  auto unorder = [](float f) {
    int i;
    std::memcpy(&i, &f, 4);
    i = ordered_bits(i);
    float r;
    std::memcpy(&r, &i, 4);
    return r;
  };
  for (int k = 0; k < 6; ++k) {
    const double mean = h[k] / (double)n;
    const double var = std::max(h[6 + k] / (double)n - mean * mean, 1e-20);
    c->cd.in_mean[k] = (float)mean;
    c->cd.in_inv_std[k] = (float)(1.0 / std::sqrt(var));
    c->cd.in_min[k] = unorder(h[12 + k]);
    c->cd.in_max[k] = unorder(h[18 + k]);
    const double rms = std::sqrt(h[24 + k] / (double)n);
    c->cd.out_scale[k] = (float)std::max(rms, 1e-12);
  }
  c->normalized = true;
  return pack(c, st);
}

ZSMPM_API zsmpm_status zsmpm_closure_train(zsmpm_closure *c, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                                           float *loss_out, void *stream) {
  if (!c || !c->normalized || c->data_n < 1 || epochs < 1 || batch < kTile || !(lr > 0.f))
    return cerr(ZSMPM_ERR_INVALID_ARG, "train needs a dataset, epochs >= 1, batch >= 32, lr > 0");
  CZ_TRY(cudaSetDevice(c->device), "cudaSetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CZ_TRY(prepare_train_kernel(c->device), "train smem");
  const int64_t n = c->data_n;
  // batches walk the data with a stride coprime with n, so that random and logged samples mix
  int64_t stride = 1;
  if (n > 1)
    for (int64_t cand : {1000003LL, 998244353LL, 1000000007LL, 15485863LL})
      if (cand % n != 0 && std::gcd(cand % n, n) == 1) {
        stride = cand % n;
        break;
      }
  const norm_dev nd = norm_of(c->cd);
  std::vector<float> losses(epochs, 0.f);
  for (int ep = 0; ep < epochs; ++ep) {
    CZ_TRY(cudaMemsetAsync(c->loss, 0, sizeof(float), st), "loss reset");
    const int64_t steps = (n + batch - 1) / batch;
    const int64_t offset = (int64_t)((seed * 104729ull + 7919ull * (uint64_t)ep) % (uint64_t)n);
    for (int64_t s = 0; s < steps; ++s) {
      const int64_t first = offset + s * batch;
      const int64_t count = std::min<int64_t>(batch, n - s * batch);
      const int tiles = (int)((count + kTile - 1) / kTile);
      k_mlp_train_tile<<<tiles, kThreads, kTrainSmem, st>>>(c->params, c->data_xt, c->data_yt, n, first, count,
                                                            stride, count, nd, c->grad, c->loss);
      ++c->adam_t;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, (double)c->adam_t)));
      const float c2 = (float)(1.0 / (1.0 - std::pow(0.999, (double)c->adam_t)));
      k_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(c->params, c->grad, c->adam_m, c->adam_v, kMlpParams, lr, b1,
                                                       b2, 1e-8f, c1, c2);
    }
    CZ_TRY(cudaGetLastError(), "train kernels");
    float l = 0.f;
    CZ_TRY(cudaMemcpyAsync(&l, c->loss, sizeof(float), cudaMemcpyDeviceToHost, st), "loss read");
    CZ_TRY(cudaStreamSynchronize(st), "train sync");
    losses[ep] = l / (float)steps;
  }
  if (loss_out) std::memcpy(loss_out, losses.data(), sizeof(float) * epochs);
  return pack(c, st);
}

ZSMPM_API zsmpm_status zsmpm_closure_loss_grad(zsmpm_closure *c, const float *x, const float *y, int64_t n,
                                               float *grad, float *loss, void *stream) {
  if (!c || !x || !y || !grad || !loss || n < 1) return cerr(ZSMPM_ERR_INVALID_ARG, "bad arguments");
  CZ_TRY(cudaSetDevice(c->device), "cudaSetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CZ_TRY(prepare_train_kernel(c->device), "train smem");
  float *xt = nullptr, *yt = nullptr;
  CZ_TRY(cudaMalloc(&xt, sizeof(float) * 6 * n), "loss_grad scratch");
  if (cudaMalloc(&yt, sizeof(float) * 6 * n) != cudaSuccess) {
    cudaFree(xt);
    return cerr(ZSMPM_ERR_CUDA, "loss_grad scratch");
  }
  cudaMemsetAsync(grad, 0, sizeof(float) * kMlpParams, st);
  cudaMemsetAsync(loss, 0, sizeof(float), st);
  k_closure_transform<<<sms() * 4, kThreads, 0, st>>>(c->cd, x, y, xt, yt, n);
  const int tiles = (int)((n + kTile - 1) / kTile);
  k_mlp_train_tile<<<tiles, kThreads, kTrainSmem, st>>>(c->params, xt, yt, n, 0, n, 1, n, norm_of(c->cd), grad, loss);
  const cudaError_t e = cudaGetLastError();
  const cudaError_t es = cudaStreamSynchronize(st);
  cudaFree(xt);
  cudaFree(yt);
  CZ_TRY(e, "loss_grad");
  CZ_TRY(es, "loss_grad sync");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_closure_infer(zsmpm_closure *c, const float *x, float *y, int64_t n, int32_t bf16,
                                           void *stream) {
  if (!c || !x || !y || n < 1) return cerr(ZSMPM_ERR_INVALID_ARG, "bad arguments");
  CZ_TRY(cudaSetDevice(c->device), "cudaSetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (bf16) {
    const zsmpm_status ps = pack(c, st);
    if (ps != ZSMPM_OK) return ps;
    k_closure_infer_bf16<<<sms() * 4, kThreads, 0, st>>>(c->cd, x, y, n);
  } else {
    k_closure_infer_fp32<<<sms() * 4, kThreads, 0, st>>>(c->cd, c->params, x, y, n);
  }
  CZ_TRY(cudaGetLastError(), "closure infer");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_closure_targets(zsmpm_closure *c, const float *x, float *y, int64_t n, void *stream) {
  if (!c || !x || !y || n < 1) return cerr(ZSMPM_ERR_INVALID_ARG, "bad arguments");
  CZ_TRY(cudaSetDevice(c->device), "cudaSetDevice");
  k_closure_targets<<<sms() * 4, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(c->md, c->cd.model, x, y, n);
  CZ_TRY(cudaGetLastError(), "closure targets");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_closure_get_state(zsmpm_closure *c, zsmpm_closure_state *out) {
  if (!c || !out) return cerr(ZSMPM_ERR_INVALID_ARG, "null argument");
  CZ_TRY(cudaSetDevice(c->device), "cudaSetDevice");
  CZ_TRY(cudaDeviceSynchronize(), "synchronize");
  CZ_TRY(cudaMemcpy(out->params, c->params, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost), "read params");
  for (int k = 0; k < 6; ++k) {
    out->in_mean[k] = c->cd.in_mean[k];
    out->in_inv_std[k] = c->cd.in_inv_std[k];
    out->in_min[k] = c->cd.in_min[k];
    out->in_max[k] = c->cd.in_max[k];
    out->out_scale[k] = c->cd.out_scale[k];
  }
  out->model = c->cd.model;
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_closure_set_state(zsmpm_closure *c, const zsmpm_closure_state *in) {
  if (!c || !in) return cerr(ZSMPM_ERR_INVALID_ARG, "null argument");
  if (in->model != c->cd.model) return cerr(ZSMPM_ERR_INVALID_ARG, "closure state of another model");
  CZ_TRY(cudaSetDevice(c->device), "cudaSetDevice");
  CZ_TRY(cudaDeviceSynchronize(), "synchronize");
  CZ_TRY(cudaMemcpy(c->params, in->params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice), "write params");
  for (int k = 0; k < 6; ++k) {
    c->cd.in_mean[k] = in->in_mean[k];
    c->cd.in_inv_std[k] = in->in_inv_std[k];
    c->cd.in_min[k] = in->in_min[k];
    c->cd.in_max[k] = in->in_max[k];
    c->cd.out_scale[k] = in->out_scale[k];
  }
  c->normalized = true;
  const zsmpm_status ps = pack(c, nullptr);
  if (ps != ZSMPM_OK) return ps;
  CZ_TRY(cudaDeviceSynchronize(), "pack");
  return ZSMPM_OK;
}

}  // extern "C"
