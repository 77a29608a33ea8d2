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
  uint4 *umma_w = nullptr;    // weights in the tcgen05 shared-memory layout (kTcWBytes)
  int *tc_status = nullptr;   // bounded-wait failures of the tcgen05 inference
  float *bias = nullptr;
  double *audit = nullptr;    // audit accumulators until the closure is attached to a scene
  float *data_x = nullptr;    // raw features [n][6]
  float *data_y = nullptr;    // raw targets [n][6] (D, tau)
  float *data_xt = nullptr;   // network inputs [n][6] (closure_inputs of data_x)
  float *data_yt = nullptr;   // network targets [n][6] (closure_net_targets of data_y)
  int64_t data_n = 0, data_cap = 0;
  int64_t data_generated = 0;  // rows generated or logged; data_n of them are projected by the plain map
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

// whether the plain map projects a raw row (the branch the network replaces): Drucker-Prager
// onto the cone (tr < 0 and dgamma > 0, compute_stress_sand), snow when a singular value
// leaves [1 - theta_c, 1 + theta_s]; elastic states and the Drucker-Prager tip are computed
// exactly in G2P and need no network
__device__ __forceinline__ bool closure_projects(const material_dev &md, int model, const float *x) {
  if (model == 1) {
    float eps[3], eh[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) eps[i] = x[i] - x[4];
    const float tr = eps[0] + eps[1] + eps[2] + x[5];
    if (tr >= 0.f) return false;
#pragma unroll
    for (int i = 0; i < 3; ++i) eh[i] = eps[i] - tr / 3.f;
    const float ehn = sqrtf(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2]);
    const float smu = 2.f * md.mu;
    return ehn + (3.f * md.lambda + smu) / smu * tr * yield_surface_of(x[3]) > 0.f;
  }
  bool out = false;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float S = expf(x[i]);
    out = out || S < 1.f - x[3] || S > 1.f + x[4];
  }
  return out;
}

// the rows the plain map projects, compacted (in any order) into (xo, yo); *count their number
__global__ void k_closure_keep_projected(material_dev md, int model, const float *x, const float *y, int64_t n,
                                         float *xo, float *yo, unsigned long long *count) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!closure_projects(md, model, x + 6 * i)) continue;
    const unsigned long long j = atomicAdd(count, 1ull);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      xo[6 * j + k] = x[6 * i + k];
      yo[6 * j + k] = y[6 * i + k];
    }
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

// ---------------------------------------------------------------- tcgen05 inference
// The same network on the 5th-generation tensor cores: one CTA of 128 threads takes 128-row
// tiles (one thread per row).  Per layer one elected thread issues tcgen05.mma (kind::f16,
// BF16 operands from shared memory, FP32 accumulators in tensor memory, M = 128) and commits
// it to an mbarrier; every thread then loads its row of the accumulator with tcgen05.ld,
// adds the bias, applies SiLU in bf16x2 (as the mma.sync path does) and writes the next
// layer's A tile back to shared memory.
//
// Shared-memory operands use the K-major layout without swizzle: 8-row x 16-byte core
// matrices; element (r, k) of an R-row matrix at (k / 8) * (16 R) + (r / 8) * 128 + (r % 8) * 16
// + (k % 8) * 2 bytes, so the stride between 8-row groups is 128 B and the stride between
// 8-element K chunks is 16 R bytes (the descriptor's stride and leading byte offsets).
constexpr int kTcRows = 128;
constexpr int kTcW1 = 0;                         // 64 x 16
constexpr int kTcW2 = kTcW1 + 64 * 16 * 2;       // 64 x 64
constexpr int kTcW3 = kTcW2 + 64 * 64 * 2;       // 64 x 64
constexpr int kTcW4 = kTcW3 + 64 * 64 * 2;       // 16 x 64 (6 rows used)
constexpr int kTcA = kTcW4 + 16 * 64 * 2;        // 128 x 64 activations
constexpr int kTcSmem = kTcA + kTcRows * 64 * 2;
constexpr int kTcWBytes = kTcA;                  // the packed weights
// the split-BF16 variant: weights and activations as hi + lo BF16 pairs (hi = bf16(v),
// lo = bf16(v - hi)), each layer A_hi W_hi + A_hi W_lo + A_lo W_hi into one FP32 accumulator:
// products to about 16 significant bits, against 8 for plain BF16 operands
constexpr int kTcSplitA = 2 * kTcWBytes;                       // A_hi, then A_lo
constexpr int kTcSplitSmem = kTcSplitA + 2 * kTcRows * 64 * 2;  // 72 KB: 3 CTAs per SM
constexpr int kTcTmemCols = 64;
constexpr long long kTcWaitLimit = 1ll << 22;    // try_wait rounds before giving up

__host__ __device__ constexpr int umma_offset(int R, int r, int k) {
  return (k >> 3) * (16 * R) + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// weights -> bf16 in the K-major layout (W[out][in]; zero padding to K = 16 and N = 16): the
// rounded weights at w, and their rounding residuals bf16(v - bf16(v)) kTcWBytes further on
__global__ void k_pack_umma(const float *p, __nv_bfloat16 *w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // element index over all four matrices
  int base, R, K, layer, local;
  if (i < 64 * 16) { layer = 0; base = kTcW1; R = 64; K = 16; local = i; }
  else if (i < 64 * 16 + 4096) { layer = 1; base = kTcW2; R = 64; K = 64; local = i - 64 * 16; }
  else if (i < 64 * 16 + 8192) { layer = 2; base = kTcW3; R = 64; K = 64; local = i - 64 * 16 - 4096; }
  else if (i < 64 * 16 + 8192 + 16 * 64) { layer = 3; base = kTcW4; R = 16; K = 64; local = i - 64 * 16 - 8192; }
  else return;
  const int r = local / K, k = local % K;
  float v = 0.f;
  if (layer == 0) v = k < 6 ? p[kOffW1 + r * 6 + k] : 0.f;
  else if (layer == 1) v = p[kOffW2 + r * 64 + k];
  else if (layer == 2) v = p[kOffW3 + r * 64 + k];
  else v = r < 6 ? p[kOffW4 + r * 64 + k] : 0.f;
  const __nv_bfloat16 hi = __float2bfloat16_rn(v);
  w[(base + umma_offset(R, r, k)) / 2] = hi;
  w[(kTcWBytes + base + umma_offset(R, r, k)) / 2] = __float2bfloat16_rn(v - __bfloat162float(hi));
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)(128u >> 4) << 32;  // 8-row groups 128 B apart
  d |= (uint64_t)1 << 46;            // descriptor version of sm_100; no swizzle, base offset 0
  return d;
}

// kind::f16 instruction descriptor: BF16 A and B (K-major), FP32 D, M = 128, N
__device__ __forceinline__ uint32_t umma_idesc(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p; \n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < kTcWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 64 columns of this thread's row of the accumulator
__device__ __forceinline__ void tmem_ld64(uint32_t addr, float (&v)[64]) {
  uint32_t r[64];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,"
      "%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
        "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
        "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
        "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
        "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 64; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// v as a hi + lo pair of bf16 (two bf16x2 words for two values)
__device__ __forceinline__ void split_bf16x2(float a, float b, uint32_t &hi, uint32_t &lo) {
  const __nv_bfloat16 ha = __float2bfloat16_rn(a), hb = __float2bfloat16_rn(b);
  hi = (uint32_t)__bfloat16_as_ushort(ha) | ((uint32_t)__bfloat16_as_ushort(hb) << 16);
  lo = pack_bf16x2(a - __bfloat162float(ha), b - __bfloat162float(hb));
}

// the split variant's epilogue: bias + SiLU in FP32, written as hi and lo rows
__device__ __forceinline__ void tc_hidden_epilogue_split(uint32_t tmem_row, const float *bias, unsigned char *a_hi,
                                                         unsigned char *a_lo, int row) {
  float v[64];
  tmem_ld64(tmem_row, v);
#pragma unroll
  for (int kc = 0; kc < 8; ++kc) {
    float a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float z = v[8 * kc + j] + bias[8 * kc + j];
      a[j] = __fdividef(z, 1.f + __expf(-z));
    }
    uint4 h, l;
    split_bf16x2(a[0], a[1], h.x, l.x);
    split_bf16x2(a[2], a[3], h.y, l.y);
    split_bf16x2(a[4], a[5], h.z, l.z);
    split_bf16x2(a[6], a[7], h.w, l.w);
    *reinterpret_cast<uint4 *>(a_hi + umma_offset(kTcRows, row, 8 * kc)) = h;
    *reinterpret_cast<uint4 *>(a_lo + umma_offset(kTcRows, row, 8 * kc)) = l;
  }
}

// one hidden layer's epilogue: bias + SiLU (bf16x2) of this thread's 64 accumulators into its
// row of the A tile
__device__ __forceinline__ void tc_hidden_epilogue(uint32_t tmem_row, const float *bias, unsigned char *a_tile,
                                                   int row) {
  float v[64];
  tmem_ld64(tmem_row, v);
#pragma unroll
  for (int kc = 0; kc < 8; ++kc) {
    uint4 q;
    q.x = silu_bf16x2(pack_bf16x2(v[8 * kc + 0] + bias[8 * kc + 0], v[8 * kc + 1] + bias[8 * kc + 1]));
    q.y = silu_bf16x2(pack_bf16x2(v[8 * kc + 2] + bias[8 * kc + 2], v[8 * kc + 3] + bias[8 * kc + 3]));
    q.z = silu_bf16x2(pack_bf16x2(v[8 * kc + 4] + bias[8 * kc + 4], v[8 * kc + 5] + bias[8 * kc + 5]));
    q.w = silu_bf16x2(pack_bf16x2(v[8 * kc + 6] + bias[8 * kc + 6], v[8 * kc + 7] + bias[8 * kc + 7]));
    *reinterpret_cast<uint4 *>(a_tile + umma_offset(kTcRows, row, 8 * kc)) = q;
  }
}

// n_dev (optional): the row count in device memory, at most n (the G2P queue of a substep).
// kSplit: the split-BF16 variant (weights and activations as hi + lo BF16, three MMAs per K step).
template <bool kSplit>
__global__ void __launch_bounds__(kTcRows) k_closure_infer_tc(closure_dev cd, const uint4 *wpack, const float *x,
                                                              float *y, int64_t n, const int *n_dev, int *status) {
  if (n_dev) n = min(n, (int64_t)*n_dev);
  if ((int64_t)blockIdx.x * kTcRows >= n) return;  // no tile for this CTA (before any allocation)
  extern __shared__ __align__(1024) unsigned char tsm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t taddr_s;
  __shared__ float sbias[kBiasTotal];
  const int t = threadIdx.x, warp = t >> 5;
  for (int i = t; i < (kSplit ? 2 : 1) * kTcWBytes / 16; i += kTcRows) reinterpret_cast<uint4 *>(tsm)[i] = wpack[i];
  for (int i = t; i < kBiasTotal; i += kTcRows) sbias[i] = cd.bias[i];
  const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&mbar);
  if (warp == 0) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&taddr_s);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(kTcTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (t == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1));
  async_proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = taddr_s;
  const uint32_t tmem_row = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 lanes
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(tsm);
  constexpr int a_off = kSplit ? kTcSplitA : kTcA;
  unsigned char *a_tile = tsm + a_off;  // A_hi (the only A tile without the split)
  unsigned char *a_lo = tsm + a_off + kTcRows * 64 * 2;
  const uint32_t a_addr = sbase + a_off, alo_addr = a_addr + kTcRows * 64 * 2;
  const uint32_t id64 = umma_idesc(64), id16 = umma_idesc(16);
  uint32_t parity = 0;
  bool ok = true;
  for (int64_t tile = blockIdx.x; tile * kTcRows < n; tile += gridDim.x) {
    const int64_t row = tile * kTcRows + t;
    // input row -> network inputs -> bf16 A tile (K = 16: 6 inputs and zeros)
    float raw[6], in[kMlpIn];
    net_scale ns;
#pragma unroll
    for (int k = 0; k < 6; ++k) raw[k] = row < n ? x[6 * row + k] : (k == 3 ? 0.02f : k == 4 ? 0.0075f : 0.f);
    closure_inputs(cd.model, cd.kappa, cd.hardening, raw, in, ns);
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) in[k] = (in[k] - cd.in_mean[k]) * cd.in_inv_std[k];
    uint4 q0;
    if (kSplit) {
      uint4 l0;
      split_bf16x2(in[0], in[1], q0.x, l0.x);
      split_bf16x2(in[2], in[3], q0.y, l0.y);
      split_bf16x2(in[4], in[5], q0.z, l0.z);
      q0.w = l0.w = 0u;
      *reinterpret_cast<uint4 *>(a_lo + umma_offset(kTcRows, t, 0)) = l0;
      *reinterpret_cast<uint4 *>(a_lo + umma_offset(kTcRows, t, 8)) = make_uint4(0u, 0u, 0u, 0u);
    } else {
      q0.x = pack_bf16x2(in[0], in[1]);
      q0.y = pack_bf16x2(in[2], in[3]);
      q0.z = pack_bf16x2(in[4], in[5]);
      q0.w = 0u;
    }
    *reinterpret_cast<uint4 *>(a_tile + umma_offset(kTcRows, t, 0)) = q0;
    *reinterpret_cast<uint4 *>(a_tile + umma_offset(kTcRows, t, 8)) = make_uint4(0u, 0u, 0u, 0u);
    // four layers: MMA by one thread, completion through the mbarrier, epilogue by all
#pragma unroll 1
    for (int layer = 0; layer < 4 && ok; ++layer) {
      async_proxy_fence();
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      if (t == 0) {
        const int ksteps = layer == 0 ? 1 : 4;
        const uint32_t w_off = layer == 0 ? kTcW1 : layer == 1 ? kTcW2 : layer == 2 ? kTcW3 : kTcW4;
        const uint32_t w_rows = layer == 3 ? 16 : 64;
        const uint32_t idesc = layer == 3 ? id16 : id64;
        for (int ks = 0; ks < ksteps; ++ks) {
          const uint64_t a_hi = umma_desc(a_addr + 2 * ks * (16 * kTcRows), 16 * kTcRows);
          const uint64_t w_hi = umma_desc(sbase + w_off + 2 * ks * (16 * w_rows), 16 * w_rows);
          umma_bf16(tmem, a_hi, w_hi, idesc, ks > 0 ? 1u : 0u);
          if (kSplit) {
            umma_bf16(tmem, a_hi, umma_desc(sbase + kTcWBytes + w_off + 2 * ks * (16 * w_rows), 16 * w_rows),
                      idesc, 1u);
            umma_bf16(tmem, umma_desc(alo_addr + 2 * ks * (16 * kTcRows), 16 * kTcRows), w_hi, idesc, 1u);
          }
        }
        umma_commit(bar);
      }
      const bool done = mbar_wait(bar, parity);
      parity ^= 1u;
      ok = __syncthreads_and(done) != 0;
      if (!ok) break;
      tc_fence_after();
      if (layer < 3) {
        if (kSplit)
          tc_hidden_epilogue_split(tmem_row, sbias + 64 * layer, a_tile, a_lo, t);
        else
          tc_hidden_epilogue(tmem_row, sbias + 64 * layer, a_tile, t);
      } else {
        float o[16];
        tmem_ld16(tmem_row, o);
        float out[kMlpOut], yr[6];
#pragma unroll
        for (int k = 0; k < kMlpOut; ++k) out[k] = (o[k] + sbias[192 + k]) * cd.out_scale[k];
        closure_from_net(ns, out, yr);
        if (row < n)
#pragma unroll
          for (int k = 0; k < 6; ++k) y[6 * row + k] = yr[k];
      }
      tc_fence_before();
    }
    if (!ok) break;
  }
  // all tensor-memory reads are complete (tcgen05.ld waits) and no MMA is in flight unless a
  // wait gave up; then one more bounded wait for it before the columns are freed
  if (!ok) {
    mbar_wait(bar, parity ^ 1u);  // the phase whose wait gave up (parity has moved past it)
    if (t == 0) atomicOr(status, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols));
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
  k_pack_umma<<<(kTcWBytes / 2 + 255) / 256, 256, 0, st>>>(c->params, reinterpret_cast<__nv_bfloat16 *>(c->umma_w));
  CZ_TRY(cudaGetLastError(), "pack fragments");
  return ZSMPM_OK;
}

}  // namespace

namespace zsmpm {
bool closure_device_view(const zsmpm_closure *c, closure_dev *out) {
  if (!c || !c->normalized) return false;
  *out = c->cd;
  out->umma_w = c->umma_w;
  out->tc_status = c->tc_status;
  return true;
}

// the G2P queue's network pass: the split-BF16 tcgen05 forward (three CTAs of 72 KB per SM)
cudaError_t launch_closure_rows(const closure_dev &cd, const float *x, float *y, const int *n_dev, long long cap,
                                cudaStream_t st) {
  k_closure_infer_tc<true><<<sms() * 3, kTcRows, kTcSplitSmem, st>>>(cd, cd.umma_w, x, y, cap, n_dev, cd.tc_status);
  return cudaGetLastError();
}

// the split variant's shared memory exceeds the 48 KB default: set once per device, before any
// capture of its launches
cudaError_t prepare_closure_kernels() {
  return cudaFuncSetAttribute(k_closure_infer_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSplitSmem);
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
  if (e == cudaSuccess) e = cudaMalloc(&c->umma_w, 2 * kTcWBytes);  // rounded weights and residuals
  if (e == cudaSuccess) e = cudaMalloc(&c->tc_status, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->tc_status, 0, sizeof(int));
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
                  (void *)c->data_y, (void *)c->data_xt, (void *)c->data_yt, (void *)c->umma_w,
                  (void *)c->tc_status})
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
  // only states that the plain map projects: G2P evaluates the network on those alone
  {
    unsigned long long *kept = reinterpret_cast<unsigned long long *>(c->stats + 30);  // 8-byte aligned slot
    CZ_TRY(cudaMemsetAsync(kept, 0, sizeof(unsigned long long), st), "dataset count");
    k_closure_keep_projected<<<sms() * 8, kThreads, 0, st>>>(c->md, c->cd.model, c->data_x, c->data_y, n,
                                                             c->data_xt, c->data_yt, kept);
    unsigned long long h_kept = 0;
    CZ_TRY(cudaMemcpyAsync(&h_kept, kept, sizeof(h_kept), cudaMemcpyDeviceToHost, st), "dataset count");
    CZ_TRY(cudaStreamSynchronize(st), "dataset count");
    if (h_kept < 1) return cerr(ZSMPM_ERR_INVALID_ARG, "no state of the dataset is projected by the return map");
    std::swap(c->data_x, c->data_xt);
    std::swap(c->data_y, c->data_yt);
    c->data_generated = n;
    c->data_n = (int64_t)h_kept;
  }
  const int64_t m = c->data_n;
  k_closure_transform<<<sms() * 8, kThreads, 0, st>>>(c->cd, c->data_x, c->data_y, c->data_xt, c->data_yt, m);
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
  k_closure_stats<<<sms() * 4, kThreads, 0, st>>>(c->data_xt, c->data_x, c->data_yt, m, c->stats);
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
    const double mean = h[k] / (double)m;
    const double var = std::max(h[6 + k] / (double)m - mean * mean, 1e-20);
    c->cd.in_mean[k] = (float)mean;
    c->cd.in_inv_std[k] = (float)(1.0 / std::sqrt(var));
    c->cd.in_min[k] = unorder(h[12 + k]);
    c->cd.in_max[k] = unorder(h[18 + k]);
    const double rms = std::sqrt(h[24 + k] / (double)m);
    c->cd.out_scale[k] = (float)std::max(rms, 1e-12);
  }
  c->normalized = true;
  return pack(c, st);
}

ZSMPM_API zsmpm_status zsmpm_closure_dataset_size(const zsmpm_closure *c, int64_t *generated, int64_t *kept) {
  if (!c || !generated || !kept) return cerr(ZSMPM_ERR_INVALID_ARG, "null argument");
  *generated = c->data_generated;
  *kept = c->data_n;
  return ZSMPM_OK;
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
  if (bf16 == 2 || bf16 == 3) {
    const zsmpm_status ps = pack(c, st);
    if (ps != ZSMPM_OK) return ps;
    const int64_t tiles = (n + kTcRows - 1) / kTcRows;
    if (bf16 == 2) {
      // six resident CTAs per SM (37.7 KB of shared memory and 64 tensor-memory columns each), so
      // that six tiles' layer chains overlap on the SM's tensor core
      const int grid = (int)std::min<int64_t>(tiles, (int64_t)sms() * 6);
      k_closure_infer_tc<false><<<grid, kTcRows, kTcSmem, st>>>(c->cd, c->umma_w, x, y, n, nullptr, c->tc_status);
    } else {
      CZ_TRY(prepare_closure_kernels(), "closure kernel attributes");
      const int grid = (int)std::min<int64_t>(tiles, (int64_t)sms() * 3);
      k_closure_infer_tc<true><<<grid, kTcRows, kTcSplitSmem, st>>>(c->cd, c->umma_w, x, y, n, nullptr,
                                                                    c->tc_status);
    }
  } else if (bf16) {
    const zsmpm_status ps = pack(c, st);
    if (ps != ZSMPM_OK) return ps;
    k_closure_infer_bf16<<<sms() * 4, kThreads, 0, st>>>(c->cd, x, y, n);
  } else {
    k_closure_infer_fp32<<<sms() * 4, kThreads, 0, st>>>(c->cd, c->params, x, y, n);
  }
  CZ_TRY(cudaGetLastError(), "closure infer");
  return ZSMPM_OK;
}

ZSMPM_API zsmpm_status zsmpm_closure_status(zsmpm_closure *c) {
  if (!c) return cerr(ZSMPM_ERR_INVALID_ARG, "null closure");
  CZ_TRY(cudaSetDevice(c->device), "cudaSetDevice");
  CZ_TRY(cudaDeviceSynchronize(), "synchronize");
  int w = 0;
  CZ_TRY(cudaMemcpy(&w, c->tc_status, sizeof(int), cudaMemcpyDeviceToHost), "read closure status");
  if (w) {
    cudaMemset(c->tc_status, 0, sizeof(int));
    return cerr(ZSMPM_ERR_TIMEOUT, "a bounded wait for a tensor-core MMA gave up");
  }
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
