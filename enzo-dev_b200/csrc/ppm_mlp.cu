// ppm_mlp.cu -- training and evaluation kernels of the learned Newton start
// (ppm_guess.cuh): training samples from logged faces, forward + backward over a
// minibatch, Adam, and a standalone run of the tensor-core inference.
//
// Training runs in FP32 on the CUDA cores with the rounding the inference applies:
// inputs, weights and the two hidden activations are rounded to BF16, every sum is
// FP32.  The backward pass treats the rounding as the identity (straight-through).
// Loss: mean over the samples of (y - r)^2, r = ln(p* / p_acoustic) / |x|^2 the
// coefficient the net predicts (ppm_guess.cuh).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "ppm_device.cuh"
#include "ppm_guess.cuh"

namespace ppm {
namespace mlp {

__device__ __forceinline__ float bf16r(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

// ---------------------------------------------------------------- training samples
// record: dl dr pl pr ul ur p* +-iterations  ->  sample: 6 features, target r, valid
// (valid: Newton converged, finite values, and a jump large enough to define r)
__global__ void features_kernel(const double* __restrict__ rec, int64_t n, double gamma,
                                double pmin, float* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double* r = rec + i * 8;
    const double dl = r[0], dr = r[1], pl = r[2], pr = r[3], ul = r[4], ur = r[5];
    float f[6];
    const float d2 = guess_features(dl, dr, pl, pr, ul, ur, gamma, f);
    // the acoustic start of twoshock.F:156-170
    const double cl = sqrt(gamma * pl * dl), cr = sqrt(gamma * pr * dr);
    double ps = (cr * pl + cl * pr + cr * cl * (ul - ur)) / (cr + cl);
    if (ps < pmin) ps = pmin;
    const double t = log(r[6] / ps) / (double)d2;
    bool ok = r[7] > 0.0 && d2 > 1.0e-12f && t == t && fabs(t) < 16.0;
    float* o = out + i * 8;
    for (int k = 0; k < 6; ++k) {
      o[k] = f[k];
      ok = ok && (f[k] == f[k]) && fabsf(f[k]) < 1.0e30f;
    }
    o[6] = ok ? (float)t : 0.0f;
    o[7] = ok ? 1.0f : 0.0f;
  }
}

// ---------------------------------------------------------------- forward + backward
// One block of kTile threads; each pass takes kTile samples (thread b = sample b) and
// accumulates the gradient of the block in registers; one atomic add per weight and
// block at the end.  Shared memory: BF16-rounded weights, and per tile the inputs, the
// two hidden layers and the two pre-activation gradients.
constexpr int kTile = 128;
constexpr int kLd = kGuessHidden + 1;  // padded row of the per-sample tables

struct GradSmem {
  float w1[kGuessIn * kGuessHidden];
  float b1[kGuessHidden];
  float w2[kGuessHidden * kGuessHidden];
  float b2[kGuessHidden];
  float w3[kGuessHidden];
  float b3;
  float x[kTile][kGuessIn];
  float dy[kTile];
  float h1[kTile][kLd];
  float h2[kTile][kLd];
  float dz1[kTile][kLd];
  float dz2[kTile][kLd];
};

__global__ void __launch_bounds__(kTile) grad_kernel(const float* __restrict__ W,
                                                     const float* __restrict__ samples,
                                                     const int64_t* __restrict__ index,
                                                     int64_t n, float inv_count,
                                                     float* __restrict__ grad,
                                                     double* __restrict__ loss) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GradSmem& S = *reinterpret_cast<GradSmem*>(smem_raw);
  const int tid = threadIdx.x;
  for (int i = tid; i < kGuessIn * kGuessHidden; i += kTile) S.w1[i] = bf16r(W[kOffW1 + i]);
  for (int i = tid; i < kGuessHidden * kGuessHidden; i += kTile) S.w2[i] = bf16r(W[kOffW2 + i]);
  for (int i = tid; i < kGuessHidden; i += kTile) {
    S.b1[i] = W[kOffB1 + i];
    S.b2[i] = W[kOffB2 + i];
    S.w3[i] = bf16r(W[kOffW3 + i]);
  }
  if (tid == 0) S.b3 = W[kOffB3];
  __syncthreads();

  // this thread's share of the gradient: W2 entries (j = tid / 2, k in a half row),
  // W1 entries tid, tid + 128, tid + 256, and one bias / w3 entry
  float gw2[32];
#pragma unroll
  for (int e = 0; e < 32; ++e) gw2[e] = 0.0f;
  float gw1[3] = {0.0f, 0.0f, 0.0f};
  float gb = 0.0f, gw3 = 0.0f, gb3 = 0.0f;
  double lsum = 0.0;
  const int j2 = tid >> 1, k0 = (tid & 1) * 32;

  const int64_t ntiles = (n + kTile - 1) / kTile;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t b = tile * kTile + tid;
    float w = 0.0f, target = 0.0f;
    float x[kGuessIn];
    if (b < n) {
      const float* s = samples + (index ? index[b] : b) * 8;
#pragma unroll
      for (int k = 0; k < kGuessIn; ++k) x[k] = bf16r(s[k]);
      target = s[6];
      w = s[7];
    } else {
#pragma unroll
      for (int k = 0; k < kGuessIn; ++k) x[k] = 0.0f;
    }
#pragma unroll
    for (int k = 0; k < kGuessIn; ++k) S.x[tid][k] = x[k];
    // forward, row of sample tid
    unsigned long long m1 = 0ull, m2 = 0ull;  // ReLU masks
    for (int j = 0; j < kGuessHidden; ++j) {
      float z = S.b1[j];
#pragma unroll
      for (int k = 0; k < kGuessIn; ++k) z += x[k] * S.w1[k * kGuessHidden + j];
      if (z > 0.0f) m1 |= 1ull << j;
      S.h1[tid][j] = bf16r(fmaxf(z, 0.0f));
    }
    float z2[kGuessHidden];
#pragma unroll
    for (int k = 0; k < kGuessHidden; ++k) z2[k] = S.b2[k];
    for (int j = 0; j < kGuessHidden; ++j) {
      const float h = S.h1[tid][j];
      const float4* row = reinterpret_cast<const float4*>(&S.w2[j * kGuessHidden]);
#pragma unroll
      for (int q = 0; q < kGuessHidden / 4; ++q) {
        const float4 v = row[q];
        z2[4 * q + 0] += h * v.x;
        z2[4 * q + 1] += h * v.y;
        z2[4 * q + 2] += h * v.z;
        z2[4 * q + 3] += h * v.w;
      }
    }
    float y = S.b3;
#pragma unroll
    for (int k = 0; k < kGuessHidden; ++k) {
      if (z2[k] > 0.0f) m2 |= 1ull << k;
      const float h2 = bf16r(fmaxf(z2[k], 0.0f));
      S.h2[tid][k] = h2;
      y += h2 * S.w3[k];
    }
    const float err = y - target;
    const float dy = w * 2.0f * err * inv_count;
    lsum += (double)(w * err * err);
    S.dy[tid] = dy;
    // backward through layer 3 and the second ReLU
#pragma unroll
    for (int k = 0; k < kGuessHidden; ++k) {
      const float d = ((m2 >> k) & 1ull) ? dy * S.w3[k] : 0.0f;
      z2[k] = d;  // dz2
      S.dz2[tid][k] = d;
    }
    // through W2 and the first ReLU
    for (int j = 0; j < kGuessHidden; ++j) {
      const float4* row = reinterpret_cast<const float4*>(&S.w2[j * kGuessHidden]);
      float acc = 0.0f;
#pragma unroll
      for (int q = 0; q < kGuessHidden / 4; ++q) {
        const float4 v = row[q];
        acc += z2[4 * q + 0] * v.x + z2[4 * q + 1] * v.y + z2[4 * q + 2] * v.z +
               z2[4 * q + 3] * v.w;
      }
      S.dz1[tid][j] = ((m1 >> j) & 1ull) ? acc : 0.0f;
    }
    __syncthreads();
    // weight gradients of the tile: sums over its samples
    for (int bb = 0; bb < kTile; ++bb) {
      const float h = S.h1[bb][j2];
#pragma unroll
      for (int e = 0; e < 32; ++e) gw2[e] += h * S.dz2[bb][k0 + e];
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int id = tid + r * kTile;  // < 384
      const int i = id / kGuessHidden, j = id % kGuessHidden;
      float acc = 0.0f;
      for (int bb = 0; bb < kTile; ++bb) acc += S.x[bb][i] * S.dz1[bb][j];
      gw1[r] += acc;
    }
    if (tid < kGuessHidden) {
      float a1 = 0.0f, a3 = 0.0f;
      for (int bb = 0; bb < kTile; ++bb) {
        a1 += S.dz1[bb][tid];
        a3 += S.h2[bb][tid] * S.dy[bb];
      }
      gb += a1;
      gw3 += a3;
    } else {
      const int k = tid - kGuessHidden;
      float a2 = 0.0f;
      for (int bb = 0; bb < kTile; ++bb) a2 += S.dz2[bb][k];
      gb += a2;
      if (tid == kGuessHidden) {
        float a = 0.0f;
        for (int bb = 0; bb < kTile; ++bb) a += S.dy[bb];
        gb3 += a;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int e = 0; e < 32; ++e) atomicAdd(&grad[kOffW2 + j2 * kGuessHidden + k0 + e], gw2[e]);
#pragma unroll
  for (int r = 0; r < 3; ++r) atomicAdd(&grad[kOffW1 + tid + r * kTile], gw1[r]);
  if (tid < kGuessHidden) {
    atomicAdd(&grad[kOffB1 + tid], gb);
    atomicAdd(&grad[kOffW3 + tid], gw3);
  } else {
    atomicAdd(&grad[kOffB2 + tid - kGuessHidden], gb);
    if (tid == kGuessHidden) atomicAdd(&grad[kOffB3], gb3);
  }
  // loss: block sum
  __shared__ double s_loss[kTile / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((tid & 31) == 0) s_loss[tid >> 5] = lsum;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < kTile / 32; ++w) t += s_loss[w];
    atomicAdd(loss, t);
  }
}

// ---------------------------------------------------------------- Adam
__global__ void adam_kernel(float* __restrict__ W, float* __restrict__ grad,
                            float* __restrict__ m, float* __restrict__ v, int n, float lr,
                            float beta1, float beta2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gr = grad[i];
  const float mi = beta1 * m[i] + (1.0f - beta1) * gr;
  const float vi = beta2 * v[i] + (1.0f - beta2) * gr * gr;
  m[i] = mi;
  v[i] = vi;
  W[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  grad[i] = 0.0f;
}

// ---------------------------------------------------------------- inference alone
// The same warp-collective tensor-core evaluation the Riemann kernel runs, for checks.
__global__ void __launch_bounds__(256) eval_kernel(const uint32_t* __restrict__ packed,
                                                   const float* __restrict__ feats, int64_t n,
                                                   float* __restrict__ y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float f[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  if (i < n)
    for (int k = 0; k < 6; ++k) f[k] = feats[i * 6 + k];
  const float out = guess_mlp_warp(packed, f);  // every lane of the warp takes part
  if (i < n) y[i] = out;
}

}  // namespace mlp

size_t guess_grad_smem_bytes() { return sizeof(mlp::GradSmem); }

cudaError_t launch_guess_features(const double* rec, int64_t n, double gamma, double pmin,
                                  float* out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  int64_t blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  mlp::features_kernel<<<(unsigned)blocks, 256, 0, st>>>(rec, n, gamma, pmin, out);
  return cudaGetLastError();
}

cudaError_t launch_guess_grad(const float* W, const float* samples, const int64_t* index,
                              int64_t n, float inv_count, float* grad, double* loss, int blocks,
                              cudaStream_t st) {
  const size_t smem = sizeof(mlp::GradSmem);
  cudaError_t e = cudaFuncSetAttribute(mlp::grad_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (n <= 0) return cudaSuccess;
  const int64_t ntiles = (n + mlp::kTile - 1) / mlp::kTile;
  if ((int64_t)blocks > ntiles) blocks = (int)ntiles;
  mlp::grad_kernel<<<blocks, mlp::kTile, smem, st>>>(W, samples, index, n, inv_count, grad, loss);
  return cudaGetLastError();
}

cudaError_t launch_guess_adam(float* W, float* grad, float* m, float* v, int step, float lr,
                              float beta1, float beta2, float eps, cudaStream_t st) {
  const float c1 = 1.0f - powf(beta1, (float)step);
  const float c2 = 1.0f - powf(beta2, (float)step);
  mlp::adam_kernel<<<(kGuessWeights + 255) / 256, 256, 0, st>>>(W, grad, m, v, kGuessWeights,
                                                                  lr, beta1, beta2, eps, c1, c2);
  return cudaGetLastError();
}

cudaError_t launch_guess_eval(const uint32_t* packed, const float* feats, int64_t n, float* y,
                              cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  mlp::eval_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(packed, feats, n, y);
  return cudaGetLastError();
}

}  // namespace ppm
