// ppm_guess.cuh -- the learned starting pressure of twoshock's Newton iteration.
//
// twoshock.F:156-170 starts the iteration for the star-state pressure p* from the
// acoustic (linearised) estimate.  A small MLP (6 -> 64 -> 64 -> 1, ReLU) predicts the
// remaining factor ln(p* / p_acoustic) from the two interface states, so the iteration
// can start closer to p*.  The acoustic estimate is exact for equal states and its
// error grows with the square of the jump, so the net predicts the coefficient
//   r = ln(p* / p_acoustic) / |x|^2,   |x|^2 = sum of the squared inputs,
// and the start is p_acoustic * exp(|x|^2 r): for weak jumps the start is then at least
// as close as the acoustic one, whatever the net's BF16 resolution.  Newton then
// refines to the reference tolerance as before; if it does not converge within the
// reference's iteration limit, the face is re-solved from the acoustic estimate, which
// reproduces the plain solver exactly.
//
// Inputs (the interface states normalised by their mean, rho_m = (dl + dr) / 2,
// p_m = (pl + pr) / 2, u_m = (ul + ur) / 2, c_m = sqrt(gamma p_m / rho_m)):
//   ln(dl / rho_m), ln(dr / rho_m), (ul - u_m) / c_m, (ur - u_m) / c_m,
//   ln(pl / p_m), ln(pr / p_m)
//
// Inference runs on the tensor cores inside the Riemann kernel: one warp evaluates the
// net for its 32 faces with BF16 operands and FP32 accumulation (two 16-row tiles per
// layer, the accumulator of one layer re-packed in registers as the operand of the
// next).  Training uses the same rounding (inputs, weights and hidden activations
// rounded to BF16, FP32 sums), so the trained weights are the ones inference sees.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

#include "ppm_device.cuh"

namespace ppm {

enum { kGuessIn = 6, kGuessHidden = 64 };

// Below this |x|^2 for all 32 faces of a warp the net is not evaluated: the acoustic
// start is then already within about |x|^2 |r| (|r| of order 0.1) of p*, which leaves
// too little for the net to save to pay for its evaluation.
constexpr float kGuessMinJump = 1.0e-4f;

// FP32 master weights, flat: W1 [6][64] (input-major), b1 [64], W2 [64][64], b2 [64],
// w3 [64], b3 [1]
enum {
  kOffW1 = 0,
  kOffB1 = kOffW1 + kGuessIn * kGuessHidden,
  kOffW2 = kOffB1 + kGuessHidden,
  kOffB2 = kOffW2 + kGuessHidden * kGuessHidden,
  kOffW3 = kOffB2 + kGuessHidden,
  kOffB3 = kOffW3 + kGuessHidden,
  kGuessWeights = kOffB3 + 1  // 4673
};

// Inference weights in the register order of mma.m16n8k16 B fragments (bf16 pairs):
//   layer 1: [n-tile 8][lane 32][2]           (K = 16: the 6 inputs, zero padded)
//   layer 2: [k-step 4][n-tile 8][lane 32][2]
//   layer 3: [k-step 4][lane 32][2]           (N = 8: w3 in column 0, zeros elsewhere)
//   then b1 [64], b2 [64], b3 as FP32 bit patterns
enum {
  kPackL1 = 0,
  kPackL2 = kPackL1 + 8 * 32 * 2,
  kPackL3 = kPackL2 + 4 * 8 * 32 * 2,
  kPackB1 = kPackL3 + 4 * 32 * 2,
  kPackB2 = kPackB1 + kGuessHidden,
  kPackB3 = kPackB2 + kGuessHidden,
  kPackWords = kPackB3 + 4
};

// The same weights for the tcgen05 kernels (ppm_guess_tc.cu), after the packed words in
// the same device buffer (word offset kTcWordOffset), bytes: W1 and W2 as the MMA's B
// operands (N x K, K-major, bf16, the canonical layout without swizzle: element (n, k) at
// ((k/8) * (N/8) + n/8) * 128 + (n%8) * 16 + (k%8) * 2), then b1, b2, w3 (its bf16 value)
// and b3 as FP32.
enum {
  kTcW1 = 0,                    // 64 x 16 (the 6 inputs, zero padded)
  kTcW2 = kTcW1 + 64 * 16 * 2,  // 64 x 64
  kTcB1 = kTcW2 + 64 * 64 * 2,
  kTcB2 = kTcB1 + 64 * 4,
  kTcW3 = kTcB2 + 64 * 4,
  kTcB3 = kTcW3 + 64 * 4,
  kTcBytes = kTcB3 + 16,
  kTcWordOffset = ((kPackWords + 255) / 256) * 256,
  kGuessBufferWords = kTcWordOffset + kTcBytes / 4
};

// Interface-state features of one face (see the header comment); returns |x|^2.  FP32
// arithmetic on the FP32 pipe: the net sees its inputs rounded to BF16, so FP64 logs
// and divides (which would load the FP64 pipe the Newton iteration is bound by) buy
// nothing.  Training computes the features with this same function.
__device__ __forceinline__ float guess_features(double dl, double dr, double pl, double pr,
                                                double ul, double ur, double gamma, float f[6]) {
  const float dlf = (float)dl, drf = (float)dr, plf = (float)pl, prf = (float)pr;
  const float ulf = (float)ul, urf = (float)ur;
  const float rho = 0.5f * (dlf + drf);
  const float p = 0.5f * (plf + prf);
  const float u = 0.5f * (ulf + urf);
  const float ic = 1.0f / sqrtf((float)gamma * p / rho);
  f[0] = logf(dlf / rho);
  f[1] = logf(drf / rho);
  f[2] = (ulf - u) * ic;
  f[3] = (urf - u) * ic;
  f[4] = logf(plf / p);
  f[5] = logf(prf / p);
  float d2 = 0.0f;
  for (int k = 0; k < 6; ++k) d2 += f[k] * f[k];
  return d2;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x (lo) in the low half
  return *reinterpret_cast<const uint32_t*>(&v);
}

// D = A (16x16, row) * B (16x8, col) + D, bf16 operands, fp32 accumulate
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], uint32_t a0, uint32_t a1,
                                               uint32_t a2, uint32_t a3, uint32_t b0,
                                               uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Warp-collective: every lane passes the features of its own face (zeros for a lane
// without a face) and gets y for that face.  All 32 lanes must call it.
//   Fragment layout (g = lane / 4, t = lane % 4): A rows g and g+8, columns 2t, 2t+1
//   (regs 0, 1) and 2t+8, 2t+9 (regs 2, 3); B column g, rows 2t, 2t+1 and 2t+8, 2t+9;
//   C rows g and g+8, columns 2t, 2t+1.
__device__ __forceinline__ float guess_mlp_warp(const uint32_t* __restrict__ W, const float f[6]) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const float* bias1 = reinterpret_cast<const float*>(W + kPackB1);
  const float* bias2 = reinterpret_cast<const float*>(W + kPackB2);
  const float b3 = __uint_as_float(__ldg(W + kPackB3));
  const uint32_t p0 = pack_bf16x2(f[0], f[1]);
  const uint32_t p1 = pack_bf16x2(f[2], f[3]);
  const uint32_t p2 = pack_bf16x2(f[4], f[5]);
  float y = 0.0f;
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    // layer-1 operand: feature pair t of faces 16m + g and 16m + g + 8
    const int s0 = 16 * m + g, s1 = s0 + 8;
    const uint32_t q0 = __shfl_sync(full, p0, s0), q1 = __shfl_sync(full, p1, s0),
                   q2 = __shfl_sync(full, p2, s0);
    const uint32_t r0 = __shfl_sync(full, p0, s1), r1 = __shfl_sync(full, p1, s1),
                   r2 = __shfl_sync(full, p2, s1);
    const uint32_t a0 = t == 0 ? q0 : (t == 1 ? q1 : (t == 2 ? q2 : 0u));
    const uint32_t a1 = t == 0 ? r0 : (t == 1 ? r1 : (t == 2 ? r2 : 0u));
    uint32_t h1[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      float c[2][4];
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) {
        const int n = 2 * kk + jj;
        const float bl = __ldg(bias1 + 8 * n + 2 * t), bh = __ldg(bias1 + 8 * n + 2 * t + 1);
        c[jj][0] = bl; c[jj][1] = bh; c[jj][2] = bl; c[jj][3] = bh;
        const uint32_t* wb = W + kPackL1 + (n * 32 + lane) * 2;
        mma_bf16_16816(c[jj], a0, a1, 0u, 0u, __ldg(wb), __ldg(wb + 1));
#pragma unroll
        for (int e = 0; e < 4; ++e) c[jj][e] = fmaxf(c[jj][e], 0.0f);
      }
      h1[kk][0] = pack_bf16x2(c[0][0], c[0][1]);
      h1[kk][1] = pack_bf16x2(c[0][2], c[0][3]);
      h1[kk][2] = pack_bf16x2(c[1][0], c[1][1]);
      h1[kk][3] = pack_bf16x2(c[1][2], c[1][3]);
    }
    uint32_t h2[4][4];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
      float c[2][4];
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) {
        const int n = 2 * k2 + jj;
        const float bl = __ldg(bias2 + 8 * n + 2 * t), bh = __ldg(bias2 + 8 * n + 2 * t + 1);
        c[jj][0] = bl; c[jj][1] = bh; c[jj][2] = bl; c[jj][3] = bh;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const uint32_t* wb = W + kPackL2 + ((kk * 8 + n) * 32 + lane) * 2;
          mma_bf16_16816(c[jj], h1[kk][0], h1[kk][1], h1[kk][2], h1[kk][3], __ldg(wb),
                         __ldg(wb + 1));
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) c[jj][e] = fmaxf(c[jj][e], 0.0f);
      }
      h2[k2][0] = pack_bf16x2(c[0][0], c[0][1]);
      h2[k2][1] = pack_bf16x2(c[0][2], c[0][3]);
      h2[k2][2] = pack_bf16x2(c[1][0], c[1][1]);
      h2[k2][3] = pack_bf16x2(c[1][2], c[1][3]);
    }
    float c3[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const uint32_t* wb = W + kPackL3 + (kk * 32 + lane) * 2;
      mma_bf16_16816(c3, h2[kk][0], h2[kk][1], h2[kk][2], h2[kk][3], __ldg(wb), __ldg(wb + 1));
    }
    // column 0 of rows g (c3[0]) and g + 8 (c3[2]) sits in lane 4g; route it to the
    // lane that owns the face
    const int src = (lane & 7) * 4;
    const float v0 = __shfl_sync(full, c3[0], src);
    const float v2 = __shfl_sync(full, c3[2], src);
    if ((lane >> 4) == m) y = ((lane & 15) < 8 ? v0 : v2) + b3;
  }
  return y;
}

// The starting pressure from the net output r and |x|^2 (clamped so that a poor
// prediction costs Newton iterations, never a non-finite start).  The factor is an FP32
// exponential: the start only has to be close, Newton refines it to the tolerance.
__device__ __forceinline__ double guess_pressure(double p_acoustic, float r, float d2,
                                                 double pmin) {
  float yc = fminf(fmaxf(d2 * r, -8.0f), 8.0f);
  if (!(yc == yc)) yc = 0.0f;
  double ps = p_acoustic * (double)expf(yc);
  if (!(ps >= pmin)) ps = pmin;
  return ps;
}

}  // namespace ppm
