// ppm_guess_tc.cu -- the learned-start net (ppm_guess.cuh) on the fifth-generation tensor
// cores: tcgen05.mma with the accumulators in tensor memory.
//
// A CTA is one warpgroup (128 threads) and takes tiles of 128 rows (faces or samples):
// thread r writes row r's six features, rounded to BF16, into shared memory as the A
// operand of layer 1 (M = 128, K = 16, zero padded); one elected thread issues the MMA
// against W1 (N = 64) into tensor-memory columns 0-63 and commits it to an mbarrier;
// every thread loads its row of the accumulator (tcgen05.ld 32x32b: warp w reads lanes
// 32w .. 32w+31), adds b1, applies the ReLU, rounds to BF16 and writes it back to
// shared memory as layer 2's A operand (K = 64); four MMAs (K = 16 each) against W2 go
// to columns 64-127; the final layer (64 -> 1) and b3 are a dot product on the FP32 pipe
// from the row's second accumulator, after its bias, ReLU and BF16 rounding -- the
// rounding the mma.sync evaluation and the training apply.  Operands use the canonical
// K-major layout without swizzle (8-row x 16-byte core matrices); the weights stay in
// shared memory for every tile of a persistent CTA.  No cluster, no multicast.
//
// Waits on the mbarrier are bounded: after about a second the CTA records a timeout
// (the caller's status), stops issuing work and frees its tensor memory.
#include <cuda_runtime.h>

#include <cstdint>

#include "ppm_guess.cuh"
#include "ppm_sweep.cuh"

namespace ppm {
namespace gtc {

constexpr int kRows = 128;      // rows per tile: the MMA's M, one per thread
constexpr int kTmemCols = 128;  // layer 1 in columns 0-63, layer 2 in 64-127
// shared memory (bytes, from a 1024-byte aligned base)
constexpr int kSmW = 0;                         // the weights image (kTcBytes)
constexpr int kSmX = 11264;                     // A of layer 1: 128 x 16 bf16
constexpr int kSmH = kSmX + kRows * 16 * 2;     // A of layer 2: 128 x 64 bf16
constexpr int kSmBar = kSmH + kRows * 64 * 2;   // mbarrier
constexpr int kSmTmem = kSmBar + 8;             // tensor-memory address from tcgen05.alloc
constexpr int kSmBytes = kSmTmem + 8;
constexpr int kSmAlloc = kSmBytes + 1024;       // room to align the base
static_assert(kTcBytes <= kSmX, "weights image");
constexpr long long kWaitCycles = 2000000000ll;  // ~1 s

// instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D, M = 128, N = 64
constexpr uint32_t kIdesc = (1u << 4)            // D format F32
                            | (1u << 7)          // A format BF16
                            | (1u << 10)         // B format BF16
                            | ((64u >> 3) << 17) // N
                            | ((128u >> 4) << 24);  // M

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: canonical K-major layout without swizzle; lbo: bytes
// between the two 8-element K halves of an MMA's K = 16, sbo: bytes between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;  // descriptor version of sm_100
  return d;                 // base offset 0, layout type 0 (no swizzle)
}

// Byte offset of element (row, k) of an operand of `rows` rows in the canonical layout.
__device__ __forceinline__ int canon(int rows, int row, int k) {
  return ((k >> 3) * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %4, {%5, %5, %5, %5}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(accumulate), "r"(kIdesc), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ bool bar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
  if (bar_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (!bar_try(bar, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}

// 64 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
  uint32_t r[64];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
      "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
      "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]),
        "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]),
        "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]),
        "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]),
        "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]),
        "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) { return pack_bf16x2(lo, hi); }
__device__ __forceinline__ float bf16_round(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

// The tiles of one launch: rows come from `row_features` (features of a row, false when
// the row has none) and results go to `row_result`.
struct Net {
  unsigned char* sm;   // aligned shared memory
  uint32_t tmem;       // tensor-memory base (lane 0, column 0)
  uint64_t* bar;
  uint32_t phase;      // completed MMA groups, for the mbarrier parity
  bool broken;
};

// CTA-wide: load the weights image, allocate tensor memory, set up the mbarrier.
__device__ __forceinline__ void net_begin(Net& N, const uint32_t* __restrict__ words,
                                          unsigned char* raw) {
  const uintptr_t base = (reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023);
  N.sm = reinterpret_cast<unsigned char*>(base);
  N.bar = reinterpret_cast<uint64_t*>(N.sm + kSmBar);
  N.phase = 0;
  N.broken = false;
  const uint4* src = reinterpret_cast<const uint4*>(words + kTcWordOffset);
  uint4* dst = reinterpret_cast<uint4*>(N.sm + kSmW);
  for (int i = threadIdx.x; i < kTcBytes / 16; i += blockDim.x) dst[i] = __ldg(src + i);
  if (threadIdx.x < 32) {  // warp 0 owns the tensor memory
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(N.sm + kSmTmem)),
                 "r"((uint32_t)kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(N.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_async_smem();  // the weights, written by the generic proxy, feed the MMAs
  fence_before();
  __syncthreads();
  fence_after();
  N.tmem = *reinterpret_cast<volatile uint32_t*>(N.sm + kSmTmem);
}

__device__ __forceinline__ void net_end(Net& N) {
  fence_before();
  __syncthreads();
  fence_after();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(N.tmem),
                 "r"((uint32_t)kTmemCols)
                 : "memory");
}

// One tile: this thread's row features f (valid: the row exists); returns the net
// output for the row.  CTA-wide; every thread calls it for every tile.
__device__ __forceinline__ float net_tile(Net& N, const float f[6], bool valid,
                                          unsigned long long* timeouts) {
  const int r = threadIdx.x;
  unsigned char* sm = N.sm;
  // layer 1's A operand: row r = the six features (BF16), zero padded to K = 16
  {
    uint4 lo = make_uint4(0u, 0u, 0u, 0u);
    if (valid) {
      lo.x = bf16x2(f[0], f[1]);
      lo.y = bf16x2(f[2], f[3]);
      lo.z = bf16x2(f[4], f[5]);
    }
    *reinterpret_cast<uint4*>(sm + kSmX + canon(kRows, r, 0)) = lo;
    *reinterpret_cast<uint4*>(sm + kSmX + canon(kRows, r, 8)) = make_uint4(0u, 0u, 0u, 0u);
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t xa = smem_addr(sm + kSmX), ha = smem_addr(sm + kSmH);
  const uint32_t w1 = smem_addr(sm + kSmW + kTcW1), w2 = smem_addr(sm + kSmW + kTcW2);
  if (r == 0 && !N.broken) {
    mma_bf16(N.tmem, smem_desc(xa, (kRows / 8) * 128, 128), smem_desc(w1, (64 / 8) * 128, 128),
             0u);
    mma_commit(N.bar);
  }
  bool ok = N.broken ? false : bar_wait(N.bar, N.phase & 1u);
  N.phase += 1;
  if (__syncthreads_or(!ok)) N.broken = true;
  fence_after();
  const float* fb1 = reinterpret_cast<const float*>(sm + kSmW + kTcB1);
  const float* fb2 = reinterpret_cast<const float*>(sm + kSmW + kTcB2);
  const float* fw3 = reinterpret_cast<const float*>(sm + kSmW + kTcW3);
  const uint32_t lane_base = (uint32_t)((r >> 5) * 32) << 16;  // this warp's 32 lanes
  float acc[64];
  if (!N.broken) {
    tmem_ld64(N.tmem + lane_base, acc);
    // layer 2's A operand: row r = relu(acc + b1), BF16, eight 16-byte chunks
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      float h[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) h[e] = fmaxf(acc[8 * c + e] + fb1[8 * c + e], 0.0f);
      *reinterpret_cast<uint4*>(sm + kSmH + canon(kRows, r, 8 * c)) =
          make_uint4(bf16x2(h[0], h[1]), bf16x2(h[2], h[3]), bf16x2(h[4], h[5]),
                     bf16x2(h[6], h[7]));
    }
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  if (r == 0 && !N.broken) {
#pragma unroll
    for (int s = 0; s < 4; ++s)  // K = 64 as four K = 16 steps (two 8-element chunks each)
      mma_bf16(N.tmem + 64, smem_desc(ha + 2 * s * (kRows / 8) * 128, (kRows / 8) * 128, 128),
               smem_desc(w2 + 2 * s * (64 / 8) * 128, (64 / 8) * 128, 128), s > 0 ? 1u : 0u);
    mma_commit(N.bar);
  }
  ok = N.broken ? false : bar_wait(N.bar, N.phase & 1u);
  N.phase += 1;
  if (__syncthreads_or(!ok)) {
    if (!N.broken && threadIdx.x == 0 && timeouts) atomicAdd(timeouts, 1ull);
    N.broken = true;
  }
  fence_after();
  float y = 0.0f;
  if (!N.broken) {
    tmem_ld64(N.tmem + 64 + lane_base, acc);
#pragma unroll
    for (int j = 0; j < 64; ++j) y += bf16_round(fmaxf(acc[j] + fb2[j], 0.0f)) * fw3[j];
    y += *reinterpret_cast<const float*>(sm + kSmW + kTcB3);
  }
  fence_before();
  __syncthreads();  // the tile's shared operands and accumulators are free again
  fence_after();
  return y;
}

// Inference alone: y[i] = net(features[i]) for n rows (6 floats each).
__global__ void __launch_bounds__(kRows) eval_tc_kernel(const uint32_t* __restrict__ words,
                                                        const float* __restrict__ feats,
                                                        int64_t n, float* __restrict__ y,
                                                        unsigned long long* timeouts) {
  extern __shared__ unsigned char raw[];
  Net N;
  net_begin(N, words, raw);
  const int64_t ntiles = (n + kRows - 1) / kRows;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t i = t * kRows + threadIdx.x;
    float f[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    const bool valid = i < n;
    if (valid)
      for (int k = 0; k < 6; ++k) f[k] = feats[i * 6 + k];
    const float out = net_tile(N, f, valid, timeouts);
    if (valid && !N.broken) y[i] = out;
  }
  net_end(N);
}

// The guess pass of a sweep with the learned start on the tensor cores: every face of
// the batch (a tile = the 128 pencils of one face plane that a Riemann block takes, the
// Riemann prefix table with 128 faces per block) gets its features from the interface
// states and the net's output; (y, |x|^2) go into the face's slot of the XUB flux plane,
// which the Riemann kernel reads before it writes the Godunov velocity there.
template <bool ONE>
__global__ void __launch_bounds__(kRows) guess_pass_kernel(const __grid_constant__ BatchArgs B) {
  extern __shared__ unsigned char raw[];
  __shared__ SweepArgs s_rec;
  Net N;
  const SweepArgs& first = ONE ? B.one : B.grids[0];
  net_begin(N, first.guess, raw);
  int cur = -1;
  for (int64_t blk = blockIdx.x; blk < B.riemann_total; blk += gridDim.x) {
    int64_t lb = blk;
    const int g = ONE ? 0 : batch_locate(B.riemann_prefix, B.ngrids, blk, lb);
    if (!ONE && g != cur) {
      __syncthreads();
      const unsigned long long* src = reinterpret_cast<const unsigned long long*>(B.grids + g);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(&s_rec);
      for (int i = threadIdx.x; i < (int)(sizeof(SweepArgs) / 8); i += blockDim.x)
        dst[i] = __ldg(src + i);
      cur = g;
    }
    __syncthreads();
    const SweepArgs& a = ONE ? B.one : s_rec;
    const int64_t chunks = (a.npencils + kRows - 1) / kRows;
    const int fi = (int)(lb / chunks);
    const int64_t pid = (lb - (int64_t)fi * chunks) * kRows + threadIdx.x;
    const bool valid = pid < a.npencils;
    const int64_t idx = (int64_t)fi * a.npencils + pid;
    float f[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    float d2 = 0.0f;
    if (valid) {
      const double* st = a.fstate + idx;
      const int64_t pl = a.plane;
      d2 = guess_features(st[0 * pl], st[1 * pl], st[2 * pl], st[3 * pl], st[4 * pl],
                          st[5 * pl], a.gamma, f);  // dl dr pl pr ul ur
    }
    const float y = net_tile(N, f, valid, B.counters + kCntTimeout);
    if (valid) {
      float2 v = make_float2(N.broken ? 0.0f : y, N.broken ? 0.0f : d2);
      *reinterpret_cast<float2*>(a.fflux + 6 * a.plane + idx) = v;  // the XUB plane
    }
  }
  net_end(N);
}

}  // namespace gtc

cudaError_t launch_guess_eval_tc(const uint32_t* words, const float* feats, int64_t n, float* y,
                                 unsigned long long* timeouts, int sms, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(gtc::eval_tc_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         gtc::kSmAlloc);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int64_t ntiles = (n + gtc::kRows - 1) / gtc::kRows;
  const int64_t grid = ntiles < (int64_t)sms * 4 ? ntiles : (int64_t)sms * 4;
  gtc::eval_tc_kernel<<<(unsigned)grid, gtc::kRows, gtc::kSmAlloc, st>>>(words, feats, n, y,
                                                                         timeouts);
  return cudaGetLastError();
}

void launch_guess_pass(const BatchArgs& B, int sms, cudaStream_t st) {
  static bool attr[2] = {false, false};
  const int one = B.ngrids == 1 ? 1 : 0;
  if (!attr[one]) {
    if (one)
      cudaFuncSetAttribute(gtc::guess_pass_kernel<true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, gtc::kSmAlloc);
    else
      cudaFuncSetAttribute(gtc::guess_pass_kernel<false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, gtc::kSmAlloc);
    attr[one] = true;
  }
  const int64_t grid = B.riemann_total < (int64_t)sms * 4 ? B.riemann_total : (int64_t)sms * 4;
  if (grid <= 0) return;
  if (one)
    gtc::guess_pass_kernel<true><<<(unsigned)grid, gtc::kRows, gtc::kSmAlloc, st>>>(B);
  else
    gtc::guess_pass_kernel<false><<<(unsigned)grid, gtc::kRows, gtc::kSmAlloc, st>>>(B);
}

}  // namespace ppm
