// ppm_noalloc.cu -- ppm_b200_euler_sweep_static: one directional sweep that allocates
// nothing.
//
// Some callers cannot allocate device memory at the moment they want to advance a
// grid: code that runs under a memory pool or arena that owns all device memory and
// forbids further cudaMalloc calls, code inside a callback where allocating could
// synchronise the device or deadlock, or embedded drivers that reserve all memory up
// front.  Such a caller still provides its own input and output arrays; this entry
// point takes the sweep's scratch (the interface-state and flux planes, the inteuler
// coefficient table, the grid record the kernels read and the status counters) from a fixed array compiled into the
// library instead of from cudaMalloc.
//
// Properties a caller must know:
//  * Limit: the face planes fit kStaticPlaneBytes (48 MiB), i.e.
//    (19 * 8 * (active cells along the sweep + 1) + 8) * (pencils) bytes; this covers grids
//    up to 64^3 active cells (70^3 with ghosts) in every direction.  Larger grids and
//    pencils longer than 1031 cells are rejected with PPM_B200_ERR_TOO_LARGE before
//    any device work.
//  * Every GPU that loads the library holds the array (about 48.1 MiB) until the
//    process exits.
//  * Set-up: the first call in a CUDA context (a device's primary context, current on
//    the calling thread) looks up the array's device address with cudaGetSymbolAddress
//    and keeps it for that context; a new context (after cudaDeviceReset, or another
//    device) looks it up again.
//  * Never call it while its stream is being captured into a CUDA graph: it copies from
//    pageable host memory and waits for its stream, which a capture cannot contain.  It
//    checks this first and returns PPM_B200_ERR_INVALID without touching the stream.
//  * Outputs must not overlap the inputs or the pressure (the kernels read their
//    inputs as read-only, non-aliased data); an overlapping call, such as an in-place
//    sweep, returns PPM_B200_ERR_INVALID.
//  * The array is shared by every call on a device and keeps the last call's
//    contents.  Calls that overlap on the GPU (different streams, or different host
//    threads) race on it; serialise them.
//  * The call is synchronous: it waits for its own stream to read the status.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "ppm_b200.h"
#include "ppm_sweep.cuh"

namespace ppm {
void launch_sweep_batch(const BatchArgs& B, int64_t march_blocks, int64_t riemann_blocks,
                        bool dual, bool grav, cudaStream_t st, cudaEvent_t* ev, bool learned,
                        bool contiguous);
}

namespace {

constexpr size_t kStaticCounterBytes = 256;                       // kMaxCounters counters
constexpr int kStaticCoefEntries = 1031;                          // longest pencil (fortran.def:1)
constexpr size_t kStaticCoefBytes = 66560;                        // >= 1031 * sizeof(Coef), 256-aligned
constexpr size_t kStaticDescBytes = 1024;                         // grid record + block prefixes
constexpr size_t kStaticPlaneBytes = size_t(48) << 20;            // interface states + fluxes
constexpr size_t kStaticBytes =
    kStaticCounterBytes + kStaticCoefBytes + kStaticDescBytes + kStaticPlaneBytes;
static_assert(kStaticCoefEntries * sizeof(ppm::Coef) <= kStaticCoefBytes, "coef area");
static_assert(sizeof(ppm::SweepArgs) <= 512, "descriptor area");
static_assert(ppm::kMaxCounters * sizeof(unsigned long long) <= kStaticCounterBytes, "counters");

constexpr int kMaxDevices = 64;

struct DeviceSlot {
  void* context = nullptr;       // the CUDA context the address belongs to
  unsigned char* base = nullptr;
};
DeviceSlot g_slots[kMaxDevices];
std::mutex g_setup_mutex;

// cuCtxGetCurrent through the runtime's driver entry point (no link against libcuda)
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctx_get_current() {
  static const CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  return fn;
}

}  // namespace

// The scratch itself.  Host code must not use this name as an address: it is a
// host-side stand-in for the device array; the device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_sweep_scratch[kStaticBytes];

namespace {

// Once per device and CUDA context, with that device current: look up the array's
// device address.  The address is kept with the context it belongs to; when the
// device's context changes (cudaDeviceReset unloads the module), it is looked up again.
int static_setup(int device, unsigned char** base) {
  if (device < 0 || device >= kMaxDevices) return PPM_B200_ERR_INVALID;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSlot& s = g_slots[device];
  void* current = nullptr;
  const CtxGetCurrentFn get = ctx_get_current();
  if (get) get(&current);  // no context yet: looked up below, which creates it
  if (!s.base || !current || current != s.context) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_sweep_scratch);
    if (e != cudaSuccess || p == nullptr) {
      fprintf(stderr, "ppm_b200: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return PPM_B200_ERR_CUDA;
    }
    s.base = static_cast<unsigned char*>(p);
    s.context = nullptr;
    if (get) get(&s.context);
  }
  *base = s.base;
  return PPM_B200_OK;
}

// true when [a, a + n) and [b, b + n) overlap (n doubles each)
bool overlaps(const double* a, const double* b, int64_t n) {
  if (!a || !b) return false;
  return a < b + n && b < a + n;
}

int fail_cuda(cudaError_t e, const char* what) {
  fprintf(stderr, "ppm_b200: %s failed: %s\n", what, cudaGetErrorString(e));
  return PPM_B200_ERR_CUDA;
}

}  // namespace

extern "C" int ppm_b200_euler_sweep_static(int dim, const ppm_b200_params* p,
                                           const ppm_b200_grid* in, const double* pressure,
                                           ppm_b200_grid* out, void* cuda_stream,
                                           ppm_b200_stats* stats) {
  // ---- argument checks (no device work yet)
  if (!p || !in || !out || !pressure || dim < 0 || dim > 2) return PPM_B200_ERR_INVALID;
  if (p->pressure_free || p->steepening || p->flattening || p->diffusion || p->conservative_rec ||
      p->positive_rec || p->eos_type != 0 || p->number_of_colours != 0 || p->learned_guess ||
      p->riemann_solver != PPM_B200_RIEMANN_TWOSHOCK ||
      p->reconstruction != PPM_B200_RECONSTRUCTION_PPM)
    return PPM_B200_ERR_UNSUPPORTED;
  if (in->rank < 1 || in->rank > 3 || dim >= in->rank) return PPM_B200_ERR_INVALID;
  for (int d = 0; d < 3; ++d)
    if (out->dims[d] != in->dims[d] || (d >= in->rank && in->dims[d] != 1))
      return PPM_B200_ERR_INVALID;
  if (in->start[dim] != 3 || in->dims[dim] - 1 - in->end[dim] != 3 || !in->cell_width[dim])
    return PPM_B200_ERR_INVALID;
  if (!in->density || !in->total_energy || !in->velocity[0] || !out->density ||
      !out->total_energy || !out->velocity[0])
    return PPM_B200_ERR_INVALID;
  for (int d = 1; d < in->rank; ++d)
    if (!in->velocity[d] || !out->velocity[d]) return PPM_B200_ERR_INVALID;
  if (p->dual_energy && (!in->gas_energy || !out->gas_energy)) return PPM_B200_ERR_INVALID;
  if (p->gravity && !in->acceleration[dim]) return PPM_B200_ERR_INVALID;
  {  // outputs must not overlap any input (the kernels read inputs as non-aliased)
    const int64_t cells = (int64_t)in->dims[0] * in->dims[1] * in->dims[2];
    const double* ins[7] = {in->density, in->total_energy, in->velocity[0], in->velocity[1],
                            in->velocity[2], in->gas_energy, pressure};
    const double* outs[6] = {out->density, out->total_energy,
                             out->velocity[0], in->rank > 1 ? out->velocity[1] : nullptr,
                             in->rank > 2 ? out->velocity[2] : nullptr,
                             p->dual_energy ? out->gas_energy : nullptr};
    for (const double* o : outs)
      for (const double* i : ins)
        if (overlaps(o, i, cells)) return PPM_B200_ERR_INVALID;
  }

  const int GD0 = in->dims[0], GD1 = in->dims[1], GD2 = in->dims[2];
  ppm::SweepArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n = in->dims[dim];
  a.is = in->start[dim];
  a.ie = in->end[dim];
  if (dim == 0) {
    a.n1 = GD1; a.n2 = GD2; a.s1 = GD0; a.s2 = (int64_t)GD0 * GD1; a.sa = 1;
  } else if (dim == 1) {
    a.n1 = GD0; a.n2 = GD2; a.s1 = 1; a.s2 = (int64_t)GD0 * GD1; a.sa = GD0;
  } else {
    a.n1 = GD0; a.n2 = GD1; a.s1 = 1; a.s2 = GD0; a.sa = (int64_t)GD0 * GD1;
  }
  a.npencils = (int64_t)a.n1 * a.n2;
  a.plane = (int64_t)(a.ie - a.is + 2) * a.npencils;
  const size_t plane_bytes =
      (size_t)(ppm::kFaceVars + ppm::kFluxVars) * (size_t)a.plane * sizeof(double) +
      (size_t)a.npencils * sizeof(int64_t);
  if (a.n > kStaticCoefEntries || plane_bytes > kStaticPlaneBytes) return PPM_B200_ERR_TOO_LARGE;

  // ---- never under stream capture: checked before anything touches the stream
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
      return PPM_B200_ERR_INVALID;
  }

  // ---- set-up of this device and context (first call only), with the caller's device
  // current
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return fail_cuda(e, "cudaGetDevice");
  unsigned char* base = nullptr;
  int rc = static_setup(device, &base);
  if (rc) return rc;
  unsigned long long* counters = reinterpret_cast<unsigned long long*>(base);
  ppm::Coef* coef = reinterpret_cast<ppm::Coef*>(base + kStaticCounterBytes);
  unsigned char* desc = base + kStaticCounterBytes + kStaticCoefBytes;
  double* planes = reinterpret_cast<double*>(desc + kStaticDescBytes);

  // ---- per-call contents: counters start at zero, the coefficient table is rewritten
  e = cudaMemsetAsync(counters, 0, kStaticCounterBytes, st);
  if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync");
  std::vector<ppm::Coef> table;
  ppm::build_coef(in->cell_width[dim], a.n, a.is, a.ie, table);
  e = cudaMemcpyAsync(coef, table.data(), table.size() * sizeof(ppm::Coef),
                      cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyAsync");

  const int vu = dim, vv = (dim + 1) % 3, vw = (dim + 2) % 3;
  auto vin = [&](int c) -> const double* { return c < in->rank ? in->velocity[c] : nullptr; };
  auto vout = [&](int c) -> double* { return c < in->rank ? out->velocity[c] : nullptr; };
  a.in_d = in->density;
  a.in_e = in->total_energy;
  a.in_u = vin(vu);
  a.in_v = vin(vv);
  a.in_w = vin(vw);
  a.in_ge = p->dual_energy ? in->gas_energy : nullptr;
  a.out_d = out->density;
  a.out_e = out->total_energy;
  a.out_u = vout(vu);
  a.out_v = vout(vv);
  a.out_w = vout(vw);
  a.out_ge = p->dual_energy ? out->gas_energy : nullptr;
  a.pres = pressure;
  a.grav = p->gravity ? in->acceleration[dim] : nullptr;
  a.coef = coef;
  a.gamma = p->gamma;
  a.dt = p->dt;
  a.dt_device = p->dt_device;
  a.eta1 = p->eta1;
  a.eta2 = p->eta2;
  a.small_rho = p->small_rho;
  a.pmin = p->tiny_number;
  a.fallback = p->riemann_fallback;
  a.fstate = planes;
  a.fflux = planes + (size_t)ppm::kFaceVars * (size_t)a.plane;

  // a batch of one grid: its record and block prefix tables go into the descriptor area
  const int64_t march_blocks = (a.npencils + ppm::kMarchThreads - 1) / ppm::kMarchThreads;
  const int64_t riemann_blocks =
      (int64_t)(a.ie - a.is + 2) * ((a.npencils + ppm::kRiemannThreads - 1) / ppm::kRiemannThreads);
  unsigned char img[kStaticDescBytes];
  std::memset(img, 0, sizeof(img));
  std::memcpy(img, &a, sizeof(a));
  const int64_t mpre[2] = {0, march_blocks}, rpre[2] = {0, riemann_blocks};
  std::memcpy(img + 512, mpre, sizeof(mpre));
  std::memcpy(img + 768, rpre, sizeof(rpre));
  e = cudaMemcpyAsync(desc, img, sizeof(img), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyAsync");
  ppm::BatchArgs B;
  B.one = a;
  B.grids = reinterpret_cast<const ppm::SweepArgs*>(desc);
  B.ngrids = 1;
  B.march_prefix = reinterpret_cast<const int64_t*>(desc + 512);
  B.riemann_prefix = reinterpret_cast<const int64_t*>(desc + 768);
  B.counters = counters;
  B.flagged = reinterpret_cast<int64_t*>(planes + (size_t)(ppm::kFaceVars + ppm::kFluxVars) *
                                                      (size_t)a.plane);
  ppm::launch_sweep_batch(B, march_blocks, riemann_blocks, p->dual_energy != 0, p->gravity != 0,
                          st, nullptr, false, dim == 0);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "sweep launch");

  // ---- status
  unsigned long long c[ppm::kMaxCounters];
  e = cudaMemcpyAsync(c, counters, sizeof(c), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyAsync");
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail_cuda(e, "cudaStreamSynchronize");
  if (stats) {
    stats->interfaces += (long long)c[ppm::kCntInterfaces];
    stats->newton_iters += (long long)c[ppm::kCntNewton];
    for (int h = 0; h < 8; ++h) stats->newton_hist[h] += (long long)c[ppm::kCntHist0 + h];
    stats->fallbacks += (long long)c[ppm::kCntFallbacks];
    stats->fatal_cells += (long long)c[ppm::kCntFatal];
    stats->warp_newton_iters += (long long)c[ppm::kCntWarpNewton];
    stats->warps += (long long)c[ppm::kCntWarps];
  }
  if (c[ppm::kCntTimeout]) return PPM_B200_ERR_TIMEOUT;
  if (c[ppm::kCntFatal]) return PPM_B200_ERR_NEGATIVE;
  if (c[ppm::kCntNonFinite]) return PPM_B200_ERR_NONFINITE;
  return PPM_B200_OK;
}
