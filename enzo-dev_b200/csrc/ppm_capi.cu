// ppm_capi.cu -- the C ABI of include/ppm_b200.h: context, persistent device scratch,
// batch descriptors, and the grid::SolvePPM_DE driver (pressure once, then the sweeps
// in the order rotated by CycleNumber % GridRank, Grid_SolvePPM_DE.C:53-146).
//
// Every call runs on a batch of grids: a single grid (ppm_b200_solve_ppm_de,
// ppm_b200_euler_sweep) or all grids of an AMR level (ppm_b200_solve_level).  Each
// kernel stage is one launch over the whole batch; the per-grid records and block
// prefix tables it reads are uploaded only when their contents change, so a
// device-resident time loop issues no host-to-device copies after its first step and
// can be replayed as a CUDA graph.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled

#include <algorithm>
#include <array>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "ppm_b200.h"
#include "ppm_guess.cuh"
#include "ppm_sweep.cuh"

namespace ppm {
// element-wise batch records, defined with the kernels in ppm_kernels.cu
struct ElemGrid {
  const double* d;
  const double* te;
  const double* v[3];
  const double* ge;
  double* p;
  double* f[6];
  const double* cw[3];
  const double* old[6];
  int rank;
  int dims[3], start[3], end[3];
  int bc[3];
  int64_t size;
  int64_t active;
};
struct ElemBatch {
  const ElemGrid* grids;
  int ngrids;
  const int64_t* size_prefix;
  const int64_t* active_prefix;
  const int64_t* row_prefix;
  double gamma, tiny_number, min_support;
  double aye, vg[3];
  unsigned long long* min_bits;
  double expansion, coef_new, coef_old;
  int interpolate;
  int presfree;
  int eos_type;
  double eos_cs;
};
void launch_expansion_batch(const ElemBatch& B, int64_t blocks, cudaStream_t st);
void launch_cfl_reset(unsigned long long* min_bits, cudaStream_t st);
void launch_cfl_finalize(const unsigned long long* min_bits, double courant, double* dt_out,
                         cudaStream_t st);
void launch_sweep_batch(const BatchArgs& B, int64_t march_blocks, int64_t riemann_blocks,
                        bool dual, bool grav, cudaStream_t st, cudaEvent_t* ev, bool learned,
                        bool contiguous);
int riemann_resident_blocks(bool dual, bool one, int threads);
// learned-start training and evaluation (ppm_mlp.cu)
cudaError_t launch_guess_features(const double* rec, int64_t n, double gamma, double pmin,
                                  float* out, cudaStream_t st);
cudaError_t launch_guess_grad(const float* W, const float* samples, const int64_t* index,
                              int64_t n, float inv_count, float* grad, double* loss, int blocks,
                              cudaStream_t st);
cudaError_t launch_guess_adam(float* W, float* grad, float* m, float* v, int step, float lr,
                              float beta1, float beta2, float eps, cudaStream_t st);
cudaError_t launch_guess_eval(const uint32_t* packed, const float* feats, int64_t n, float* y,
                              cudaStream_t st);
cudaError_t launch_guess_eval_tc(const uint32_t* words, const float* feats, int64_t n, float* y,
                                 unsigned long long* timeouts, int sms, cudaStream_t st);
void launch_pressure_batch(const ElemBatch& B, int64_t blocks, cudaStream_t st);
void launch_timestep_batch(const ElemBatch& B, int64_t blocks, double courant, double* dt_out,
                           cudaStream_t st);
void launch_boundary_batch(const ElemBatch& B, int64_t blocks, cudaStream_t st);
struct CopyBox {
  int dst, src;
  int d0[3], s0[3], ext[3];
  int pad;
};
void launch_copy_zones(const ElemGrid* grids, const CopyBox* boxes, const int64_t* prefix,
                       int nboxes, int64_t blocks, cudaStream_t st);
struct FluxPhase {
  int start[3], dim[3];
  long long offset;
  int correct_left, correct_right;
  int id[3], io[3], rd[3], ro[3];
  int subling;
  const double* il[6];
  double* rl[6];
  const double* ir[6];
  double* rr[6];
};
struct FluxFix {
  double* f[6];
  int dims[3], rank, dual;
  double tiny_number;
  int nphases;
  double* const* species;
  int nspecies;
};
void launch_correct_fluxes(const FluxFix& X, const FluxPhase* phases, cudaStream_t st);
}  // namespace ppm

using ppm::BatchArgs;
using ppm::build_coef;
using ppm::Coef;
using ppm::ElemBatch;
using ppm::ElemGrid;
using ppm::FluxCapture;
using ppm::SweepArgs;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// A device copy of a host byte image, re-uploaded only when the image changes.  The
// upload is queued on the context stream from pinned staging memory, so it neither
// waits for the device nor races kernels queued before it (they read the old image).
constexpr int kStages = 4;  // staging buffers per slot, reused round robin
struct Mirror {
  DevBuf dev;
  std::vector<unsigned char> host;
  uint64_t version = 0;
  void* stage[kStages] = {nullptr, nullptr, nullptr, nullptr};
  size_t stage_bytes[kStages] = {0, 0, 0, 0};
  cudaEvent_t done[kStages] = {nullptr, nullptr, nullptr, nullptr};  // copy out of stage k
  int next = 0;
};

// descriptor slots: one per sweep direction and position, per element kernel and per
// table, so a time loop that repeats the same calls uploads nothing after its first step
enum {
  kSlotSweep0 = 0,     // 0..8: sweep records + block prefixes, per (direction, position
                       //       of the sweep in the rotated order): the ring buffers a
                       //       sweep reads and writes depend on both
  kSlotPressure = 9,   // element records of the pressure kernel
  kSlotCoef0 = 10,     // 10..12: inteuler coefficient tables per direction
  kSlotCw = 13,        // cell widths of the time-step kernel
  kSlotTimestep = 14,  // element records of the time-step kernel
  kSlotBoundary = 15,  // element records of the ghost-fill kernel
  kSlotExpansion = 16, // element records of the comoving-expansion kernel
  kSlotCflCw = 17,     // cell widths read by the time step folded into the last sweep
  kSlotCopy = 18,      // element records of the sibling-zone copy
  kSlotCopyBoxes = 19, // its boxes and block prefix
  kSlotColours = 20,   // colour field pointers of every grid of a sweep batch
  kSlotCount = 21
};
// captured level graphs kept at most (a changed grid list leaves the old ones unused)
constexpr size_t kMaxGraphs = 16;
// events around a timed sweep: before each of its five kernels and after the last
constexpr int kSweepEvents = 6;

struct ppm_b200_context {
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  long long launches = 0;
  int sticky_error = 0;
  // persistent device scratch, grown on demand
  DevBuf host_set[6];       // device copies of host-memory fields (single grid)
  DevBuf host_acc[3];       // device copies of host-memory accelerations
  DevBuf host_old[6];       // device copies of host-memory fields at OldTime
  DevBuf host_col;          // device copies of host-memory colour fields (single grid)
  DevBuf ring;              // two ring sets of the six updated fields, every grid of the batch
  DevBuf pressure;          // pressure of every grid of the batch
  DevBuf face_scratch;      // interface states, fluxes and the flagged-pencil list
  DevBuf counters;          // kMaxCounters unsigned long long
  DevBuf misc;              // [0] min_bits, [1] dt, [2] min_bits of the folded time step
  DevBuf captures;
  DevBuf capture_buf;
  DevBuf col_capture;       // colour fluxes of the capture requests (ncolour per request)
  DevBuf flux_fix;          // flux arrays and phases of ppm_b200_correct_fluxes
  std::vector<double> capture_host;
  std::vector<double> col_capture_host;
  // descriptor slots, in banks: bank 0 serves every entry point; a level solved in
  // waves takes one bank per wave, so a graph holding all the waves finds each wave's
  // descriptors where that wave left them.  `mirror` is the current bank.
  std::vector<std::unique_ptr<std::array<Mirror, kSlotCount>>> banks;
  Mirror* mirror = nullptr;
  // level schedule (ppm_b200_set_level_config / the autotuner) and the Riemann settings
  // of the batch being prepared (prepare_sweep reads them)
  ppm_b200_level_config level{};
  int sweep_mode = PPM_B200_SWEEP_SPLIT;  // ppm_b200_set_sweep_mode
  int wave_rt = ppm::kRiemannThreads;
  int wave_persist = 0;
  // event timing of sweep launches
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;  // kSweepEvents per timed sweep
  size_t ev_used = 0;
  double stage_ms[5] = {0, 0, 0, 0, 0};  // per-kernel totals of the last profile read
  // time step of the next cycle, folded into each solve's last sweep (ppm_b200_set_cfl)
  double* cfl_dt = nullptr;
  double cfl_courant = 1.0, cfl_aye = 1.0, cfl_vg[3] = {0.0, 0.0, 0.0};
  unsigned debug_tma_extra = 0;  // ppm_b200_debug_tma_stall
  // learned Newton start: packed inference weights (ppm_b200_set_guess)
  DevBuf guess;
  bool has_guess = false;
  // log of sampled Riemann problems of the plain solver (ppm_b200_riemann_log)
  double* log = nullptr;
  long long log_cap = 0;
  int log_stride = 0;
  DevBuf log_count;
  // CUDA graphs of level solves, keyed by everything a launch takes by value
  bool use_graphs = false;
  std::map<std::string, cudaGraphExec_t> graphs;
};

namespace {

int cuda_fail(ppm_b200_context* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return PPM_B200_OK;
  fprintf(stderr, "ppm_b200: %s failed: %s\n", what, cudaGetErrorString(e));
  if (ctx) ctx->sticky_error = PPM_B200_ERR_CUDA;
  return PPM_B200_ERR_CUDA;
}

#define CK(call)                                              \
  do {                                                        \
    cudaError_t _e = (call);                                  \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call);  \
  } while (0)

void drop_graphs(ppm_b200_context* ctx) {
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
}

int ensure(ppm_b200_context* ctx, DevBuf& b, size_t bytes) {
  if (b.bytes >= bytes) return PPM_B200_OK;
  if (b.p) {
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaFree(b.p));
    b.p = nullptr;
    b.bytes = 0;
    drop_graphs(ctx);  // captured graphs may reference the old allocation
  }
  CK(cudaMalloc(&b.p, bytes));
  b.bytes = bytes;
  return PPM_B200_OK;
}

// Upload `img` into mirror slot m unless the device copy already holds it.
// Make bank w the current descriptor bank (allocated on first use).
void select_bank(ppm_b200_context* ctx, size_t w) {
  while (ctx->banks.size() <= w) ctx->banks.emplace_back(new std::array<Mirror, kSlotCount>());
  ctx->mirror = ctx->banks[w]->data();
}

int mirror_put(ppm_b200_context* ctx, Mirror& m, const std::vector<unsigned char>& img) {
  if (m.host.size() == img.size() && m.dev.p &&
      std::memcmp(m.host.data(), img.data(), img.size()) == 0)
    return PPM_B200_OK;
  int rc = ensure(ctx, m.dev, std::max<size_t>(img.size(), 256));
  if (rc) return rc;
  const int k = m.next;
  m.next = (m.next + 1) % kStages;
  if (m.done[k]) {
    CK(cudaEventSynchronize(m.done[k]));  // the copy that last used this staging buffer
  } else {
    CK(cudaEventCreateWithFlags(&m.done[k], cudaEventDisableTiming));
  }
  if (m.stage_bytes[k] < img.size()) {
    if (m.stage[k]) CK(cudaFreeHost(m.stage[k]));
    m.stage[k] = nullptr;
    m.stage_bytes[k] = 0;
    const size_t cap = std::max<size_t>(img.size() + img.size() / 2, 4096);
    CK(cudaMallocHost(&m.stage[k], cap));
    m.stage_bytes[k] = cap;
  }
  if (!img.empty()) {
    std::memcpy(m.stage[k], img.data(), img.size());
    CK(cudaMemcpyAsync(m.dev.p, m.stage[k], img.size(), cudaMemcpyHostToDevice, ctx->stream));
  }
  CK(cudaEventRecord(m.done[k], ctx->stream));
  m.host = img;
  m.version += 1;
  return PPM_B200_OK;
}

void mirror_free(Mirror& m) {
  for (int k = 0; k < kStages; ++k) {
    if (m.done[k]) cudaEventDestroy(m.done[k]);
    if (m.stage[k]) cudaFreeHost(m.stage[k]);
    m.done[k] = nullptr;
    m.stage[k] = nullptr;
    m.stage_bytes[k] = 0;
  }
}

template <class T>
void append(std::vector<unsigned char>& img, const T* p, size_t n) {
  const size_t at = img.size();
  img.resize(at + n * sizeof(T));
  if (n) std::memcpy(img.data() + at, p, n * sizeof(T));
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int64_t grid_size(const ppm_b200_grid* g) {
  return (int64_t)g->dims[0] * g->dims[1] * g->dims[2];
}

int64_t grid_active(const ppm_b200_grid* g) {
  int64_t n = 1;
  for (int d = 0; d < g->rank; ++d) n *= g->end[d] - g->start[d] + 1;
  return n;
}

int check_supported(const ppm_b200_params* p) {
  if (!p) return PPM_B200_ERR_INVALID;
  // EOSType: ideal gas, or 3 (isothermal; the other polytropes need the unit system)
  if (p->diffusion || p->conservative_rec || p->positive_rec ||
      (p->eos_type != 0 && p->eos_type != 3))
    return PPM_B200_ERR_UNSUPPORTED;
  if (p->pressure_free != 0 && p->pressure_free != 1) return PPM_B200_ERR_UNSUPPORTED;
  if (p->number_of_colours < 0 || p->number_of_colours > PPM_B200_MAX_COLOURS)
    return PPM_B200_ERR_UNSUPPORTED;
  // slope corrections: calcdiss's flattening types 1-3, inteuler's steepening
  if ((p->flattening < 0 || p->flattening > 3) ||
      (p->steepening != 0 && p->steepening != 1))
    return PPM_B200_ERR_UNSUPPORTED;
  // the solver switch of Grid_xEulerSweep.C:223-283 (two-shock, HLL, HLLC)
  if (p->learned_guess < 0 || p->learned_guess > 2) return PPM_B200_ERR_UNSUPPORTED;
  if (p->riemann_solver != PPM_B200_RIEMANN_TWOSHOCK && p->riemann_solver != PPM_B200_RIEMANN_HLL &&
      p->riemann_solver != PPM_B200_RIEMANN_HLLC)
    return PPM_B200_ERR_UNSUPPORTED;
  if (p->reconstruction != PPM_B200_RECONSTRUCTION_PPM) return PPM_B200_ERR_UNSUPPORTED;
  return PPM_B200_OK;
}

int check_grid(const ppm_b200_grid* g, const ppm_b200_params* p) {
  if (!g || g->rank < 1 || g->rank > 3) return PPM_B200_ERR_INVALID;
  if (!g->density || !g->total_energy || !g->velocity[0]) return PPM_B200_ERR_INVALID;
  if (p->dual_energy && !g->gas_energy) return PPM_B200_ERR_INVALID;
  if (p->number_of_colours > 0) {
    if (!g->colours) return PPM_B200_ERR_INVALID;
    for (int n = 0; n < p->number_of_colours; ++n)
      if (!g->colours[n]) return PPM_B200_ERR_INVALID;
  }
  for (int d = 0; d < 3; ++d) {
    if (d < g->rank) {
      if (g->end[d] - g->start[d] + 1 > 1) {
        // the sweep needs exactly three ghost zones on each side (NumberOfGhostZones = 3)
        if (g->start[d] != 3 || g->dims[d] - 1 - g->end[d] != 3) return PPM_B200_ERR_INVALID;
        if (!g->cell_width[d]) return PPM_B200_ERR_INVALID;
        if (g->dims[d] > 1031) return PPM_B200_ERR_TOO_LARGE;  // fortran.def:1
      }
      if (d > 0 && !g->velocity[d]) return PPM_B200_ERR_INVALID;
      if (p->gravity && !g->acceleration[d]) return PPM_B200_ERR_INVALID;
    } else if (g->dims[d] != 1) {
      return PPM_B200_ERR_INVALID;
    }
  }
  return PPM_B200_OK;
}

// A learned start needs weights (ppm_b200_set_guess) on this context.
int check_guess(const ppm_b200_context* ctx, const ppm_b200_params* p) {
  if (p->learned_guess && !ctx->has_guess) return PPM_B200_ERR_INVALID;
  return PPM_B200_OK;
}

// Host: FP32 master weights -> BF16 B fragments of mma.m16n8k16 + FP32 biases, in the
// order guess_mlp_warp reads them (ppm_guess.cuh).
uint16_t bf16_bits(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);  // round to nearest even (finite inputs)
  return (uint16_t)(u >> 16);
}

uint32_t bf16_pair(float lo, float hi) {
  return (uint32_t)bf16_bits(lo) | ((uint32_t)bf16_bits(hi) << 16);
}

// The tcgen05 image (ppm_guess.cuh kTc*) appended at word kTcWordOffset.
void pack_guess_tc(const float* w, std::vector<uint32_t>& out) {
  using namespace ppm;
  out.resize(kGuessBufferWords, 0u);
  unsigned char* img = reinterpret_cast<unsigned char*>(out.data() + kTcWordOffset);
  auto put_b = [&](int base, int N, int n, int k, float v) {
    const uint16_t h = bf16_bits(v);
    const size_t off = (size_t)base + (size_t)((k / 8) * (N / 8) + n / 8) * 128 +
                       (size_t)(n % 8) * 16 + (size_t)(k % 8) * 2;
    std::memcpy(img + off, &h, 2);
  };
  for (int n = 0; n < kGuessHidden; ++n)
    for (int k = 0; k < 16; ++k)
      put_b(kTcW1, kGuessHidden, n, k, k < kGuessIn ? w[kOffW1 + k * kGuessHidden + n] : 0.0f);
  for (int n = 0; n < kGuessHidden; ++n)
    for (int k = 0; k < kGuessHidden; ++k)
      put_b(kTcW2, kGuessHidden, n, k, w[kOffW2 + k * kGuessHidden + n]);
  auto put_f = [&](int off, float v) { std::memcpy(img + off, &v, 4); };
  for (int j = 0; j < kGuessHidden; ++j) {
    put_f(kTcB1 + 4 * j, w[kOffB1 + j]);
    put_f(kTcB2 + 4 * j, w[kOffB2 + j]);
    uint32_t u = (uint32_t)bf16_bits(w[kOffW3 + j]) << 16;  // w3 as the bf16 value it holds
    float f;
    std::memcpy(&f, &u, 4);
    put_f(kTcW3 + 4 * j, f);
  }
  put_f(kTcB3, w[kOffB3]);
}

void pack_guess(const float* w, std::vector<uint32_t>& out) {
  using namespace ppm;
  out.assign(kPackWords, 0u);
  auto w1 = [&](int k, int n) { return k < kGuessIn ? w[kOffW1 + k * kGuessHidden + n] : 0.0f; };
  auto w2 = [&](int k, int n) { return w[kOffW2 + k * kGuessHidden + n]; };
  for (int lane = 0; lane < 32; ++lane) {
    const int g = lane >> 2, t = lane & 3;
    for (int n = 0; n < 8; ++n) {
      const int col = 8 * n + g;
      uint32_t* o = &out[kPackL1 + (n * 32 + lane) * 2];
      o[0] = bf16_pair(w1(2 * t, col), w1(2 * t + 1, col));
      o[1] = bf16_pair(w1(2 * t + 8, col), w1(2 * t + 9, col));
    }
    for (int kk = 0; kk < 4; ++kk)
      for (int n = 0; n < 8; ++n) {
        const int col = 8 * n + g, r0 = 16 * kk + 2 * t;
        uint32_t* o = &out[kPackL2 + ((kk * 8 + n) * 32 + lane) * 2];
        o[0] = bf16_pair(w2(r0, col), w2(r0 + 1, col));
        o[1] = bf16_pair(w2(r0 + 8, col), w2(r0 + 9, col));
      }
    for (int kk = 0; kk < 4; ++kk) {
      const int r0 = 16 * kk + 2 * t;
      uint32_t* o = &out[kPackL3 + (kk * 32 + lane) * 2];
      if (g == 0) {
        o[0] = bf16_pair(w[kOffW3 + r0], w[kOffW3 + r0 + 1]);
        o[1] = bf16_pair(w[kOffW3 + r0 + 8], w[kOffW3 + r0 + 9]);
      }
    }
  }
  for (int j = 0; j < kGuessHidden; ++j) {
    std::memcpy(&out[kPackB1 + j], &w[kOffB1 + j], 4);
    std::memcpy(&out[kPackB2 + j], &w[kOffB2 + j], 4);
  }
  std::memcpy(&out[kPackB3], &w[kOffB3], 4);
}

struct FieldSet {
  double* f[6];  // d, e, v1, v2, v3, ge
  int ncol = 0;  // colour fields (the grid's own set only: colours are updated in place)
  double* col[ppm::kMaxColours];
};

// Device pointers of one grid for one call.
struct GridIO {
  const ppm_b200_grid* g;
  FieldSet user;            // the grid's fields (device)
  FieldSet ring[2];         // scratch ring sets
  const double* acc[3];
  double* pres;
};

// One capture request on the host: where the 6 captured values of a request go.
struct HostCapture {
  int sub;     // subgrid
  int side;    // 0 left, 1 right
  int64_t offset;
};

// Per-grid coefficient tables of one direction, deduplicated by content.
struct CoefTables {
  std::vector<Coef> all;
  std::vector<int64_t> offset;  // per grid, entries into `all`
};

void build_coef_tables(int dim, const std::vector<GridIO>& io, CoefTables& ct) {
  ct.all.clear();
  ct.offset.assign(io.size(), 0);
  std::map<std::vector<double>, int64_t> seen;
  for (size_t k = 0; k < io.size(); ++k) {
    const ppm_b200_grid* g = io[k].g;
    const int n = g->dims[dim];
    std::vector<double> key(g->cell_width[dim], g->cell_width[dim] + n);
    key.push_back((double)g->start[dim]);
    key.push_back((double)g->end[dim]);
    auto it = seen.find(key);
    if (it != seen.end()) {
      ct.offset[k] = it->second;
      continue;
    }
    std::vector<Coef> c;
    build_coef(g->cell_width[dim], n, g->start[dim], g->end[dim], c);
    ct.offset[k] = (int64_t)ct.all.size();
    seen[key] = ct.offset[k];
    ct.all.insert(ct.all.end(), c.begin(), c.end());
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against the
// driver library); null when the driver does not offer it
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// The x sweep of a single grid: 2-D tensor maps (cells x pencils) of its six input
// fields, for the update kernel's TMA tiles.  They need a pencil to be a whole row of
// the array (the x sweep covers every row, ghosts included), a 16-byte aligned base and
// rows of a multiple of 16 bytes (even GridDimension[0]); otherwise B.x_tma stays 0 and
// the kernel uses plain loads.
void set_x_tiles(BatchArgs& B, const SweepArgs& a) {
  B.x_tma = 0;
  if (a.sa != 1 || a.s1 != a.n || a.s2 != (int64_t)a.n * a.n1 ||
      a.npencils != (int64_t)a.n1 * a.n2 || a.n % 2 != 0 || a.npencils >= (int64_t(1) << 31))
    return;
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return;
  const double* f[6] = {a.in_d, a.in_e, a.in_u, a.in_v, a.in_w, a.in_ge};
  for (int k = 0; k < 6; ++k) {
    std::memset(&B.xin[k], 0, sizeof(B.xin[k]));
    if (!f[k]) continue;
    if ((uintptr_t)f[k] % 16 != 0) return;
    cuuint64_t dim[2] = {(cuuint64_t)a.n, (cuuint64_t)a.npencils};
    cuuint64_t stride[1] = {(cuuint64_t)a.n * sizeof(double)};
    cuuint32_t box[2] = {ppm::kXTileCells, ppm::kXTileRows};
    cuuint32_t estride[2] = {1, 1};
    if (enc(&B.xin[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(f[k]), dim,
            stride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_64B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return;
  }
  B.x_tma = 1;
}

// Everything one directional sweep of a batch needs on the device.
struct SweepPlan {
  BatchArgs B;
  int64_t march_blocks = 0, riemann_blocks = 0;
  std::vector<FluxCapture> reqs;    // single-grid subgrid-flux capture
  std::vector<HostCapture> hreq;
  int64_t cap_offset = 0;           // this sweep's first request in the capture buffers
  bool contiguous = false;          // x sweep: pencils along the contiguous axis
};

// Subgrid flux capture requests of one sweep of a single grid (Grid_xEulerSweep.C:313-377
// and its y/z siblings): one request per (flux-plane cell, side), sorted by pencil.
int build_captures(const ppm_b200_grid* g, int dim, int nsub, const ppm_b200_fluxes* sub,
                   const long long ggs[3], SweepPlan& plan) {
  plan.reqs.clear();
  plan.hreq.clear();
  if (nsub <= 0 || !sub) return PPM_B200_OK;
  const int is = g->start[dim], ie = g->end[dim];
  int n1, n2, ax1, ax2;
  if (dim == 0) { n1 = g->dims[1]; n2 = g->dims[2]; ax1 = 1; ax2 = 2; }
  else if (dim == 1) { n1 = g->dims[0]; n2 = g->dims[2]; ax1 = 0; ax2 = 2; }
  else { n1 = g->dims[0]; n2 = g->dims[1]; ax1 = 0; ax2 = 1; }
  for (int s = 0; s < nsub; ++s) {
    const ppm_b200_fluxes& fx = sub[s];
    // flux-plane axes as the reference names them: (idim, jdim)
    const int ia = (dim == 0) ? 1 : 0;
    const int ja = (dim == 2) ? 1 : 2;
    const long long fi0 = fx.right_start[dim][ia] - ggs[ia];
    const long long fi1 = fx.right_end[dim][ia] - ggs[ia];
    const long long fj0 = fx.right_start[dim][ja] - ggs[ja];
    const long long fj1 = fx.right_end[dim][ja] - ggs[ja];
    const long long nfi = fi1 - fi0 + 1;
    const long long lface = fx.left_start[dim][dim] - ggs[dim];
    const long long rface = fx.right_start[dim][dim] - ggs[dim] + 1;
    if (lface < is || rface > ie + 1) return PPM_B200_ERR_INVALID;
    for (long long cj = fj0; cj <= fj1; ++cj)
      for (long long ci = fi0; ci <= fi1; ++ci) {
        long long c[3] = {0, 0, 0};
        c[ia] = ci;
        c[ja] = cj;
        const int64_t t1 = c[ax1], t2 = c[ax2];
        if (t1 < 0 || t1 >= n1 || t2 < 0 || t2 >= n2) return PPM_B200_ERR_INVALID;
        const int64_t pencil = t2 * n1 + t1;
        const long long offset = (ci - fi0) + (cj - fj0) * nfi;
        for (int side = 0; side < 2; ++side) {
          FluxCapture r;
          r.pencil = pencil;
          r.face = (int)(side == 0 ? lface : rface);
          r.pad = (int)plan.hreq.size();
          r.dst = 0;
          plan.reqs.push_back(r);
          plan.hreq.push_back(HostCapture{s, side, offset});
        }
      }
  }
  std::sort(plan.reqs.begin(), plan.reqs.end(), [](const FluxCapture& x, const FluxCapture& y) {
    return x.pencil != y.pencil ? x.pencil < y.pencil : x.face < y.face;
  });
  return PPM_B200_OK;
}

// Places the capture requests of several sweeps one after another in the capture
// buffers (sized before any sweep is queued, so no buffer moves under queued work).
int reserve_captures(ppm_b200_context* ctx, SweepPlan* plans, int n, int ncolour) {
  int64_t total = 0;
  for (int s = 0; s < n; ++s) {
    plans[s].cap_offset = total;
    total += (int64_t)plans[s].reqs.size();
  }
  if (total == 0) return PPM_B200_OK;
  int rc = ensure(ctx, ctx->captures, (size_t)total * sizeof(FluxCapture));
  if (rc) return rc;
  if (ncolour > 0) {
    rc = ensure(ctx, ctx->col_capture, (size_t)total * (size_t)ncolour * sizeof(double));
    if (rc) return rc;
  }
  return ensure(ctx, ctx->capture_buf, (size_t)total * 6 * sizeof(double));
}

// Face scratch of one directional sweep of a batch: 19 planes of (active cells along
// the sweep + 1) x pencils per grid, then one flagged-pencil slot per pencil.  The
// size differs between directions for non-cubic grids.
// planes of slope-correction coefficients a grid's sweep needs (cells is-1 .. ie+1)
size_t correction_planes(const ppm_b200_params* p) {
  return (p->flattening ? 1 : 0) + (p->steepening ? 1 : 0);
}

// colour face planes of a sweep (planes of the face scratch) and its fallback-face flags
// (bytes, one plane per grid after the flagged-pencil list)
size_t colour_planes(const ppm_b200_params* p) {
  return p->number_of_colours > 0 ? (size_t)ppm::kColVars : 0;
}

// SweepArgs::solver of a RiemannSolver value: 0 two-shock, 1 HLL, 2 HLLC
int solver_code(const ppm_b200_params* p) {
  return p->riemann_solver == PPM_B200_RIEMANN_HLL ? 1
         : p->riemann_solver == PPM_B200_RIEMANN_HLLC ? 2 : 0;
}

// kernels one sweep launches: reconstruct x2, Riemann, update, fallback, and the
// corrections and colour kernels when present
int sweep_kernels(const ppm_b200_params* p) {
  return 5 + (correction_planes(p) > 0 ? 1 : 0) + (p->number_of_colours > 0 ? 1 : 0);
}

size_t sweep_scratch_bytes(int dim, const std::vector<GridIO>& io, const ppm_b200_params* p) {
  size_t doubles = 0, pencils = 0, flags = 0;
  for (const auto& x : io) {
    const ppm_b200_grid* g = x.g;
    const size_t np = (size_t)grid_size(g) / (size_t)g->dims[dim];
    doubles += (size_t)(ppm::kFaceVars + ppm::kFluxVars + colour_planes(p)) *
               (size_t)(g->end[dim] - g->start[dim] + 2) * np;
    doubles += correction_planes(p) * (size_t)(g->end[dim] - g->start[dim] + 3) * np;
    pencils += np;
    if (p->number_of_colours > 0) flags += (size_t)(g->end[dim] - g->start[dim] + 2) * np;
  }
  return doubles * sizeof(double) + pencils * sizeof(int64_t) + flags;
}

int prepare_sweep(ppm_b200_context* ctx, int dim, int position, const ppm_b200_params* p,
                  const std::vector<GridIO>& io, const std::vector<int>& src,
                  const std::vector<int>& dst, SweepPlan& plan, bool cfl = false) {
  const int ng = (int)io.size();
  // the folded time step reads the transverse cell widths: one deduplicated table
  std::vector<std::array<int64_t, 3>> cwoff(ng, std::array<int64_t, 3>{{-1, -1, -1}});
  const double* cw_dev = nullptr;
  if (cfl) {
    std::vector<double> cws;
    std::map<std::vector<double>, int64_t> seen;
    for (int k = 0; k < ng; ++k)
      for (int d = 0; d < io[k].g->rank; ++d) {
        const ppm_b200_grid* g = io[k].g;
        std::vector<double> key(g->cell_width[d], g->cell_width[d] + g->dims[d]);
        auto it = seen.find(key);
        if (it != seen.end()) {
          cwoff[k][d] = it->second;
        } else {
          cwoff[k][d] = (int64_t)cws.size();
          seen[key] = cwoff[k][d];
          cws.insert(cws.end(), key.begin(), key.end());
        }
      }
    std::vector<unsigned char> cimg;
    append(cimg, cws.data(), cws.size());
    int rc0 = mirror_put(ctx, ctx->mirror[kSlotCflCw], cimg);
    if (rc0) return rc0;
    cw_dev = (const double*)ctx->mirror[kSlotCflCw].dev.p;
  }
  // coefficient tables (deduplicated), uploaded into this direction's table slot
  CoefTables ct;
  build_coef_tables(dim, io, ct);
  std::vector<unsigned char> timg;
  append(timg, ct.all.data(), ct.all.size());
  int rc = mirror_put(ctx, ctx->mirror[kSlotCoef0 + dim], timg);
  if (rc) return rc;
  const Coef* coef_dev = (const Coef*)ctx->mirror[kSlotCoef0 + dim].dev.p;

  // the two-shock stage with the plain start takes the batch's block size and
  // persistence; every other Riemann stage runs kRiemannThreads faces per block
  const bool plain_riemann = !p->learned_guess && p->number_of_colours == 0 &&
                             solver_code(p) == 0 && p->pressure_free != 1;
  const int rt = plain_riemann ? ctx->wave_rt : ppm::kRiemannThreads;
  const bool persist = plain_riemann && ctx->wave_persist != 0;
  // face scratch: planes of every grid, then the flagged-pencil list
  std::vector<SweepArgs> rec(ng);
  std::vector<int64_t> mpre(ng + 1, 0), rpre(ng + 1, 0), fpre(ng + 1, 0);
  // the fused face kernel serves the same plain two-shock path, without slope corrections
  const bool fused = plain_riemann && ctx->sweep_mode == PPM_B200_SWEEP_FUSED &&
                     correction_planes(p) == 0;
  size_t scratch_doubles = 0, flag_bytes = 0;
  int64_t total_pencils = 0;
  // colour field pointers of every grid, ncolour per grid
  const int nc = p->number_of_colours;
  double* const* col_dev = nullptr;
  if (nc > 0) {
    std::vector<double*> cptr;
    for (int k = 0; k < ng; ++k) {
      if (io[k].user.ncol != nc) return PPM_B200_ERR_INVALID;
      cptr.insert(cptr.end(), io[k].user.col, io[k].user.col + nc);
    }
    std::vector<unsigned char> cimg;
    append(cimg, cptr.data(), cptr.size());
    int rc0 = mirror_put(ctx, ctx->mirror[kSlotColours], cimg);
    if (rc0) return rc0;
    col_dev = (double* const*)ctx->mirror[kSlotColours].dev.p;
  }
  for (int k = 0; k < ng; ++k) {
    const ppm_b200_grid* g = io[k].g;
    const int GD0 = g->dims[0], GD1 = g->dims[1], GD2 = g->dims[2];
    SweepArgs& a = rec[k];
    std::memset(&a, 0, sizeof(a));
    a.n = g->dims[dim];
    a.is = g->start[dim];
    a.ie = g->end[dim];
    if (dim == 0) {
      a.n1 = GD1; a.n2 = GD2; a.s1 = GD0; a.s2 = (int64_t)GD0 * GD1; a.sa = 1;
    } else if (dim == 1) {
      a.n1 = GD0; a.n2 = GD2; a.s1 = 1; a.s2 = (int64_t)GD0 * GD1; a.sa = GD0;
    } else {
      a.n1 = GD0; a.n2 = GD1; a.s1 = 1; a.s2 = GD0; a.sa = (int64_t)GD0 * GD1;
    }
    a.npencils = (int64_t)a.n1 * a.n2;
    a.plane = (int64_t)(a.ie - a.is + 2) * a.npencils;
    scratch_doubles += (size_t)(ppm::kFaceVars + ppm::kFluxVars + colour_planes(p)) *
                       (size_t)a.plane;
    scratch_doubles += correction_planes(p) * (size_t)(a.ie - a.is + 3) * (size_t)a.npencils;
    total_pencils += a.npencils;
    if (nc > 0) flag_bytes += (size_t)a.plane;
    const int64_t mb = (a.npencils + ppm::kMarchThreads - 1) / ppm::kMarchThreads;
    const int64_t rb = (int64_t)(a.ie - a.is + 2) * ((a.npencils + rt - 1) / rt);
    mpre[k + 1] = mpre[k] + mb;
    rpre[k + 1] = rpre[k] + rb;
    fpre[k + 1] = fpre[k] + ppm::face_blocks(a.npencils, a.is, a.ie);
  }
  // callers that queue several sweeps size the scratch for all of them first, so this
  // never moves the buffer under a sweep prepared earlier
  rc = ensure(ctx, ctx->face_scratch,
              scratch_doubles * sizeof(double) + (size_t)total_pencils * sizeof(int64_t) +
                  flag_bytes);
  if (rc) return rc;
  double* scratch = (double*)ctx->face_scratch.p;
  unsigned char* flags = (unsigned char*)(scratch + scratch_doubles) +
                         (size_t)total_pencils * sizeof(int64_t);
  size_t at = 0, flag_at = 0;
  const int vu = dim, vv = (dim + 1) % 3, vw = (dim + 2) % 3;
  for (int k = 0; k < ng; ++k) {
    const ppm_b200_grid* g = io[k].g;
    const FieldSet& in = src[k] < 0 ? io[k].user : io[k].ring[src[k]];
    const FieldSet& out = dst[k] < 0 ? io[k].user : io[k].ring[dst[k]];
    auto vin = [&](int c) -> const double* { return c < g->rank ? in.f[2 + c] : nullptr; };
    auto vout = [&](int c) -> double* { return c < g->rank ? out.f[2 + c] : nullptr; };
    SweepArgs& a = rec[k];
    a.in_d = in.f[0];
    a.in_e = in.f[1];
    a.in_u = vin(vu);
    a.in_v = vin(vv);
    a.in_w = vin(vw);
    a.in_ge = p->dual_energy ? in.f[5] : nullptr;
    a.out_d = out.f[0];
    a.out_e = out.f[1];
    a.out_u = vout(vu);
    a.out_v = vout(vv);
    a.out_w = vout(vw);
    a.out_ge = p->dual_energy ? out.f[5] : nullptr;
    a.pres = io[k].pres;
    a.grav = p->gravity ? io[k].acc[dim] : nullptr;
    a.coef = coef_dev + ct.offset[k];
    a.gamma = p->gamma;
    a.dt = p->dt;
    a.dt_device = p->dt_device;
    a.eta1 = p->eta1;
    a.eta2 = p->eta2;
    a.small_rho = p->small_rho;
    a.pmin = p->tiny_number;
    // HLL has no fallback: a negative density stops the reference (flux_hll.F:378-380)
    a.solver = solver_code(p);
    a.presfree = p->pressure_free == 1 ? 1 : 0;
    a.eos_type = p->eos_type;
    a.eos_cs = p->eos_sound_speed;
    a.fallback = p->riemann_solver == PPM_B200_RIEMANN_HLL ? 0 : p->riemann_fallback;
    a.guess = p->learned_guess ? (const uint32_t*)ctx->guess.p : nullptr;
    if (ctx->log && !p->learned_guess) {
      a.log = ctx->log;
      a.log_count = (unsigned long long*)ctx->log_count.p;
      a.log_cap = ctx->log_cap;
      a.log_stride = ctx->log_stride;
    }
    a.fstate = scratch + at;
    a.fflux = a.fstate + (size_t)ppm::kFaceVars * (size_t)a.plane;
    at += (size_t)(ppm::kFaceVars + ppm::kFluxVars) * (size_t)a.plane;
    a.flatten = p->flattening;
    a.steepen = p->steepening;
    const size_t cplane = (size_t)(a.ie - a.is + 3) * (size_t)a.npencils;
    if (p->flattening) {
      a.flat = scratch + at;
      at += cplane;
    }
    if (p->steepening) {
      a.steep = scratch + at;
      at += cplane;
    }
    if (nc > 0) {
      a.ncolour = nc;
      a.col = col_dev + (size_t)k * (size_t)nc;
      a.fcol = scratch + at;
      at += (size_t)ppm::kColVars * (size_t)a.plane;
      a.fhll = flags + flag_at;
      flag_at += (size_t)a.plane;
    }
    a.dim = dim;
    a.rank = g->rank;
    if (cfl) {
      const int ax1 = dim == 0 ? 1 : 0, ax2 = dim == 2 ? 1 : 2;
      a.cfl_min_bits = ((unsigned long long*)ctx->misc.p) + 2;
      a.cw1 = cwoff[k][ax1] >= 0 ? cw_dev + cwoff[k][ax1] : nullptr;
      a.cw2 = cwoff[k][ax2] >= 0 ? cw_dev + cwoff[k][ax2] : nullptr;
      a.ts1 = g->start[ax1];
      a.te1 = g->end[ax1];
      a.ts2 = g->start[ax2];
      a.te2 = g->end[ax2];
      a.aye = ctx->cfl_aye;
      for (int d = 0; d < 3; ++d) a.vg[d] = ctx->cfl_vg[d];
      a.min_support = p->min_support;
    }
  }

  // subgrid flux capture (single grid): requests built by build_captures, buffers
  // placed by reserve_captures
  if (!plan.reqs.empty()) {
    SweepArgs& a = rec[0];
    for (size_t k = 0; k < plan.reqs.size(); ++k)
      plan.reqs[k].dst = (plan.cap_offset + (int64_t)k) * 6;
    FluxCapture* dev_reqs = (FluxCapture*)ctx->captures.p + plan.cap_offset;
    CK(cudaMemcpyAsync(dev_reqs, plan.reqs.data(), plan.reqs.size() * sizeof(FluxCapture),
                       cudaMemcpyHostToDevice, ctx->stream));
    a.captures = dev_reqs;
    a.ncaptures = (int64_t)plan.reqs.size();
    a.capture_buf = (double*)ctx->capture_buf.p;
    if (nc > 0) a.col_capture = (double*)ctx->col_capture.p;
  }

  // descriptor image: records | march prefix | riemann prefix
  std::vector<unsigned char> img;
  append(img, rec.data(), rec.size());
  const size_t off_m = align256(img.size());
  img.resize(off_m);
  append(img, mpre.data(), mpre.size());
  const size_t off_r = align256(img.size());
  img.resize(off_r);
  append(img, rpre.data(), rpre.size());
  const size_t off_f = align256(img.size());
  img.resize(off_f);
  append(img, fpre.data(), fpre.size());
  const int slot = kSlotSweep0 + 3 * dim + position;
  rc = mirror_put(ctx, ctx->mirror[slot], img);
  if (rc) return rc;
  unsigned char* base = (unsigned char*)ctx->mirror[slot].dev.p;
  std::memset(&plan.B.one, 0, sizeof(plan.B.one));
  if (ng == 1) plan.B.one = rec[0];
  plan.B.x_tma = 0;
  if (ng == 1 && dim == 0) set_x_tiles(plan.B, rec[0]);
  plan.B.x_tma_extra_tx = plan.B.x_tma ? ctx->debug_tma_extra : 0u;
  plan.B.corrections = correction_planes(p) > 0 ? 1 : 0;
  plan.B.ncolour = nc;
  plan.B.solver = solver_code(p);
  plan.B.presfree = p->pressure_free == 1 ? 1 : 0;
  plan.B.hll_flags = nc > 0 ? flags : nullptr;
  plan.B.hll_bytes = (int64_t)flag_bytes;
  plan.B.grids = (const SweepArgs*)base;
  plan.B.ngrids = ng;
  plan.B.march_prefix = (const int64_t*)(base + off_m);
  plan.B.riemann_prefix = (const int64_t*)(base + off_r);
  plan.B.counters = (unsigned long long*)ctx->counters.p;
  plan.B.flagged = (int64_t*)(scratch + scratch_doubles);
  plan.march_blocks = mpre[ng];
  plan.riemann_blocks = rpre[ng];
  plan.B.riemann_threads = rt;
  plan.B.persistent = persist ? 1 : 0;
  plan.B.riemann_total = rpre[ng];
  plan.B.fused = fused ? 1 : 0;
  plan.B.face_prefix = (const int64_t*)(base + off_f);
  plan.B.face_blocks = fpre[ng];
  // the tensor-core guess pass takes 128 faces per tile, as the Riemann kernel's blocks
  plan.B.learned_pass = (p->learned_guess == 2 && nc == 0) ? 1 : 0;
  plan.B.sms = ctx->sms;
  if (persist)
    plan.riemann_blocks = std::min<int64_t>(
        rpre[ng], (int64_t)ctx->sms *
                      ppm::riemann_resident_blocks(p->dual_energy != 0, ng == 1, rt));
  plan.contiguous = dim == 0;
  return PPM_B200_OK;
}

int enqueue_sweep(ppm_b200_context* ctx, const SweepPlan& plan, const ppm_b200_params* p,
                  bool capturing) {
  cudaEvent_t* ev = nullptr;
  if (ctx->profiling && !capturing) {
    while (ctx->ev_pool.size() < ctx->ev_used + kSweepEvents) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      ctx->ev_pool.push_back(e);
    }
    ev = &ctx->ev_pool[ctx->ev_used];
    ctx->ev_used += kSweepEvents;
  }
  ppm::launch_sweep_batch(plan.B, plan.march_blocks, plan.riemann_blocks, p->dual_energy != 0,
                          p->gravity != 0, ctx->stream, ev, p->learned_guess != 0,
                          plan.contiguous);
  ctx->launches += sweep_kernels(p);
  CK(cudaGetLastError());
  return PPM_B200_OK;
}

int scatter_captures(ppm_b200_context* ctx, int dim, const ppm_b200_params* p,
                     const ppm_b200_grid* g, const SweepPlan& plan, ppm_b200_fluxes* sub) {
  if (plan.reqs.empty()) return PPM_B200_OK;
  ctx->capture_host.resize(plan.reqs.size() * 6);
  CK(cudaMemcpyAsync(ctx->capture_host.data(), (double*)ctx->capture_buf.p + plan.cap_offset * 6,
                     plan.reqs.size() * 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  const int nc = p->number_of_colours;
  if (nc > 0) {
    ctx->col_capture_host.resize(plan.reqs.size() * (size_t)nc);
    CK(cudaMemcpyAsync(ctx->col_capture_host.data(),
                       (double*)ctx->col_capture.p + plan.cap_offset * nc,
                       plan.reqs.size() * (size_t)nc * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  // active extents for the transverse-velocity rule (nxz/nyz/nzz > 1)
  long long nact[3];
  for (int d = 0; d < 3; ++d) nact[d] = d < g->rank ? g->end[d] - g->start[d] + 1 : 1;
  const int vu = dim, vv = (dim + 1) % 3, vw = (dim + 2) % 3;
  // capture slot order: df, ef, uf, vf, wf, gef -> BaryonField slots
  const int slot_of_role[3] = {2 + vu, 2 + vv, 2 + vw};
  for (size_t k = 0; k < plan.reqs.size(); ++k) {
    const HostCapture& h = plan.hreq[plan.reqs[k].pad];
    ppm_b200_fluxes& fx = sub[h.sub];
    double* const* dst = h.side == 0 ? &fx.left[0][0] : &fx.right[0][0];
    auto put = [&](int slot, double v) {
      double* arr = dst[slot * 3 + dim];
      if (arr) arr[h.offset] = v;
    };
    const double* v = &ctx->capture_host[k * 6];
    put(0, v[0]);
    put(1, v[1]);
    for (int r = 0; r < 3; ++r) {
      int comp = slot_of_role[r] - 2;
      if (r != 0 && nact[comp] <= 1) continue;
      if (comp >= g->rank) continue;
      put(slot_of_role[r], v[2 + r]);
    }
    if (p->dual_energy) put(5, v[5]);
    // colours (Grid_xEulerSweep.C:361-371): entry n*3 + dim of the colour arrays
    double* const* cdst = h.side == 0 ? fx.colour_left : fx.colour_right;
    if (nc > 0 && cdst)
      for (int n = 0; n < nc; ++n)
        if (cdst[n * 3 + dim]) cdst[n * 3 + dim][h.offset] = ctx->col_capture_host[k * nc + n];
  }
  return PPM_B200_OK;
}

int read_counters(ppm_b200_context* ctx, ppm_b200_stats* st, int* status) {
  unsigned long long c[ppm::kMaxCounters];
  CK(cudaMemcpyAsync(c, ctx->counters.p, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemsetAsync(ctx->counters.p, 0, sizeof(c), ctx->stream));
  if (st) {
    st->interfaces += (long long)c[ppm::kCntInterfaces];
    st->newton_iters += (long long)c[ppm::kCntNewton];
    for (int h = 0; h < 8; ++h) st->newton_hist[h] += (long long)c[ppm::kCntHist0 + h];
    st->fallbacks += (long long)c[ppm::kCntFallbacks];
    st->fatal_cells += (long long)c[ppm::kCntFatal];
    st->guess_rejected += (long long)c[ppm::kCntGuessRejected];
    st->warp_newton_iters += (long long)c[ppm::kCntWarpNewton];
    st->warps += (long long)c[ppm::kCntWarps];
  }
  int s = PPM_B200_OK;
  if (c[ppm::kCntTimeout]) s = PPM_B200_ERR_TIMEOUT;
  else if (c[ppm::kCntFatal]) s = PPM_B200_ERR_NEGATIVE;
  else if (c[ppm::kCntNonFinite]) s = PPM_B200_ERR_NONFINITE;
  if (status) *status = s;
  return PPM_B200_OK;
}

// Element descriptors of a batch (pressure, time step, ghost fill), one image slot.
struct ElemPlan {
  ElemBatch B;
  int64_t size_blocks = 0, active_blocks = 0, row_blocks = 0;
};
constexpr int kFillRowsPerBlock = 32;  // rows of the padded grid per ghost-fill block

int prepare_elem(ppm_b200_context* ctx, int slot, const ppm_b200_params* p,
                 const std::vector<GridIO>& io, bool with_cw, const int* bc, ElemPlan& plan,
                 const std::vector<FieldSet>* old = nullptr) {
  const int ng = (int)io.size();
  std::vector<ElemGrid> rec(ng);
  std::vector<int64_t> spre(ng + 1, 0), apre(ng + 1, 0), rpre(ng + 1, 0);
  // cell widths (time step only), deduplicated, in their own slot
  std::vector<std::array<int64_t, 3>> cwoff(ng, std::array<int64_t, 3>{{-1, -1, -1}});
  if (with_cw) {
    std::vector<double> cws;
    std::map<std::vector<double>, int64_t> seen;
    for (int k = 0; k < ng; ++k)
      for (int d = 0; d < io[k].g->rank; ++d) {
        const ppm_b200_grid* g = io[k].g;
        std::vector<double> key(g->cell_width[d], g->cell_width[d] + g->dims[d]);
        auto it = seen.find(key);
        if (it != seen.end()) {
          cwoff[k][d] = it->second;
        } else {
          cwoff[k][d] = (int64_t)cws.size();
          seen[key] = cwoff[k][d];
          cws.insert(cws.end(), key.begin(), key.end());
        }
      }
    std::vector<unsigned char> cimg;
    append(cimg, cws.data(), cws.size());
    int rc = mirror_put(ctx, ctx->mirror[kSlotCw], cimg);
    if (rc) return rc;
  }
  const double* cw_dev = (const double*)ctx->mirror[kSlotCw].dev.p;
  for (int k = 0; k < ng; ++k) {
    const ppm_b200_grid* g = io[k].g;
    ElemGrid& e = rec[k];
    std::memset(&e, 0, sizeof(e));
    e.d = io[k].user.f[0];
    e.te = io[k].user.f[1];
    e.v[0] = io[k].user.f[2];
    e.v[1] = g->rank > 1 ? io[k].user.f[3] : nullptr;
    e.v[2] = g->rank > 2 ? io[k].user.f[4] : nullptr;
    e.ge = p->dual_energy ? io[k].user.f[5] : nullptr;
    e.p = io[k].pres;
    for (int n = 0; n < 6; ++n) e.f[n] = io[k].user.f[n];
    if (!p->dual_energy) e.f[5] = nullptr;
    for (int d = 0; d < 3; ++d) {
      e.cw[d] = (with_cw && cwoff[k][d] >= 0) ? cw_dev + cwoff[k][d] : nullptr;
      e.dims[d] = g->dims[d];
      e.start[d] = g->start[d];
      e.end[d] = g->end[d];
      e.bc[d] = bc ? bc[d] : 0;
    }
    if (old)
      for (int n = 0; n < 6; ++n) e.old[n] = (*old)[k].f[n];
    e.rank = g->rank;
    e.size = grid_size(g);
    e.active = grid_active(g);
    spre[k + 1] = spre[k] + (e.size + 255) / 256;
    apre[k + 1] = apre[k] + (e.active + 255) / 256;
    const int64_t rows = (int64_t)g->dims[1] * g->dims[2];
    rpre[k + 1] = rpre[k] + (rows + kFillRowsPerBlock - 1) / kFillRowsPerBlock;
  }
  std::vector<unsigned char> img;
  append(img, rec.data(), rec.size());
  const size_t off_s = align256(img.size());
  img.resize(off_s);
  append(img, spre.data(), spre.size());
  const size_t off_a = align256(img.size());
  img.resize(off_a);
  append(img, apre.data(), apre.size());
  const size_t off_r = align256(img.size());
  img.resize(off_r);
  append(img, rpre.data(), rpre.size());
  int rc = mirror_put(ctx, ctx->mirror[slot], img);
  if (rc) return rc;
  unsigned char* base = (unsigned char*)ctx->mirror[slot].dev.p;
  plan.B.grids = (const ElemGrid*)base;
  plan.B.ngrids = ng;
  plan.B.size_prefix = (const int64_t*)(base + off_s);
  plan.B.active_prefix = (const int64_t*)(base + off_a);
  plan.B.row_prefix = (const int64_t*)(base + off_r);
  plan.B.gamma = p->gamma;
  plan.B.tiny_number = p->tiny_number;
  plan.B.min_support = p->min_support;
  plan.B.aye = 1.0;
  plan.B.vg[0] = plan.B.vg[1] = plan.B.vg[2] = 0.0;
  plan.B.min_bits = (unsigned long long*)ctx->misc.p;
  plan.B.expansion = plan.B.coef_new = plan.B.coef_old = 0.0;
  plan.B.interpolate = 0;
  plan.B.presfree = p->pressure_free == 1 ? 1 : 0;
  plan.B.eos_type = p->eos_type;
  plan.B.eos_cs = p->eos_sound_speed;
  plan.size_blocks = spre[ng];
  plan.active_blocks = apre[ng];
  plan.row_blocks = rpre[ng];
  return PPM_B200_OK;
}

// Resolve the device field set of a grid: device pointers as given, or the context's
// device copies of host fields (copied in here; single grid only).
// colours: also the colour fields (the sweeps; the other entry points do not read them).
int stage_in(ppm_b200_context* ctx, const ppm_b200_params* p, ppm_b200_grid* g, int memory,
             FieldSet& fs, const double* acc[3], bool colours = false, bool need_acc = false) {
  // the accelerations: read by the sweeps alone, which need one per axis under gravity
  const bool with_acc = need_acc && p->gravity;
  if (with_acc)
    for (int k = 0; k < g->rank; ++k)
      if (!g->acceleration[k]) return PPM_B200_ERR_INVALID;
  double* src[6] = {g->density, g->total_energy, g->velocity[0],
                    g->rank > 1 ? g->velocity[1] : nullptr,
                    g->rank > 2 ? g->velocity[2] : nullptr,
                    p->dual_energy ? g->gas_energy : nullptr};
  const size_t bytes = (size_t)grid_size(g) * sizeof(double);
  for (int k = 0; k < 3; ++k) acc[k] = nullptr;
  fs.ncol = colours ? p->number_of_colours : 0;
  if (memory == PPM_B200_MEM_DEVICE) {
    for (int k = 0; k < 6; ++k) fs.f[k] = src[k];
    for (int k = 0; k < g->rank; ++k) acc[k] = with_acc ? g->acceleration[k] : nullptr;
    for (int n = 0; n < fs.ncol; ++n) fs.col[n] = g->colours[n];
    return PPM_B200_OK;
  }
  if (memory != PPM_B200_MEM_HOST) return PPM_B200_ERR_INVALID;
  if (fs.ncol > 0) {
    int rc = ensure(ctx, ctx->host_col, bytes * (size_t)fs.ncol);
    if (rc) return rc;
    for (int n = 0; n < fs.ncol; ++n) {
      fs.col[n] = (double*)ctx->host_col.p + (size_t)n * (size_t)grid_size(g);
      CK(cudaMemcpyAsync(fs.col[n], g->colours[n], bytes, cudaMemcpyHostToDevice,
                         ctx->stream));
    }
  }
  for (int k = 0; k < 6; ++k) {
    fs.f[k] = nullptr;
    if (!src[k]) continue;
    int rc = ensure(ctx, ctx->host_set[k], bytes);
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->host_set[k].p, src[k], bytes, cudaMemcpyHostToDevice, ctx->stream));
    fs.f[k] = (double*)ctx->host_set[k].p;
  }
  if (with_acc) {
    for (int k = 0; k < g->rank; ++k) {
      int rc = ensure(ctx, ctx->host_acc[k], bytes);
      if (rc) return rc;
      CK(cudaMemcpyAsync(ctx->host_acc[k].p, g->acceleration[k], bytes, cudaMemcpyHostToDevice,
                         ctx->stream));
      acc[k] = (const double*)ctx->host_acc[k].p;
    }
  }
  return PPM_B200_OK;
}

int stage_out(ppm_b200_context* ctx, const ppm_b200_params* p, ppm_b200_grid* g,
              const FieldSet& fs) {
  double* dst[6] = {g->density, g->total_energy, g->velocity[0],
                    g->rank > 1 ? g->velocity[1] : nullptr,
                    g->rank > 2 ? g->velocity[2] : nullptr,
                    p->dual_energy ? g->gas_energy : nullptr};
  const size_t bytes = (size_t)grid_size(g) * sizeof(double);
  for (int k = 0; k < 6; ++k)
    if (dst[k] && fs.f[k])
      CK(cudaMemcpyAsync(dst[k], fs.f[k], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  for (int n = 0; n < fs.ncol; ++n)
    CK(cudaMemcpyAsync(g->colours[n], fs.col[n], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return PPM_B200_OK;
}

// Ring sets and pressure of every grid in one allocation each.
int assign_scratch(ppm_b200_context* ctx, std::vector<GridIO>& io) {
  size_t ring_doubles = 0, pres_doubles = 0;
  for (auto& x : io) {
    int nf = 0;
    for (int k = 0; k < 6; ++k) nf += x.user.f[k] ? 1 : 0;
    ring_doubles += 2 * (size_t)nf * (size_t)grid_size(x.g);
    pres_doubles += (size_t)grid_size(x.g);
  }
  int rc = ensure(ctx, ctx->ring, std::max<size_t>(ring_doubles, 1) * sizeof(double));
  if (rc) return rc;
  rc = ensure(ctx, ctx->pressure, std::max<size_t>(pres_doubles, 1) * sizeof(double));
  if (rc) return rc;
  double* r = (double*)ctx->ring.p;
  double* pr = (double*)ctx->pressure.p;
  for (auto& x : io) {
    const size_t n = (size_t)grid_size(x.g);
    for (int s = 0; s < 2; ++s)
      for (int k = 0; k < 6; ++k) {
        x.ring[s].f[k] = nullptr;
        if (!x.user.f[k]) continue;
        x.ring[s].f[k] = r;
        r += n;
      }
    x.pres = pr;
    pr += n;
  }
  return PPM_B200_OK;
}

// The sweep order of Grid_SolvePPM_DE.C:53, :86-146 (all grids of a batch share rank).
int sweep_order(const ppm_b200_grid* g, int cycle, int order[3]) {
  const int rank = g->rank;
  const int nact[3] = {g->end[0] - g->start[0] + 1, rank > 1 ? g->end[1] - g->start[1] + 1 : 1,
                       rank > 2 ? g->end[2] - g->start[2] + 1 : 1};
  int n = 0;
  const int ixyz = cycle % rank;
  for (int k = ixyz; k < ixyz + rank; ++k) {
    const int dim = k % rank;
    if (nact[dim] > 1) order[n++] = dim;
  }
  return n;
}

// Plans for pressure + the sweeps of one SolvePPM_DE over a batch; captures only for a
// single grid.  Ring: user -> S0 [-> S1] -> user; a single sweep is copied back.
struct SolvePlan {
  ElemPlan pressure;
  SweepPlan sweep[3];
  int order[3];
  int nsweeps = 0;
};

int prepare_solve(ppm_b200_context* ctx, const ppm_b200_params* p, int cycle,
                  std::vector<GridIO>& io, int nsub, ppm_b200_fluxes* sub, const long long ggs[3],
                  SolvePlan& sp) {
  int rc = assign_scratch(ctx, io);
  if (rc) return rc;
  rc = prepare_elem(ctx, kSlotPressure, p, io, false, nullptr, sp.pressure);
  if (rc) return rc;
  sp.nsweeps = sweep_order(io[0].g, cycle, sp.order);
  for (size_t k = 1; k < io.size(); ++k) {
    int o2[3];
    const int n2 = sweep_order(io[k].g, cycle, o2);
    if (n2 != sp.nsweeps) return PPM_B200_ERR_INVALID;
    for (int s = 0; s < n2; ++s)
      if (o2[s] != sp.order[s]) return PPM_B200_ERR_INVALID;
  }
  const int ng = (int)io.size();
  for (int s = 0; s < sp.nsweeps; ++s) {
    rc = build_captures(io[0].g, sp.order[s], ng == 1 ? nsub : 0, sub, ggs, sp.sweep[s]);
    if (rc) return rc;
  }
  rc = reserve_captures(ctx, sp.sweep, sp.nsweeps, p->number_of_colours);
  if (rc) return rc;
  // one face scratch serves the sweeps in turn: size it for the largest before any
  // sweep records its pointers
  size_t scratch = 0;
  for (int s = 0; s < sp.nsweeps; ++s)
    scratch = std::max(scratch, sweep_scratch_bytes(sp.order[s], io, p));
  rc = ensure(ctx, ctx->face_scratch, scratch);
  if (rc) return rc;
  const void* scratch_base = ctx->face_scratch.p;
  for (int s = 0; s < sp.nsweeps; ++s) {
    const int in_set = (s == 0) ? -1 : (s - 1) % 2;
    const int out_set = (s == sp.nsweeps - 1 && sp.nsweeps >= 2) ? -1 : s % 2;
    std::vector<int> src(ng, in_set), dst(ng, out_set);
    const bool cfl = ctx->cfl_dt != nullptr && s == sp.nsweeps - 1;
    rc = prepare_sweep(ctx, sp.order[s], s, p, io, src, dst, sp.sweep[s], cfl);
    if (rc) return rc;
  }
  if (ctx->face_scratch.p != scratch_base) {  // would leave earlier sweeps on freed memory
    fprintf(stderr, "ppm_b200: face scratch moved while sweeps were prepared\n");
    return PPM_B200_ERR_CUDA;
  }
  return PPM_B200_OK;
}

// cfl_first / cfl_last: this solve is the first / last of a level's waves, which share
// one folded time step: the minimum is reset before the first wave's last sweep and the
// time step written after the last wave's (every wave reads the old one until then).
int enqueue_solve(ppm_b200_context* ctx, const ppm_b200_params* p, const std::vector<GridIO>& io,
                  const SolvePlan& sp, bool capturing, bool cfl_first = true,
                  bool cfl_last = true) {
  ppm::launch_pressure_batch(sp.pressure.B, sp.pressure.size_blocks, ctx->stream);
  ctx->launches += 1;
  CK(cudaGetLastError());
  unsigned long long* cfl_bits = ((unsigned long long*)ctx->misc.p) + 2;
  for (int s = 0; s < sp.nsweeps; ++s) {
    const bool cfl = ctx->cfl_dt != nullptr && s == sp.nsweeps - 1;
    if (cfl && cfl_first) ppm::launch_cfl_reset(cfl_bits, ctx->stream);
    int rc = enqueue_sweep(ctx, sp.sweep[s], p, capturing);
    if (rc) return rc;
    if (cfl && cfl_last) {
      ppm::launch_cfl_finalize(cfl_bits, ctx->cfl_courant, ctx->cfl_dt, ctx->stream);
      ctx->launches += 1;
      CK(cudaGetLastError());
    }
  }
  if (sp.nsweeps == 1) {
    for (const auto& x : io) {
      const size_t bytes = (size_t)grid_size(x.g) * sizeof(double);
      for (int k = 0; k < 6; ++k)
        if (x.user.f[k])
          CK(cudaMemcpyAsync(x.user.f[k], x.ring[0].f[k], bytes, cudaMemcpyDeviceToDevice,
                             ctx->stream));
    }
  }
  if (p->eos_type > 0) {  // energies consistent with the EOS again (Grid_SolvePPM_DE.C:155-157)
    ppm::launch_pressure_batch(sp.pressure.B, sp.pressure.size_blocks, ctx->stream);
    ctx->launches += 1;
    CK(cudaGetLastError());
  }
  return PPM_B200_OK;
}

// ------------------------------------------------------------ level schedules (waves)
// A wave: grids of a level solved as one batch (indices into the level's io list, which
// is sorted largest first), with the Riemann settings of that batch.
struct Wave {
  std::vector<int> grids;
  int riemann_threads = ppm::kRiemannThreads;
  int persistent = 0;
};

int size_class(const ppm_b200_context* ctx, const ppm_b200_grid* g) {
  const long long a = grid_active(g);
  if (a < ctx->level.class_cells[0]) return 0;
  if (a < ctx->level.class_cells[1]) return 1;
  return 2;
}

// Device bytes a batch of grids takes beyond its fields: two ring sets and the pressure
// per grid, and the face scratch of its largest sweep direction.
size_t batch_scratch_bytes(const ppm_b200_params* p, const std::vector<GridIO>& io,
                           const std::vector<int>& idx) {
  size_t fields = 0;
  std::vector<GridIO> sub;
  for (int k : idx) {
    const GridIO& x = io[k];
    int nf = 0;
    for (int f = 0; f < 6; ++f) nf += x.user.f[f] ? 1 : 0;
    fields += (2 * (size_t)nf + 1) * (size_t)grid_size(x.g) * sizeof(double);
    sub.push_back(x);
  }
  size_t faces = 0;
  if (!sub.empty())
    for (int d = 0; d < sub[0].g->rank; ++d) faces = std::max(faces, sweep_scratch_bytes(d, sub, p));
  return fields + faces;
}

// The waves of a level solve under the context's level configuration.
void plan_waves(const ppm_b200_context* ctx, const ppm_b200_params* p,
                const std::vector<GridIO>& io, std::vector<Wave>& waves) {
  const ppm_b200_level_config& c = ctx->level;
  const int ng = (int)io.size();
  waves.clear();
  auto rt_of = [](int v) { return (v == 64 || v == 256) ? v : (int)ppm::kRiemannThreads; };
  if (c.schedule == PPM_B200_LEVEL_PER_GRID) {
    for (int k = 0; k < ng; ++k) {
      Wave w;
      w.grids.push_back(k);
      w.riemann_threads = rt_of(c.riemann_threads[3]);
      w.persistent = c.persistent[3] != 0;
      waves.push_back(w);
    }
    return;
  }
  // groups: all grids, or the size classes in order (largest first, as io is sorted)
  std::vector<std::vector<int>> groups;
  std::vector<int> group_cfg;
  if (c.schedule == PPM_B200_LEVEL_CLASSES) {
    for (int cls = 2; cls >= 0; --cls) {
      std::vector<int> gcls;
      for (int k = 0; k < ng; ++k)
        if (size_class(ctx, io[k].g) == cls) gcls.push_back(k);
      if (!gcls.empty()) {
        groups.push_back(gcls);
        group_cfg.push_back(cls);
      }
    }
  } else {
    std::vector<int> all(ng);
    for (int k = 0; k < ng; ++k) all[k] = k;
    groups.push_back(all);
    group_cfg.push_back(3);
  }
  // each group cut into waves that fit the scratch bound (a grid alone always fits)
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    Wave w;
    w.riemann_threads = rt_of(c.riemann_threads[group_cfg[gi]]);
    w.persistent = c.persistent[group_cfg[gi]] != 0;
    for (int k : groups[gi]) {
      if (c.max_scratch_bytes > 0 && !w.grids.empty()) {
        std::vector<int> trial = w.grids;
        trial.push_back(k);
        if (batch_scratch_bytes(p, io, trial) > (size_t)c.max_scratch_bytes) {
          waves.push_back(w);
          w.grids.clear();
        }
      }
      w.grids.push_back(k);
    }
    if (!w.grids.empty()) waves.push_back(w);
  }
}

// Sizes the ring sets, pressure and face scratch for the largest wave before any wave is
// prepared, so no later wave moves a buffer an earlier one recorded.
int reserve_level_scratch(ppm_b200_context* ctx, const ppm_b200_params* p,
                          const std::vector<GridIO>& io, const std::vector<Wave>& waves) {
  size_t ring = 0, pres = 0, faces = 0;
  for (const Wave& w : waves) {
    size_t r = 0, q = 0;
    std::vector<GridIO> sub;
    for (int k : w.grids) {
      const GridIO& x = io[k];
      int nf = 0;
      for (int f = 0; f < 6; ++f) nf += x.user.f[f] ? 1 : 0;
      r += 2 * (size_t)nf * (size_t)grid_size(x.g);
      q += (size_t)grid_size(x.g);
      sub.push_back(x);
    }
    ring = std::max(ring, r);
    pres = std::max(pres, q);
    for (int d = 0; d < sub[0].g->rank; ++d) faces = std::max(faces, sweep_scratch_bytes(d, sub, p));
  }
  int rc = ensure(ctx, ctx->ring, std::max<size_t>(ring, 1) * sizeof(double));
  if (rc) return rc;
  rc = ensure(ctx, ctx->pressure, std::max<size_t>(pres, 1) * sizeof(double));
  if (rc) return rc;
  return ensure(ctx, ctx->face_scratch, faces);
}

// Graph key: the by-value launch arguments of a level solve (kernel parameter structs,
// block counts, flags) and the versions of the sweep descriptor images, which hold the
// field pointers that a one-sweep solve also copies by value.  Descriptor and table
// contents are read by the kernels when the graph runs, so they need no key.
template <class T>
void key_put(std::string& k, const T& v) {
  k.append(reinterpret_cast<const char*>(&v), sizeof(T));
}

std::string graph_key(ppm_b200_context* ctx, const ppm_b200_params* p, const SolvePlan& sp) {
  std::string k;
  key_put(k, ctx->cfl_dt);
  key_put(k, ctx->cfl_courant);
  key_put(k, p->learned_guess);
  key_put(k, p->dual_energy);
  key_put(k, p->gravity);
  key_put(k, sp.nsweeps);
  const ElemBatch& e = sp.pressure.B;
  key_put(k, e.grids);
  key_put(k, e.ngrids);
  key_put(k, e.size_prefix);
  key_put(k, e.active_prefix);
  key_put(k, e.row_prefix);
  key_put(k, e.gamma);
  key_put(k, e.tiny_number);
  key_put(k, e.min_support);
  key_put(k, e.eos_type);
  key_put(k, e.eos_cs);
  key_put(k, e.min_bits);
  key_put(k, sp.pressure.size_blocks);
  for (int s = 0; s < sp.nsweeps; ++s) {
    const BatchArgs& b = sp.sweep[s].B;
    key_put(k, sp.order[s]);
    key_put(k, b.grids);
    key_put(k, b.ngrids);
    key_put(k, b.march_prefix);
    key_put(k, b.riemann_prefix);
    key_put(k, b.counters);
    key_put(k, b.flagged);
    key_put(k, sp.sweep[s].march_blocks);
    key_put(k, sp.sweep[s].riemann_blocks);
    key_put(k, sp.sweep[s].contiguous);
    key_put(k, b.x_tma);
    key_put(k, b.x_tma_extra_tx);
    key_put(k, b.corrections);
    key_put(k, b.ncolour);
    key_put(k, b.solver);
    key_put(k, b.presfree);
    key_put(k, b.hll_flags);
    key_put(k, b.hll_bytes);
    key_put(k, b.riemann_threads);
    key_put(k, b.persistent);
    key_put(k, b.riemann_total);
    key_put(k, b.fused);
    key_put(k, b.face_prefix);
    key_put(k, b.face_blocks);
    key_put(k, ctx->mirror[kSlotSweep0 + 3 * sp.order[s] + s].version);
  }
  return k;
}

int finish_status(ppm_b200_context* ctx, ppm_b200_stats* stats) {
  int status = PPM_B200_OK;
  int rc = read_counters(ctx, stats, &status);
  if (rc) return rc;
  return status;
}

}  // namespace

extern "C" {

int ppm_b200_version(void) { return PPM_B200_VERSION; }

int ppm_b200_abi_check(const long long* layout, int n) {
  static const long long mine[] = {PPM_B200_ABI_LAYOUT(PPM_B200_ABI_ITEM)};
  const int count = (int)(sizeof(mine) / sizeof(mine[0]));
  if (!layout || n != count) return PPM_B200_ERR_INVALID;
  for (int i = 0; i < count; ++i)
    if (layout[i] != mine[i]) return PPM_B200_ERR_INVALID;
  return PPM_B200_OK;
}

const char* ppm_b200_error_string(int code) {
  switch (code) {
    case PPM_B200_OK: return "ok";
    case PPM_B200_ERR_UNSUPPORTED: return "configuration not supported by ppm_b200";
    case PPM_B200_ERR_INVALID: return "invalid argument";
    case PPM_B200_ERR_CUDA: return "CUDA runtime error";
    case PPM_B200_ERR_NEGATIVE: return "negative density or energy the reference aborts on";
    case PPM_B200_ERR_NONFINITE: return "non-finite value in the output";
    case PPM_B200_ERR_TOO_LARGE: return "size exceeds the fixed limit of this entry point";
    case PPM_B200_ERR_TIMEOUT: return "a bounded device wait on an asynchronous copy gave up";
    default: return "unknown error";
  }
}

int ppm_b200_create(int device, void* cuda_stream, ppm_b200_context** out) {
  if (!out) return PPM_B200_ERR_INVALID;
  *out = nullptr;
  ppm_b200_context* ctx = new ppm_b200_context();
  ctx->device = device;
  select_bank(ctx, 0);
  ctx->level.schedule = PPM_B200_LEVEL_BATCHED;
  for (int k = 0; k < 4; ++k) {
    ctx->level.riemann_threads[k] = ppm::kRiemannThreads;
    ctx->level.persistent[k] = 0;
  }
  ctx->level.class_cells[0] = 48LL * 48 * 48;
  ctx->level.class_cells[1] = 96LL * 96 * 96;
  ctx->level.max_scratch_bytes = 0;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    delete ctx;
    return cuda_fail(nullptr, e, "cudaSetDevice");
  }
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
  if (cuda_stream) {
    ctx->stream = (cudaStream_t)cuda_stream;
  } else {
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete ctx;
      return cuda_fail(nullptr, e, "cudaStreamCreate");
    }
    ctx->own_stream = true;
  }
  int rc = ensure(ctx, ctx->counters, ppm::kMaxCounters * sizeof(unsigned long long));
  if (!rc) rc = ensure(ctx, ctx->misc, 4 * sizeof(double));
  if (!rc) rc = cuda_fail(ctx, cudaMemset(ctx->counters.p, 0, ctx->counters.bytes), "cudaMemset");
  if (rc) {
    ppm_b200_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return PPM_B200_OK;
}

int ppm_b200_destroy(ppm_b200_context* ctx) {
  if (!ctx) return PPM_B200_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  drop_graphs(ctx);
  auto fr = [](DevBuf& b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
  };
  for (auto& b : ctx->host_set) fr(b);
  for (auto& b : ctx->host_acc) fr(b);
  for (auto& b : ctx->host_old) fr(b);
  fr(ctx->host_col);
  fr(ctx->ring);
  fr(ctx->pressure);
  fr(ctx->face_scratch);
  fr(ctx->counters);
  fr(ctx->misc);
  fr(ctx->captures);
  fr(ctx->capture_buf);
  fr(ctx->col_capture);
  fr(ctx->flux_fix);
  fr(ctx->guess);
  fr(ctx->log_count);
  for (auto& bank : ctx->banks)
    for (auto& m : *bank) {
      fr(m.dev);
      mirror_free(m);
    }
  for (auto e : ctx->ev_pool) cudaEventDestroy(e);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return PPM_B200_OK;
}

long long ppm_b200_launch_count(ppm_b200_context* ctx) { return ctx ? ctx->launches : -1; }

int ppm_b200_profile(ppm_b200_context* ctx, int enable) {
  if (!ctx) return PPM_B200_ERR_INVALID;
  ctx->profiling = enable != 0;
  return PPM_B200_OK;
}

int ppm_b200_profile_read(ppm_b200_context* ctx, double* sweep_ms, long long* sweep_launches) {
  if (!ctx) return PPM_B200_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  double total = 0.0;
  double stage[kSweepEvents - 1] = {0, 0, 0, 0, 0};
  for (size_t k = 0; k + kSweepEvents <= ctx->ev_used; k += kSweepEvents) {
    for (int j = 0; j + 1 < kSweepEvents; ++j) {
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, ctx->ev_pool[k + j], ctx->ev_pool[k + j + 1]));
      stage[j] += ms;
      total += ms;
    }
  }
  if (sweep_ms) *sweep_ms = total;
  if (sweep_launches) *sweep_launches = (long long)(ctx->ev_used / kSweepEvents);
  for (int j = 0; j + 1 < kSweepEvents; ++j) ctx->stage_ms[j] = stage[j];
  ctx->ev_used = 0;
  return PPM_B200_OK;
}

int ppm_b200_profile_stages(ppm_b200_context* ctx, double stage_ms[5]) {
  if (!ctx || !stage_ms) return PPM_B200_ERR_INVALID;
  for (int j = 0; j < 5; ++j) stage_ms[j] = ctx->stage_ms[j];
  return PPM_B200_OK;
}

int ppm_b200_device_bytes(ppm_b200_context* ctx, long long* bytes) {
  if (!ctx || !bytes) return PPM_B200_ERR_INVALID;
  size_t n = 0;
  for (const DevBuf* b : {&ctx->host_set[0], &ctx->host_set[1], &ctx->host_set[2],
                          &ctx->host_set[3], &ctx->host_set[4], &ctx->host_set[5],
                          &ctx->host_acc[0], &ctx->host_acc[1], &ctx->host_acc[2],
                          &ctx->host_col, &ctx->ring, &ctx->pressure, &ctx->face_scratch,
                          &ctx->counters, &ctx->misc, &ctx->captures, &ctx->capture_buf,
                          &ctx->col_capture, &ctx->flux_fix, &ctx->guess, &ctx->log_count})
    n += b->bytes;
  for (const auto& bank : ctx->banks)
    for (const auto& m : *bank) n += m.dev.bytes;
  *bytes = (long long)n;
  return PPM_B200_OK;
}

int ppm_b200_set_sweep_mode(ppm_b200_context* ctx, int mode) {
  if (!ctx || (mode != PPM_B200_SWEEP_SPLIT && mode != PPM_B200_SWEEP_FUSED))
    return PPM_B200_ERR_INVALID;
  ctx->sweep_mode = mode;
  return PPM_B200_OK;
}

int ppm_b200_set_level_config(ppm_b200_context* ctx, const ppm_b200_level_config* cfg) {
  if (!ctx || !cfg) return PPM_B200_ERR_INVALID;
  if (cfg->schedule < PPM_B200_LEVEL_BATCHED || cfg->schedule > PPM_B200_LEVEL_PER_GRID)
    return PPM_B200_ERR_INVALID;
  for (int k = 0; k < 4; ++k)
    if (cfg->riemann_threads[k] != 64 && cfg->riemann_threads[k] != 128 &&
        cfg->riemann_threads[k] != 256)
      return PPM_B200_ERR_INVALID;
  if (cfg->class_cells[0] < 0 || cfg->class_cells[1] < cfg->class_cells[0] ||
      cfg->max_scratch_bytes < 0)
    return PPM_B200_ERR_INVALID;
  ctx->level = *cfg;
  return PPM_B200_OK;
}

int ppm_b200_get_level_config(ppm_b200_context* ctx, ppm_b200_level_config* cfg) {
  if (!ctx || !cfg) return PPM_B200_ERR_INVALID;
  *cfg = ctx->level;
  return PPM_B200_OK;
}

int ppm_b200_autotune_level(ppm_b200_context* ctx, const ppm_b200_params* p, int cycle_number,
                            ppm_b200_grid* grids, int ngrids, ppm_b200_level_tuning* rep) {
  if (!ctx || !p || !grids || ngrids <= 0) return PPM_B200_ERR_INVALID;
  int rc = check_supported(p);
  if (rc) return rc;
  // the tuned settings apply to the two-shock stage with the plain start
  if (p->number_of_colours > 0 || p->learned_guess || solver_code(p) != 0 ||
      p->pressure_free == 1)
    return PPM_B200_ERR_UNSUPPORTED;
  for (int k = 0; k < ngrids; ++k) {
    rc = check_grid(&grids[k], p);
    if (rc) return rc;
  }
  CK(cudaSetDevice(ctx->device));
  // copies of every grid's fields: the tuning solves advance these, not the caller's
  std::vector<ppm_b200_grid> cg(grids, grids + ngrids);
  size_t doubles = 0;
  for (int k = 0; k < ngrids; ++k) {
    const ppm_b200_grid& g = grids[k];
    const size_t n = (size_t)grid_size(&g);
    doubles += n * (2 + (size_t)g.rank + (p->dual_energy ? 1 : 0));
  }
  DevBuf copies;
  rc = ensure(ctx, copies, doubles * sizeof(double));
  if (rc) return rc;
  double* at = (double*)copies.p;
  for (int k = 0; k < ngrids; ++k) {
    ppm_b200_grid& g = cg[k];
    const size_t n = (size_t)grid_size(&g);
    auto take = [&](double*& f) -> int {
      if (!f) return PPM_B200_OK;
      CK(cudaMemcpyAsync(at, f, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
      f = at;
      at += n;
      return PPM_B200_OK;
    };
    int r = take(g.density);
    if (!r) r = take(g.total_energy);
    for (int d = 0; d < 3 && !r; ++d) r = d < g.rank ? take(g.velocity[d]) : PPM_B200_OK;
    if (!r && p->dual_energy) r = take(g.gas_energy);
    if (r) {
      cudaFree(copies.p);
      return r;
    }
  }
  // the tuning solves neither fold a time step nor replay graphs; the caller's settings
  // come back afterwards
  const ppm_b200_level_config saved = ctx->level;
  double* const saved_cfl = ctx->cfl_dt;
  const bool saved_graphs = ctx->use_graphs;
  ctx->cfl_dt = nullptr;
  ctx->use_graphs = false;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int err = PPM_B200_OK;
  auto time_level = [&](const ppm_b200_level_config& cfg, std::vector<ppm_b200_grid>& list) {
    ctx->level = cfg;
    if (err || list.empty()) return 0.0;
    int r = ppm_b200_solve_level(ctx, p, cycle_number, list.data(), (int)list.size(), nullptr);
    if (!r && cudaEventRecord(e0, ctx->stream) != cudaSuccess) r = PPM_B200_ERR_CUDA;
    if (!r) r = ppm_b200_solve_level(ctx, p, cycle_number, list.data(), (int)list.size(), nullptr);
    if (!r && cudaEventRecord(e1, ctx->stream) != cudaSuccess) r = PPM_B200_ERR_CUDA;
    float ms = 0.0f;
    if (!r && (cudaEventSynchronize(e1) != cudaSuccess ||
               cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
      r = PPM_B200_ERR_CUDA;
    if (r) err = r;
    return (double)ms;
  };
  const int threads[3] = {64, 128, 256};
  auto candidate = [&](int sched, int slot, int k) {
    ppm_b200_level_config c = saved;
    c.schedule = sched;
    c.max_scratch_bytes = saved.max_scratch_bytes;
    c.riemann_threads[slot] = threads[k / 2];
    c.persistent[slot] = k % 2;
    return c;
  };
  ppm_b200_level_tuning t;
  std::memset(&t, 0, sizeof(t));
  int best_class[3] = {2, 2, 2};  // candidate index: 128 faces, not persistent
  for (int cls = 0; cls < 3; ++cls) {
    std::vector<ppm_b200_grid> list;
    for (const auto& g : cg)
      if (size_class(ctx, &g) == cls) {
        list.push_back(g);
        t.class_active[cls] += grid_active(&g);
      }
    t.class_grids[cls] = (int)list.size();
    double best = 0.0;
    for (int k = 0; k < 6 && !list.empty(); ++k) {
      t.class_ms[cls][k] = time_level(candidate(PPM_B200_LEVEL_BATCHED, 3, k), list);
      if (k == 0 || t.class_ms[cls][k] < best) {
        best = t.class_ms[cls][k];
        best_class[cls] = k;
      }
    }
  }
  int best_all = 2;
  for (int k = 0; k < 6; ++k) {
    t.batched_ms[k] = time_level(candidate(PPM_B200_LEVEL_BATCHED, 3, k), cg);
    if (t.batched_ms[k] < t.batched_ms[best_all]) best_all = k;
  }
  ppm_b200_level_config by_class = saved;
  by_class.schedule = PPM_B200_LEVEL_CLASSES;
  for (int cls = 0; cls < 3; ++cls) {
    by_class.riemann_threads[cls] = threads[best_class[cls] / 2];
    by_class.persistent[cls] = best_class[cls] % 2;
  }
  t.classes_ms = time_level(by_class, cg);
  ppm_b200_level_config chosen = candidate(PPM_B200_LEVEL_BATCHED, 3, best_all);
  if (t.classes_ms < t.batched_ms[best_all]) chosen = by_class;
  t.chosen = chosen;
  // restore, drop the counters of the tuning solves, free the copies
  ctx->level = err ? saved : chosen;
  ctx->cfl_dt = saved_cfl;
  ctx->use_graphs = saved_graphs;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int status = PPM_B200_OK;
  int r2 = read_counters(ctx, nullptr, &status);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(copies.p);
  if (err) return err;
  if (r2) return r2;
  if (rep) *rep = t;
  return status;
}

int ppm_b200_set_graphs(ppm_b200_context* ctx, int enable) {
  if (!ctx) return PPM_B200_ERR_INVALID;
  if (!enable && !ctx->graphs.empty()) CK(cudaStreamSynchronize(ctx->stream));
  ctx->use_graphs = enable != 0;
  if (!ctx->use_graphs) drop_graphs(ctx);
  return PPM_B200_OK;
}

int ppm_b200_synchronize(ppm_b200_context* ctx, ppm_b200_stats* stats) {
  if (!ctx) return PPM_B200_ERR_INVALID;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->stream));
  int status = PPM_B200_OK;
  int rc = read_counters(ctx, stats, &status);
  if (rc) return rc;
  if (ctx->sticky_error) {
    rc = ctx->sticky_error;
    ctx->sticky_error = 0;
    return rc;
  }
  return status;
}

int ppm_b200_solve_ppm_de(ppm_b200_context* ctx, const ppm_b200_params* p, int cycle_number,
                          ppm_b200_grid* g, int memory, int nsub, ppm_b200_fluxes* sub,
                          const long long ggs_in[3], ppm_b200_stats* stats) {
  if (!ctx || !p || !g) return PPM_B200_ERR_INVALID;
  int rc = check_supported(p);
  if (rc) return rc;
  rc = check_grid(g, p);
  if (rc) return rc;
  rc = check_guess(ctx, p);
  if (rc) return rc;
  if (nsub > 0 && !sub) return PPM_B200_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  const long long zero3[3] = {0, 0, 0};
  const long long* ggs = ggs_in ? ggs_in : zero3;
  std::vector<GridIO> io(1);
  io[0].g = g;
  rc = stage_in(ctx, p, g, memory, io[0].user, io[0].acc, true, true);
  if (rc) return rc;
  SolvePlan sp;
  rc = prepare_solve(ctx, p, cycle_number, io, nsub, sub, ggs, sp);
  if (rc) return rc;
  rc = enqueue_solve(ctx, p, io, sp, false);
  if (rc) return rc;
  for (int s = 0; s < sp.nsweeps; ++s) {
    rc = scatter_captures(ctx, sp.order[s], p, g, sp.sweep[s], sub);
    if (rc) return rc;
  }
  if (memory == PPM_B200_MEM_HOST) {
    rc = stage_out(ctx, p, g, io[0].user);
    if (rc) return rc;
  }
  if (memory == PPM_B200_MEM_HOST || stats || nsub > 0) return finish_status(ctx, stats);
  return PPM_B200_OK;
}

int ppm_b200_solve_level(ppm_b200_context* ctx, const ppm_b200_params* p, int cycle_number,
                         ppm_b200_grid* grids, int ngrids, ppm_b200_stats* stats) {
  if (!ctx || !p || !grids || ngrids <= 0) return PPM_B200_ERR_INVALID;
  int rc = check_supported(p);
  if (rc) return rc;
  for (int k = 0; k < ngrids; ++k) {
    rc = check_grid(&grids[k], p);
    if (rc) return rc;
    if (grids[k].rank != grids[0].rank) return PPM_B200_ERR_INVALID;
  }
  rc = check_guess(ctx, p);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  // largest grids first: the block scheduler then starts the longest pencils first
  std::vector<int> idx(ngrids);
  for (int k = 0; k < ngrids; ++k) idx[k] = k;
  std::stable_sort(idx.begin(), idx.end(),
                   [&](int x, int y) { return grid_size(&grids[x]) > grid_size(&grids[y]); });
  std::vector<GridIO> io(ngrids);
  for (int k = 0; k < ngrids; ++k) {
    io[k].g = &grids[idx[k]];
    rc = stage_in(ctx, p, &grids[idx[k]], PPM_B200_MEM_DEVICE, io[k].user, io[k].acc, true,
                  true);
    if (rc) return rc;
  }
  // the level's waves (one for the batched schedule without a scratch bound), each
  // prepared into its own descriptor bank with its Riemann settings
  std::vector<Wave> waves;
  plan_waves(ctx, p, io, waves);
  rc = reserve_level_scratch(ctx, p, io, waves);
  if (rc) return rc;
  std::vector<SolvePlan> plans(waves.size());
  std::vector<std::vector<GridIO>> wio(waves.size());
  std::string key;
  for (size_t w = 0; w < waves.size(); ++w) {
    for (int k : waves[w].grids) wio[w].push_back(io[k]);
    select_bank(ctx, w);
    ctx->wave_rt = waves[w].riemann_threads;
    ctx->wave_persist = waves[w].persistent;
    rc = prepare_solve(ctx, p, cycle_number, wio[w], 0, nullptr, nullptr, plans[w]);
    if (rc == PPM_B200_OK) key += graph_key(ctx, p, plans[w]);
    if (rc) break;
  }
  select_bank(ctx, 0);
  ctx->wave_rt = ppm::kRiemannThreads;
  ctx->wave_persist = 0;
  if (rc) return rc;
  auto enqueue_all = [&](bool capturing) {
    for (size_t w = 0; w < waves.size(); ++w) {
      int r = enqueue_solve(ctx, p, wio[w], plans[w], capturing, w == 0,
                            w + 1 == waves.size());
      if (r) return r;
    }
    return (int)PPM_B200_OK;
  };
  // graph replay needs every per-step value on the device (dt included)
  const bool graph = ctx->use_graphs && p->dt_device != nullptr && !ctx->profiling;
  if (graph) {
    auto it = ctx->graphs.find(key);
    if (it == ctx->graphs.end()) {
      if (ctx->graphs.size() >= kMaxGraphs) {
        CK(cudaStreamSynchronize(ctx->stream));
        drop_graphs(ctx);
      }
      cudaGraph_t gr;
      CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      const long long before = ctx->launches;
      rc = enqueue_all(true);
      cudaError_t e = cudaStreamEndCapture(ctx->stream, &gr);
      if (rc) return rc;
      if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
      cudaGraphExec_t ex;
      e = cudaGraphInstantiate(&ex, gr, 0);
      cudaGraphDestroy(gr);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
      ctx->launches = before;  // counted when the graph runs
      it = ctx->graphs.emplace(key, ex).first;
    }
    CK(cudaGraphLaunch(it->second, ctx->stream));
    for (const auto& sp : plans)
      ctx->launches += 1 + sweep_kernels(p) * sp.nsweeps + (p->eos_type > 0 ? 1 : 0);
    if (ctx->cfl_dt) ctx->launches += 1;  // the folded time step's finalize kernel
  } else {
    rc = enqueue_all(false);
    if (rc) return rc;
  }
  if (stats) return finish_status(ctx, stats);
  return PPM_B200_OK;
}

int ppm_b200_euler_sweep(ppm_b200_context* ctx, int dim, const ppm_b200_params* p,
                         ppm_b200_grid* g, const double* pressure, int memory, int nsub,
                         ppm_b200_fluxes* sub, const long long ggs_in[3], ppm_b200_stats* stats) {
  if (!ctx || !p || !g || !pressure || dim < 0 || dim > 2) return PPM_B200_ERR_INVALID;
  int rc = check_supported(p);
  if (rc) return rc;
  rc = check_grid(g, p);
  if (rc) return rc;
  if (dim >= g->rank) return PPM_B200_ERR_INVALID;
  rc = check_guess(ctx, p);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  const long long zero3[3] = {0, 0, 0};
  const long long* ggs = ggs_in ? ggs_in : zero3;
  std::vector<GridIO> io(1);
  io[0].g = g;
  rc = stage_in(ctx, p, g, memory, io[0].user, io[0].acc, true, true);
  if (rc) return rc;
  rc = assign_scratch(ctx, io);
  if (rc) return rc;
  if (memory == PPM_B200_MEM_HOST) {
    CK(cudaMemcpyAsync(io[0].pres, pressure, (size_t)grid_size(g) * sizeof(double),
                       cudaMemcpyHostToDevice, ctx->stream));
  } else {
    io[0].pres = const_cast<double*>(pressure);
  }
  SweepPlan plan;
  rc = build_captures(g, dim, nsub, sub, ggs, plan);
  if (rc) return rc;
  rc = reserve_captures(ctx, &plan, 1, p->number_of_colours);
  if (rc) return rc;
  std::vector<int> src(1, -1), dst(1, 0);
  rc = prepare_sweep(ctx, dim, 0, p, io, src, dst, plan);
  if (rc) return rc;
  rc = enqueue_sweep(ctx, plan, p, false);
  if (rc) return rc;
  rc = scatter_captures(ctx, dim, p, g, plan, sub);
  if (rc) return rc;
  const size_t bytes = (size_t)grid_size(g) * sizeof(double);
  for (int k = 0; k < 6; ++k)
    if (io[0].user.f[k])
      CK(cudaMemcpyAsync(io[0].user.f[k], io[0].ring[0].f[k], bytes, cudaMemcpyDeviceToDevice,
                         ctx->stream));
  if (memory == PPM_B200_MEM_HOST) {
    rc = stage_out(ctx, p, g, io[0].user);
    if (rc) return rc;
  }
  if (memory == PPM_B200_MEM_HOST || stats || nsub > 0) return finish_status(ctx, stats);
  return PPM_B200_OK;
}

int ppm_b200_compute_pressure(ppm_b200_context* ctx, const ppm_b200_params* p, ppm_b200_grid* g,
                              double* pressure, int memory) {
  if (!ctx || !p || !g || !pressure) return PPM_B200_ERR_INVALID;
  // this call does not read the acceleration: a gravity run's grids need none here
  ppm_b200_params q = *p;
  q.gravity = 0;
  p = &q;
  if (p->eos_type != 0 && p->eos_type != 3) return PPM_B200_ERR_UNSUPPORTED;
  int rc = check_grid(g, p);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  std::vector<GridIO> io(1);
  io[0].g = g;
  rc = stage_in(ctx, p, g, memory, io[0].user, io[0].acc);
  if (rc) return rc;
  if (memory == PPM_B200_MEM_HOST) {
    rc = ensure(ctx, ctx->pressure, (size_t)grid_size(g) * sizeof(double));
    if (rc) return rc;
    io[0].pres = (double*)ctx->pressure.p;
  } else {
    io[0].pres = pressure;
  }
  ElemPlan ep;
  rc = prepare_elem(ctx, kSlotPressure, p, io, false, nullptr, ep);
  if (rc) return rc;
  ppm::launch_pressure_batch(ep.B, ep.size_blocks, ctx->stream);
  ctx->launches += 1;
  CK(cudaGetLastError());
  if (memory == PPM_B200_MEM_HOST) {
    CK(cudaMemcpyAsync(pressure, io[0].pres, (size_t)grid_size(g) * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->stream));
    if (p->eos_type > 0) {  // the total energy was reset with the pressure
      rc = stage_out(ctx, p, g, io[0].user);
      if (rc) return rc;
    }
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return PPM_B200_OK;
}

static int timestep_batch(ppm_b200_context* ctx, const ppm_b200_params* p,
                          std::vector<GridIO>& io, double courant, double aye,
                          const double vgrid_in[3], double* dt_device, double* dt_host) {
  if (p->eos_type != 0 && p->eos_type != 3) return PPM_B200_ERR_UNSUPPORTED;
  for (auto& x : io)
    for (int d = 0; d < x.g->rank; ++d)
      if (!x.g->cell_width[d]) return PPM_B200_ERR_INVALID;
  ElemPlan ep;
  int rc = prepare_elem(ctx, kSlotTimestep, p, io, true, nullptr, ep);
  if (rc) return rc;
  const double zero3[3] = {0.0, 0.0, 0.0};
  const double* vg = vgrid_in ? vgrid_in : zero3;
  ep.B.aye = aye;
  for (int d = 0; d < 3; ++d) ep.B.vg[d] = vg[d];
  double* dt_slot = dt_device ? dt_device : ((double*)ctx->misc.p) + 1;
  ppm::launch_timestep_batch(ep.B, ep.active_blocks, courant, dt_slot, ctx->stream);
  ctx->launches += 2;
  CK(cudaGetLastError());
  if (dt_host) {
    CK(cudaMemcpyAsync(dt_host, dt_slot, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return PPM_B200_OK;
}

int ppm_b200_compute_timestep(ppm_b200_context* ctx, const ppm_b200_params* p, ppm_b200_grid* g,
                              int memory, double courant, double aye, const double vgrid_in[3],
                              double* dt_device, double* dt_host) {
  if (!ctx || !p || !g) return PPM_B200_ERR_INVALID;
  // this call does not read the acceleration: a gravity run's grids need none here
  ppm_b200_params q = *p;
  q.gravity = 0;
  p = &q;
  int rc = check_grid(g, p);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  std::vector<GridIO> io(1);
  io[0].g = g;
  rc = stage_in(ctx, p, g, memory, io[0].user, io[0].acc);
  if (rc) return rc;
  return timestep_batch(ctx, p, io, courant, aye, vgrid_in, dt_device, dt_host);
}

int ppm_b200_compute_timestep_level(ppm_b200_context* ctx, const ppm_b200_params* p,
                                    ppm_b200_grid* grids, int ngrids, double courant, double aye,
                                    const double vgrid[3], double* dt_device, double* dt_host) {
  if (!ctx || !p || !grids || ngrids <= 0) return PPM_B200_ERR_INVALID;
  // this call does not read the acceleration: a gravity run's grids need none here
  ppm_b200_params q = *p;
  q.gravity = 0;
  p = &q;
  CK(cudaSetDevice(ctx->device));
  std::vector<GridIO> io(ngrids);
  for (int k = 0; k < ngrids; ++k) {
    int rc = check_grid(&grids[k], p);
    if (rc) return rc;
    io[k].g = &grids[k];
    rc = stage_in(ctx, p, &grids[k], PPM_B200_MEM_DEVICE, io[k].user, io[k].acc);
    if (rc) return rc;
  }
  return timestep_batch(ctx, p, io, courant, aye, vgrid, dt_device, dt_host);
}

// Colour fields of a level as extra element records of six fields each, with their
// grid's geometry, so that the ghost-fill and zone-copy kernels treat them like the
// hydro fields.  Record order: the ng grids, then grid k's colour chunks at
// ng + k * colour_chunks(nc) + c.
int colour_chunks(int nc) { return (nc + 5) / 6; }

void append_colour_records(std::vector<GridIO>& io, int ng, int nc) {
  const int nch = colour_chunks(nc);
  for (int k = 0; k < ng; ++k)
    for (int c = 0; c < nch; ++c) {
      GridIO x{};
      x.g = io[k].g;
      for (int j = 0; j < 6; ++j) {
        const int n = 6 * c + j;
        x.user.f[j] = n < nc ? io[k].user.col[n] : nullptr;
      }
      io.push_back(x);
    }
}

// the fields a ghost fill or zone copy moves: hydro fields, and colours when nc > 0
int check_fill_grid(const ppm_b200_grid* g, int dual_energy, int nc) {
  if (!g->density || !g->total_energy || !g->velocity[0]) return PPM_B200_ERR_INVALID;
  for (int d = 1; d < g->rank; ++d)
    if (!g->velocity[d]) return PPM_B200_ERR_INVALID;
  if (dual_energy && !g->gas_energy) return PPM_B200_ERR_INVALID;
  if (nc < 0 || nc > PPM_B200_MAX_COLOURS) return PPM_B200_ERR_INVALID;
  if (nc > 0) {
    if (!g->colours) return PPM_B200_ERR_INVALID;
    for (int n = 0; n < nc; ++n)
      if (!g->colours[n]) return PPM_B200_ERR_INVALID;
  }
  return PPM_B200_OK;
}

static int boundary_batch(ppm_b200_context* ctx, ppm_b200_grid* grids, int ngrids,
                          int dual_energy, int ncolour, const int bc_type[3]) {
  if (!ctx || !grids || ngrids <= 0 || !bc_type) return PPM_B200_ERR_INVALID;
  for (int d = 0; d < 3; ++d)
    if (bc_type[d] < 0 || bc_type[d] > 2) return PPM_B200_ERR_INVALID;
  for (int k = 0; k < ngrids; ++k) {
    int rc = check_fill_grid(&grids[k], dual_energy, ncolour);
    if (rc) return rc;
  }
  CK(cudaSetDevice(ctx->device));
  ppm_b200_params p;
  std::memset(&p, 0, sizeof(p));
  p.dual_energy = dual_energy;
  p.number_of_colours = ncolour;
  std::vector<GridIO> io(ngrids);
  for (int k = 0; k < ngrids; ++k) {
    io[k].g = &grids[k];
    int rc = stage_in(ctx, &p, &grids[k], PPM_B200_MEM_DEVICE, io[k].user, io[k].acc, true);
    if (rc) return rc;
  }
  append_colour_records(io, ngrids, ncolour);
  p.dual_energy = 1;  // keep every record's sixth field (a grid's is null unless dual)
  ElemPlan ep;
  int rc = prepare_elem(ctx, kSlotBoundary, &p, io, false, bc_type, ep);
  if (rc) return rc;
  ppm::launch_boundary_batch(ep.B, ep.row_blocks, ctx->stream);
  ctx->launches += 1;
  CK(cudaGetLastError());
  return PPM_B200_OK;
}

// The boxes of Grid_CopyZonesFromGrid.C:100-160 over a level, from integer positions:
// grid a's whole region (ghosts included) against grid b's active region shifted by
// every periodic image (shift 0 of a itself excluded).
static void copy_boxes(const ppm_b200_grid* grids, int ngrids, const long long* left,
                       const long long domain[3], const int periodic[3],
                       std::vector<ppm::CopyBox>& boxes) {
  const int rank = grids[0].rank;
  int span[3];
  for (int d = 0; d < 3; ++d) span[d] = (d < rank && periodic[d]) ? 1 : 0;
  for (int a = 0; a < ngrids; ++a)
    for (int b = 0; b < ngrids; ++b)
      for (int sz = -span[2]; sz <= span[2]; ++sz)
        for (int sy = -span[1]; sy <= span[1]; ++sy)
          for (int sx = -span[0]; sx <= span[0]; ++sx) {
            const int sh[3] = {sx, sy, sz};
            if (a == b && sx == 0 && sy == 0 && sz == 0) continue;
            ppm::CopyBox x{};
            x.dst = a;
            x.src = b;
            bool empty = false;
            for (int d = 0; d < 3 && !empty; ++d) {
              if (d >= rank) {
                x.d0[d] = x.s0[d] = 0;
                x.ext[d] = 1;
                continue;
              }
              const long long off = (long long)sh[d] * domain[d];
              const long long la = left[3 * a + d], lb = left[3 * b + d];
              const long long lo = std::max(la, lb + grids[b].start[d] + off);
              const long long hi = std::min(la + grids[a].dims[d] - 1, lb + grids[b].end[d] + off);
              if (hi < lo) {
                empty = true;
                break;
              }
              x.d0[d] = (int)(lo - la);
              x.s0[d] = (int)(lo - off - lb);
              x.ext[d] = (int)(hi - lo + 1);
            }
            if (!empty) boxes.push_back(x);
          }
}

static int copy_zones_level(ppm_b200_context* ctx, ppm_b200_grid* grids, int ngrids,
                            const long long* left, const long long domain[3],
                            const int periodic[3], int dual_energy, int ncolour) {
  if (!ctx || ngrids < 0 || (ngrids > 0 && (!grids || !left)) || !domain || !periodic)
    return PPM_B200_ERR_INVALID;
  if (ngrids == 0) return PPM_B200_OK;
  const int rank = grids[0].rank;
  for (int k = 0; k < ngrids; ++k) {
    if (grids[k].rank != rank) return PPM_B200_ERR_INVALID;
    int rc = check_fill_grid(&grids[k], dual_energy, ncolour);
    if (rc) return rc;
  }
  for (int d = 0; d < rank; ++d)
    if (domain[d] <= 0) return PPM_B200_ERR_INVALID;
  std::vector<ppm::CopyBox> boxes;
  copy_boxes(grids, ngrids, left, domain, periodic, boxes);
  if (boxes.empty()) return PPM_B200_OK;
  CK(cudaSetDevice(ctx->device));
  ppm_b200_params p;
  std::memset(&p, 0, sizeof(p));
  p.dual_energy = dual_energy;
  p.number_of_colours = ncolour;
  std::vector<GridIO> io(ngrids);
  for (int k = 0; k < ngrids; ++k) {
    io[k].g = &grids[k];
    int rc = stage_in(ctx, &p, &grids[k], PPM_B200_MEM_DEVICE, io[k].user, io[k].acc, true);
    if (rc) return rc;
  }
  if (ncolour > 0) {  // every box again for each colour chunk of its two grids
    append_colour_records(io, ngrids, ncolour);
    const int nch = colour_chunks(ncolour);
    const size_t nb = boxes.size();
    for (int c = 0; c < nch; ++c)
      for (size_t b = 0; b < nb; ++b) {
        ppm::CopyBox x = boxes[b];
        x.dst = ngrids + x.dst * nch + c;
        x.src = ngrids + x.src * nch + c;
        boxes.push_back(x);
      }
  }
  p.dual_energy = 1;  // keep every record's sixth field (a grid's is null unless dual)
  ElemPlan ep;
  int rc = prepare_elem(ctx, kSlotCopy, &p, io, false, nullptr, ep);
  if (rc) return rc;
  std::vector<int64_t> pre(boxes.size() + 1, 0);
  for (size_t b = 0; b < boxes.size(); ++b) {
    const int64_t cells = (int64_t)boxes[b].ext[0] * boxes[b].ext[1] * boxes[b].ext[2];
    pre[b + 1] = pre[b] + (cells + 255) / 256;
  }
  std::vector<unsigned char> img;
  append(img, boxes.data(), boxes.size());
  const size_t off_p = align256(img.size());
  img.resize(off_p);
  append(img, pre.data(), pre.size());
  rc = mirror_put(ctx, ctx->mirror[kSlotCopyBoxes], img);
  if (rc) return rc;
  const unsigned char* base = (const unsigned char*)ctx->mirror[kSlotCopyBoxes].dev.p;
  ppm::launch_copy_zones(ep.B.grids, (const ppm::CopyBox*)base, (const int64_t*)(base + off_p),
                         (int)boxes.size(), pre.back(), ctx->stream);
  ctx->launches += 1;
  CK(cudaGetLastError());
  return PPM_B200_OK;
}

// grid::CorrectForRefinedFluxes for the proper subgrids of one grid (see the header):
// the phases and their index arithmetic on the host (Grid_CorrectForRefinedFluxes.C:
// 118-266), the flux arrays copied to the device, one kernel, the refined fluxes (which
// an undone correction resets to the initial ones) copied back.
// subling: the SUBling calls (initial = the grid's own boundary fluxes, the same for every
// refined entry), with the level's extent gdims and periodic faces (:147-221, :284-305)
static int correct_fluxes(ppm_b200_context* ctx, const ppm_b200_params* p, ppm_b200_grid* g,
                          int memory, int nsub, const ppm_b200_fluxes* initial,
                          ppm_b200_fluxes* refined, const long long gl[3], bool subling = false,
                          const long long* gdims = nullptr, const int* periodic = nullptr) {
  if (!ctx || !p || !g || nsub < 0 || (nsub > 0 && (!initial || !refined)) || !gl)
    return PPM_B200_ERR_INVALID;
  if (subling && (!gdims || !periodic)) return PPM_B200_ERR_INVALID;
  if (nsub == 0) return PPM_B200_OK;
  if (g->rank < 1 || g->rank > 3) return PPM_B200_ERR_INVALID;
  // species colours: the colours the caller marks as keeping their density fraction
  const bool species = p->number_of_colours > 0 && p->colour_species != nullptr;
  if (species) {
    if (p->number_of_colours > PPM_B200_MAX_COLOURS || !g->colours) return PPM_B200_ERR_INVALID;
    for (int n = 0; n < p->number_of_colours; ++n)
      if (!g->colours[n]) return PPM_B200_ERR_INVALID;
  }
  CK(cudaSetDevice(ctx->device));
  GridIO io;
  io.g = g;
  int rc = stage_in(ctx, p, g, memory, io.user, io.acc, species);
  if (rc) return rc;
  std::vector<double*> species_ptr;
  if (species)
    for (int n = 0; n < p->number_of_colours; ++n)
      if (p->colour_species[n]) species_ptr.push_back(io.user.col[n]);
  const int rank = g->rank;
  const int* GD = g->dims;
  // fields present: d, te, v1..v_rank, ge if dual (slots of ppm_b200_fluxes)
  bool present[6];
  for (int s = 0; s < 6; ++s) present[s] = io.user.f[s] != nullptr;
  struct HostPhase {
    ppm::FluxPhase ph;
    int n, dim;
    size_t icount, rcount;  // initial / refined flux values per array
  };
  std::vector<HostPhase> phases;
  for (int n = 0; n < nsub; ++n) {
    const ppm_b200_fluxes& I = subling ? initial[0] : initial[n];
    const ppm_b200_fluxes& R = refined[n];
    for (int dim = 0; dim < rank; ++dim) {
      if (GD[dim] <= 1) continue;
      ppm::FluxPhase ph{};
      ph.subling = subling ? 1 : 0;
      ph.correct_left = ph.correct_right = 1;
      long long rls[3], rle[3];
      int RefinedDim[3] = {0, 0, 0}, RefinedOffset[3] = {0, 0, 0}, InitialOffset[3] = {0, 0, 0};
      for (int i = 0; i < 3; ++i) {
        rls[i] = R.left_start[dim][i];
        rle[i] = R.left_end[dim][i];
      }
      if (subling) {
        const long long GlobalDim = gdims[dim];
        for (int i = 0; i < 3; ++i)
          RefinedDim[i] = (int)(R.left_end[dim][i] - R.left_start[dim][i] + 1);
        long long rrs = R.right_start[dim][dim];
        if (rls[dim] == 0 && periodic[dim]) {
          rls[dim] = rle[dim] = GlobalDim - 1;
        } else {
          rls[dim]--;
          rle[dim]--;
        }
        if (rrs == GlobalDim - 1 && periodic[dim]) rrs = 0; else rrs++;
        ph.correct_right = I.right_start[dim][dim] == rls[dim] ? 1 : 0;
        ph.correct_left = I.left_start[dim][dim] == rrs ? 1 : 0;
        for (int i = 0; i < 3; ++i)
          RefinedOffset[i] = (int)std::max<long long>(I.left_start[dim][i] - rls[i], 0);
        rls[dim] = 0;
        RefinedOffset[dim] = 0;
      }
      if (!ph.correct_left && !ph.correct_right) continue;
      int Start[3] = {0, 0, 0}, End[3] = {0, 0, 0}, Dim[3];
      for (int i = 0; i < rank; ++i) {
        Start[i] = (int)(std::max(I.left_start[dim][i], rls[i]) - gl[i]);
        End[i] = (int)(std::min(I.left_end[dim][i], rle[i]) - gl[i]);
        if (Start[i] < 0 || End[i] > GD[i]) return PPM_B200_ERR_INVALID;
      }
      Start[dim] = std::max(Start[dim] - 1, 0);
      End[dim] = Start[dim];
      for (int i = 0; i < 3; ++i) Dim[i] = End[i] - Start[i] + 1;
      long long off = I.right_start[dim][dim] - I.left_start[dim][dim] + 2;
      off = std::min<long long>(off, GD[dim] - 1);
      if (subling) {
        off -= 2;
        Start[dim]++;
        End[dim]++;
        for (int i = 0; i < rank; ++i) {
          if (i != dim) {
            Dim[i] = g->end[i] - g->start[i] + 1;
            InitialOffset[i] = (int)std::max<long long>(rls[i] - I.left_start[dim][i], 0);
          } else {
            Dim[i] = 1;
            InitialOffset[i] = 0;
          }
        }
      }
      if (Start[dim] == g->start[dim] - 1) ph.correct_left = 0;
      if (Start[dim] + off == g->end[dim] + 1) ph.correct_right = 0;
      const long long off_dim = off;
      for (int i = 0; i < dim; ++i) off *= GD[i];
      ph.offset = off;
      for (int i = 0; i < 3; ++i) {
        ph.start[i] = Start[i];
        ph.dim[i] = End[i] - Start[i] + 1;
        ph.id[i] = Dim[i];
        ph.io[i] = InitialOffset[i];
        ph.rd[i] = subling ? RefinedDim[i] : Dim[i];
        ph.ro[i] = subling ? RefinedOffset[i] : 0;
      }
      // the layers' zones and flux indexes stay inside the grid and the flux arrays
      for (int i = 0; i < 3; ++i) {
        if (ph.start[i] < 0 || ph.start[i] + ph.dim[i] > GD[i]) return PPM_B200_ERR_INVALID;
        if (ph.io[i] + ph.dim[i] > ph.id[i] || (subling && ph.ro[i] + ph.dim[i] > ph.rd[i]))
          return PPM_B200_ERR_INVALID;
      }
      if (ph.start[dim] + off_dim >= GD[dim] || ph.start[dim] + off_dim < 0)
        return PPM_B200_ERR_INVALID;
      for (int s = 0; s < 6; ++s)
        if (present[s] && (!I.left[s][dim] || !I.right[s][dim] || !R.left[s][dim] ||
                           !R.right[s][dim]))
          return PPM_B200_ERR_INVALID;
      const size_t icount = (size_t)ph.id[0] * ph.id[1] * ph.id[2];
      const size_t rcount = (size_t)ph.rd[0] * ph.rd[1] * ph.rd[2];
      phases.push_back({ph, n, dim, icount, rcount});
    }
  }
  if (phases.empty()) {
    if (memory == PPM_B200_MEM_HOST) CK(cudaStreamSynchronize(ctx->stream));
    return PPM_B200_OK;
  }
  // flux arrays on the device: per phase and present field, il | rl | ir | rr
  size_t total = 0;
  for (const auto& h : phases)
    for (int s = 0; s < 6; ++s)
      if (present[s]) total += 2 * h.icount + 2 * h.rcount;
  rc = ensure(ctx, ctx->flux_fix, std::max<size_t>(total, 1) * sizeof(double) +
                                      phases.size() * sizeof(ppm::FluxPhase) + 256 +
                                      species_ptr.size() * sizeof(double*));
  if (rc) return rc;
  double* dev = (double*)ctx->flux_fix.p;
  size_t at = 0;
  for (auto& h : phases) {
    const ppm_b200_fluxes& I = subling ? initial[0] : initial[h.n];
    const ppm_b200_fluxes& R = refined[h.n];
    for (int s = 0; s < 6; ++s) {
      if (!present[s]) continue;
      const double* src[4] = {I.left[s][h.dim], R.left[s][h.dim], I.right[s][h.dim],
                              R.right[s][h.dim]};
      const size_t cnt[4] = {h.icount, h.rcount, h.icount, h.rcount};
      double* dst[4];
      for (int q = 0; q < 4; ++q) {
        dst[q] = dev + at;
        at += cnt[q];
        CK(cudaMemcpyAsync(dst[q], src[q], cnt[q] * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
      }
      h.ph.il[s] = dst[0];
      h.ph.rl[s] = dst[1];
      h.ph.ir[s] = dst[2];
      h.ph.rr[s] = dst[3];
    }
  }
  std::vector<ppm::FluxPhase> host_ph(phases.size());
  for (size_t q = 0; q < phases.size(); ++q) host_ph[q] = phases[q].ph;
  ppm::FluxPhase* dph = (ppm::FluxPhase*)(dev + at);
  if ((uintptr_t)dph % alignof(ppm::FluxPhase)) return PPM_B200_ERR_CUDA;
  CK(cudaMemcpyAsync(dph, host_ph.data(), host_ph.size() * sizeof(ppm::FluxPhase),
                     cudaMemcpyHostToDevice, ctx->stream));
  double** dsp = reinterpret_cast<double**>(dph + host_ph.size());
  if (!species_ptr.empty())
    CK(cudaMemcpyAsync(dsp, species_ptr.data(), species_ptr.size() * sizeof(double*),
                       cudaMemcpyHostToDevice, ctx->stream));
  ppm::FluxFix X{};
  X.species = dsp;
  X.nspecies = (int)species_ptr.size();
  for (int s = 0; s < 6; ++s) X.f[s] = io.user.f[s];
  for (int d = 0; d < 3; ++d) X.dims[d] = GD[d];
  X.rank = rank;
  X.dual = p->dual_energy ? 1 : 0;
  X.tiny_number = p->tiny_number;
  X.nphases = (int)phases.size();
  ppm::launch_correct_fluxes(X, dph, ctx->stream);
  ctx->launches += 1;
  CK(cudaGetLastError());
  // the refined fluxes back (an undone correction set them to the initial ones)
  for (const auto& h : phases) {
    ppm_b200_fluxes& R = refined[h.n];
    for (int s = 0; s < 6; ++s) {
      if (!present[s]) continue;
      CK(cudaMemcpyAsync(R.left[s][h.dim], h.ph.rl[s], h.rcount * sizeof(double),
                         cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaMemcpyAsync(R.right[s][h.dim], h.ph.rr[s], h.rcount * sizeof(double),
                         cudaMemcpyDeviceToHost, ctx->stream));
    }
  }
  if (memory == PPM_B200_MEM_HOST) {
    rc = stage_out(ctx, p, g, io.user);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return PPM_B200_OK;
}

// Old fields of a grid on the device: device pointers as given, or copies of host arrays.
static int stage_old(ppm_b200_context* ctx, const ppm_b200_params* p, const ppm_b200_grid* g,
                     const ppm_b200_grid* old, int memory, FieldSet& fs) {
  const double* src[6] = {old->density, old->total_energy, old->velocity[0],
                          g->rank > 1 ? old->velocity[1] : nullptr,
                          g->rank > 2 ? old->velocity[2] : nullptr,
                          p->dual_energy ? old->gas_energy : nullptr};
  if (!src[0] || !src[1] || !src[2] || (g->rank > 1 && !src[3]) || (g->rank > 2 && !src[4]) ||
      (p->dual_energy && !src[5]))
    return PPM_B200_ERR_INVALID;
  for (int d = 0; d < 3; ++d)
    if (old->dims[d] != g->dims[d]) return PPM_B200_ERR_INVALID;
  const size_t bytes = (size_t)grid_size(g) * sizeof(double);
  for (int k = 0; k < 6; ++k) {
    fs.f[k] = nullptr;
    if (!src[k]) continue;
    if (memory == PPM_B200_MEM_DEVICE) {
      fs.f[k] = const_cast<double*>(src[k]);
    } else {
      int rc = ensure(ctx, ctx->host_old[k], bytes);
      if (rc) return rc;
      CK(cudaMemcpyAsync(ctx->host_old[k].p, src[k], bytes, cudaMemcpyHostToDevice,
                         ctx->stream));
      fs.f[k] = (double*)ctx->host_old[k].p;
    }
  }
  return PPM_B200_OK;
}

// grid::ComovingExpansionTerms over a batch (see ppm_b200_expansion_terms).
static int expansion_batch(ppm_b200_context* ctx, const ppm_b200_params* p,
                           std::vector<GridIO>& io, const std::vector<FieldSet>* old,
                           double time, double old_time, double coefficient) {
  ElemPlan ep;
  int rc = prepare_elem(ctx, kSlotExpansion, p, io, false, nullptr, ep, old);
  if (rc) return rc;
  ep.B.expansion = coefficient;
  // Grid_ComovingExpansionTerms.C:84-89 and Grid_ComputePressure.C:51-58: the mid time
  // between OldTime and Time, as an interpolation weight of the current fields
  ep.B.interpolate = 0;
  if (old) {
    const double ptime = 0.5 * (time + old_time);
    if (ptime != time) {
      double coef = 1.0;
      if (time - old_time > 0) coef = (ptime - old_time) / (time - old_time);
      ep.B.coef_new = coef;
      ep.B.coef_old = 1 - coef;
      ep.B.interpolate = 1;
    }
  }
  ppm::launch_expansion_batch(ep.B, ep.size_blocks, ctx->stream);
  ctx->launches += 1;
  CK(cudaGetLastError());
  return PPM_B200_OK;
}

int ppm_b200_expansion_terms(ppm_b200_context* ctx, const ppm_b200_params* p, ppm_b200_grid* g,
                             const ppm_b200_grid* old, double time, double old_time,
                             double coefficient, int memory) {
  if (!ctx || !p || !g) return PPM_B200_ERR_INVALID;
  // this call does not read the acceleration: a gravity run's grids need none here
  ppm_b200_params q = *p;
  q.gravity = 0;
  p = &q;
  int rc = check_grid(g, p);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  std::vector<GridIO> io(1);
  io[0].g = g;
  rc = stage_in(ctx, p, g, memory, io[0].user, io[0].acc);
  if (rc) return rc;
  std::vector<FieldSet> ofs(1);
  if (old) {
    rc = stage_old(ctx, p, g, old, memory, ofs[0]);
    if (rc) return rc;
  }
  rc = expansion_batch(ctx, p, io, old ? &ofs : nullptr, time, old_time, coefficient);
  if (rc) return rc;
  if (memory == PPM_B200_MEM_HOST) {
    rc = stage_out(ctx, p, g, io[0].user);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return PPM_B200_OK;
}

int ppm_b200_expansion_terms_level(ppm_b200_context* ctx, const ppm_b200_params* p,
                                   ppm_b200_grid* grids, const ppm_b200_grid* olds,
                                   int ngrids, double time, double old_time,
                                   double coefficient) {
  if (!ctx || !p || !grids || ngrids <= 0) return PPM_B200_ERR_INVALID;
  // this call does not read the acceleration: a gravity run's grids need none here
  ppm_b200_params q = *p;
  q.gravity = 0;
  p = &q;
  CK(cudaSetDevice(ctx->device));
  std::vector<GridIO> io(ngrids);
  std::vector<FieldSet> ofs(ngrids);
  for (int k = 0; k < ngrids; ++k) {
    int rc = check_grid(&grids[k], p);
    if (rc) return rc;
    io[k].g = &grids[k];
    rc = stage_in(ctx, p, &grids[k], PPM_B200_MEM_DEVICE, io[k].user, io[k].acc);
    if (rc) return rc;
    if (olds) {
      rc = stage_old(ctx, p, &grids[k], &olds[k], PPM_B200_MEM_DEVICE, ofs[k]);
      if (rc) return rc;
    }
  }
  return expansion_batch(ctx, p, io, olds ? &ofs : nullptr, time, old_time, coefficient);
}

int ppm_b200_set_cfl(ppm_b200_context* ctx, double* dt_device, double courant, double aye,
                     const double vgrid[3]) {
  if (!ctx) return PPM_B200_ERR_INVALID;
  ctx->cfl_dt = dt_device;
  ctx->cfl_courant = courant;
  ctx->cfl_aye = aye;
  for (int d = 0; d < 3; ++d) ctx->cfl_vg[d] = vgrid ? vgrid[d] : 0.0;
  return PPM_B200_OK;
}

int ppm_b200_set_guess(ppm_b200_context* ctx, const float* weights) {
  if (!ctx) return PPM_B200_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  if (!weights) {
    ctx->has_guess = false;
    return PPM_B200_OK;
  }
  std::vector<uint32_t> packed;
  pack_guess(weights, packed);
  pack_guess_tc(weights, packed);
  int rc = ensure(ctx, ctx->guess, packed.size() * sizeof(uint32_t));
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));  // a queued solve may still read the old weights
  CK(cudaMemcpy(ctx->guess.p, packed.data(), packed.size() * sizeof(uint32_t),
                cudaMemcpyHostToDevice));
  ctx->has_guess = true;
  return PPM_B200_OK;
}

int ppm_b200_riemann_log(ppm_b200_context* ctx, double* records, long long capacity,
                         int stride) {
  if (!ctx || capacity < 0 || stride < 0) return PPM_B200_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  if (!records || capacity == 0 || stride == 0) {
    ctx->log = nullptr;
    ctx->log_cap = 0;
    ctx->log_stride = 0;
    return PPM_B200_OK;
  }
  int rc = ensure(ctx, ctx->log_count, sizeof(unsigned long long));
  if (rc) return rc;
  CK(cudaMemsetAsync(ctx->log_count.p, 0, sizeof(unsigned long long), ctx->stream));
  ctx->log = records;
  ctx->log_cap = capacity;
  ctx->log_stride = stride;
  return PPM_B200_OK;
}

int ppm_b200_riemann_log_count(ppm_b200_context* ctx, long long* count) {
  if (!ctx || !count) return PPM_B200_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  unsigned long long c = 0;
  if (ctx->log_count.p) {
    CK(cudaMemcpyAsync(&c, ctx->log_count.p, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  *count = (long long)std::min<unsigned long long>(c, (unsigned long long)ctx->log_cap);
  return PPM_B200_OK;
}

int ppm_b200_guess_features(ppm_b200_context* ctx, const double* records, long long n,
                            double gamma, double pmin, float* samples) {
  if (!ctx || n < 0 || (n > 0 && (!records || !samples))) return PPM_B200_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  CK(ppm::launch_guess_features(records, n, gamma, pmin, samples, ctx->stream));
  ctx->launches += 1;
  return PPM_B200_OK;
}

int ppm_b200_guess_grad(ppm_b200_context* ctx, const float* weights, const float* samples,
                        const long long* index, long long n, float* grad, double* loss) {
  if (!ctx || n < 0 || !weights || !grad || !loss || (n > 0 && !samples))
    return PPM_B200_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  if (n == 0) return PPM_B200_OK;
  CK(ppm::launch_guess_grad(weights, samples, (const int64_t*)index, n, 1.0f / (float)n, grad,
                            loss, ctx->sms, ctx->stream));
  ctx->launches += 1;
  return PPM_B200_OK;
}

int ppm_b200_guess_adam(ppm_b200_context* ctx, float* weights, float* grad, float* m, float* v,
                        int step, float lr, float beta1, float beta2, float eps) {
  if (!ctx || !weights || !grad || !m || !v || step < 1) return PPM_B200_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  CK(ppm::launch_guess_adam(weights, grad, m, v, step, lr, beta1, beta2, eps, ctx->stream));
  ctx->launches += 1;
  return PPM_B200_OK;
}

int ppm_b200_guess_eval(ppm_b200_context* ctx, const float* features, long long n, float* y) {
  if (!ctx || n < 0 || (n > 0 && (!features || !y))) return PPM_B200_ERR_INVALID;
  if (!ctx->has_guess) return PPM_B200_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  CK(ppm::launch_guess_eval_tc((const uint32_t*)ctx->guess.p, features, n, y,
                               (unsigned long long*)ctx->counters.p + ppm::kCntTimeout,
                               ctx->sms, ctx->stream));
  ctx->launches += 1;
  return PPM_B200_OK;
}

int ppm_b200_set_boundary(ppm_b200_context* ctx, ppm_b200_grid* g, int dual_energy,
                          int number_of_colours, const int bc_type[3]) {
  return boundary_batch(ctx, g, 1, dual_energy, number_of_colours, bc_type);
}

int ppm_b200_set_boundary_level(ppm_b200_context* ctx, ppm_b200_grid* grids, int ngrids,
                                int dual_energy, int number_of_colours, const int bc_type[3]) {
  return boundary_batch(ctx, grids, ngrids, dual_energy, number_of_colours, bc_type);
}

int ppm_b200_copy_zones_level(ppm_b200_context* ctx, ppm_b200_grid* grids, int ngrids,
                              const long long* left, const long long domain[3],
                              const int periodic[3], int dual_energy, int number_of_colours) {
  return copy_zones_level(ctx, grids, ngrids, left, domain, periodic, dual_energy,
                          number_of_colours);
}

int ppm_b200_debug_tma_stall(ppm_b200_context* ctx, int extra_bytes) {
  if (!ctx || extra_bytes < 0 || extra_bytes > 4096 || extra_bytes % 16 != 0)
    return PPM_B200_ERR_INVALID;
  ctx->debug_tma_extra = (unsigned)extra_bytes;
  return PPM_B200_OK;
}

int ppm_b200_correct_fluxes(ppm_b200_context* ctx, const ppm_b200_params* params,
                            ppm_b200_grid* grid, int memory, int nsub,
                            const ppm_b200_fluxes* initial, ppm_b200_fluxes* refined,
                            const long long grid_global_start[3]) {
  return correct_fluxes(ctx, params, grid, memory, nsub, initial, refined, grid_global_start);
}

int ppm_b200_correct_fluxes_sublings(ppm_b200_context* ctx, const ppm_b200_params* params,
                                     ppm_b200_grid* grid, int memory, int nsib,
                                     const ppm_b200_fluxes* own, ppm_b200_fluxes* refined,
                                     const long long grid_global_start[3],
                                     const long long level_dims[3], const int periodic[3]) {
  return correct_fluxes(ctx, params, grid, memory, nsib, own, refined, grid_global_start, true,
                        level_dims, periodic);
}

}  // extern "C"
