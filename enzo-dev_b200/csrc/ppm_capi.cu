// ppm_capi.cu -- the C ABI of include/ppm_b200.h: context, persistent device scratch,
// coefficient tables, and the grid::SolvePPM_DE driver (pressure once, then the three
// sweeps in the order rotated by CycleNumber % GridRank, Grid_SolvePPM_DE.C:53-146).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ppm_b200.h"
#include "ppm_sweep.cuh"

// launchers defined in ppm_kernels.cu
namespace ppm {
void launch_sweep_split(const SweepArgs& a, bool dual, bool grav, cudaStream_t st);
void launch_pressure_plain(const double* d, const double* te, const double* v1, const double* v2,
                           const double* v3, const double* ge, double* p, int64_t size,
                           double gamma, double tiny_number, double min_support, int sms,
                           cudaStream_t st);
void launch_timestep_plain(const double* d, const double* te, const double* const v[3],
                           const double* ge, int rank, const int dims[3], const int start[3],
                           const int end[3], double gamma, double tiny_number, double min_support,
                           double aye, const double vg[3], const double* const cw[3],
                           unsigned long long* min_bits, double courant, double* dt_out, int sms,
                           cudaStream_t st);
void launch_boundary_plain(double* const* f, int nf, const int dims[3], const int start[3],
                           const int end[3], const int bc[3], int sms, cudaStream_t st);
}  // namespace ppm

using ppm::Coef;
using ppm::FluxCapture;
using ppm::SweepArgs;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct ppm_b200_context {
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  long long launches = 0;
  int sticky_error = 0;
  // persistent device scratch, grown on demand
  DevBuf field_set[2][6];   // two ring sets of d, e, v1, v2, v3, ge
  DevBuf host_set[6];       // device copies of host-memory fields
  DevBuf host_acc[3];       // device copies of host-memory accelerations
  DevBuf pressure;
  DevBuf coef[3];
  std::vector<Coef> coef_host[3];
  DevBuf cw_dev[3];
  std::vector<double> cw_host[3];
  DevBuf counters;          // kMaxCounters unsigned long long
  DevBuf misc;              // [0] min_bits, [1] dt
  DevBuf captures;
  DevBuf capture_buf;
  std::vector<double> capture_host;
  DevBuf face_scratch;      // interface states and fluxes of the three-stage sweep
  // event timing of sweep launches
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
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

int ensure(ppm_b200_context* ctx, DevBuf& b, size_t bytes) {
  if (b.bytes >= bytes) return PPM_B200_OK;
  if (b.p) {
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaFree(b.p));
    b.p = nullptr;
    b.bytes = 0;
  }
  CK(cudaMalloc(&b.p, bytes));
  b.bytes = bytes;
  return PPM_B200_OK;
}

int64_t grid_size(const ppm_b200_grid* g) {
  return (int64_t)g->dims[0] * g->dims[1] * g->dims[2];
}

// inteuler.F:140-158 on the host, same expressions, 1-based i mapped to entry i-1.
void build_coef(const double* dxi_in, int n, int is0, int ie0, std::vector<Coef>& out) {
  out.assign(n, Coef{0, 0, 0, 0, 0, 0, 0, 0});
  auto dxi = [&](int i) { return dxi_in[i - 1]; };
  const int i1 = is0 + 1, i2 = ie0 + 1;
  for (int i = 1; i <= n; ++i) out[i - 1].dx = dxi(i);
  for (int i = i1 - 2; i <= i2 + 2; i++) {
    double qa = dxi(i) / (dxi(i - 1) + dxi(i) + dxi(i + 1));
    out[i - 1].c1 = qa * (2.0 * dxi(i - 1) + dxi(i)) / (dxi(i + 1) + dxi(i));
    out[i - 1].c2 = qa * (2.0 * dxi(i + 1) + dxi(i)) / (dxi(i - 1) + dxi(i));
  }
  for (int i = i1 - 1; i <= i2 + 2; i++) {
    double qa = dxi(i - 2) + dxi(i - 1) + dxi(i) + dxi(i + 1);
    double qb = dxi(i - 1) / (dxi(i - 1) + dxi(i));
    double qc = (dxi(i - 2) + dxi(i - 1)) / (2.0 * dxi(i - 1) + dxi(i));
    double qd = (dxi(i + 1) + dxi(i)) / (2.0 * dxi(i) + dxi(i - 1));
    qb = qb + 2.0 * dxi(i) * qb / qa * (qc - qd);
    out[i - 1].c3 = 1.0 - qb;
    out[i - 1].c4 = qb;
    out[i - 1].c5 = dxi(i) / qa * qd;
    out[i - 1].c6 = -(dxi(i - 1) / qa * qc);
    out[i - 1].dx2i = 0.5 / dxi(i);
  }
}

int upload_coef(ppm_b200_context* ctx, int dim, const ppm_b200_grid* g) {
  const int n = g->dims[dim];
  std::vector<Coef> c;
  build_coef(g->cell_width[dim], n, g->start[dim], g->end[dim], c);
  auto& cache = ctx->coef_host[dim];
  if (cache.size() == c.size() && std::memcmp(cache.data(), c.data(), c.size() * sizeof(Coef)) == 0)
    return PPM_B200_OK;
  int rc = ensure(ctx, ctx->coef[dim], c.size() * sizeof(Coef));
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));  // the previous table may still be in use
  CK(cudaMemcpy(ctx->coef[dim].p, c.data(), c.size() * sizeof(Coef), cudaMemcpyHostToDevice));
  cache = c;
  return PPM_B200_OK;
}

int upload_cw(ppm_b200_context* ctx, int dim, const ppm_b200_grid* g) {
  const int n = g->dims[dim];
  std::vector<double> c(g->cell_width[dim], g->cell_width[dim] + n);
  auto& cache = ctx->cw_host[dim];
  if (cache == c) return PPM_B200_OK;
  int rc = ensure(ctx, ctx->cw_dev[dim], n * sizeof(double));
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(ctx->cw_dev[dim].p, c.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  cache = c;
  return PPM_B200_OK;
}

int check_supported(const ppm_b200_params* p) {
  if (!p) return PPM_B200_ERR_INVALID;
  if (p->pressure_free || p->steepening || p->flattening || p->diffusion ||
      p->conservative_rec || p->positive_rec || p->eos_type != 0 || p->number_of_colours != 0)
    return PPM_B200_ERR_UNSUPPORTED;
  if (p->riemann_solver != PPM_B200_RIEMANN_TWOSHOCK) return PPM_B200_ERR_UNSUPPORTED;
  if (p->reconstruction != PPM_B200_RECONSTRUCTION_PPM) return PPM_B200_ERR_UNSUPPORTED;
  if (p->learned_guess) return PPM_B200_ERR_UNSUPPORTED;
  return PPM_B200_OK;
}

int check_grid(const ppm_b200_grid* g, const ppm_b200_params* p) {
  if (!g || g->rank < 1 || g->rank > 3) return PPM_B200_ERR_INVALID;
  if (!g->density || !g->total_energy || !g->velocity[0]) return PPM_B200_ERR_INVALID;
  if (p->dual_energy && !g->gas_energy) return PPM_B200_ERR_INVALID;
  for (int d = 0; d < 3; ++d) {
    if (d < g->rank) {
      if (g->end[d] - g->start[d] + 1 > 1) {
        // the sweep needs exactly three ghost zones on each side (NumberOfGhostZones = 3)
        if (g->start[d] != 3 || g->dims[d] - 1 - g->end[d] != 3) return PPM_B200_ERR_INVALID;
        if (!g->cell_width[d]) return PPM_B200_ERR_INVALID;
      }
      if (d > 0 && !g->velocity[d]) return PPM_B200_ERR_INVALID;
      if (p->gravity && !g->acceleration[d]) return PPM_B200_ERR_INVALID;
    } else if (g->dims[d] != 1) {
      return PPM_B200_ERR_INVALID;
    }
  }
  return PPM_B200_OK;
}

struct FieldSet {
  double* f[6];  // d, e, v1, v2, v3, ge
};

// One capture request on the host: where the 6 captured values of a request go.
struct HostCapture {
  int sub;     // subgrid
  int side;    // 0 left, 1 right
  int64_t offset;
};

int run_sweep(ppm_b200_context* ctx, int dim, const ppm_b200_params* p, const ppm_b200_grid* g,
              const FieldSet& in, const FieldSet& out, const double* pressure,
              const double* const acc[3], int nsub, ppm_b200_fluxes* sub, const long long ggs[3]) {
  int rc = upload_coef(ctx, dim, g);
  if (rc) return rc;
  const int GD0 = g->dims[0], GD1 = g->dims[1], GD2 = g->dims[2];
  SweepArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n = g->dims[dim];
  a.is = g->start[dim];
  a.ie = g->end[dim];
  int ax1, ax2;  // transverse axes: t1 (fast), t2
  if (dim == 0) {
    a.n1 = GD1; a.n2 = GD2; a.s1 = GD0; a.s2 = (int64_t)GD0 * GD1; a.sa = 1; ax1 = 1; ax2 = 2;
  } else if (dim == 1) {
    a.n1 = GD0; a.n2 = GD2; a.s1 = 1; a.s2 = (int64_t)GD0 * GD1; a.sa = GD0; ax1 = 0; ax2 = 2;
  } else {
    a.n1 = GD0; a.n2 = GD1; a.s1 = 1; a.s2 = GD0; a.sa = (int64_t)GD0 * GD1; ax1 = 0; ax2 = 1;
  }
  a.npencils = (int64_t)a.n1 * a.n2;
  const int vu = dim, vv = (dim + 1) % 3, vw = (dim + 2) % 3;
  auto vel_in = [&](int c) -> const double* { return c < g->rank ? in.f[2 + c] : nullptr; };
  auto vel_out = [&](int c) -> double* { return c < g->rank ? out.f[2 + c] : nullptr; };
  a.in_d = in.f[0];
  a.in_e = in.f[1];
  a.in_u = vel_in(vu);
  a.in_v = vel_in(vv);
  a.in_w = vel_in(vw);
  a.in_ge = p->dual_energy ? in.f[5] : nullptr;
  a.out_d = out.f[0];
  a.out_e = out.f[1];
  a.out_u = vel_out(vu);
  a.out_v = vel_out(vv);
  a.out_w = vel_out(vw);
  a.out_ge = p->dual_energy ? out.f[5] : nullptr;
  a.pres = pressure;
  a.grav = p->gravity ? acc[dim] : nullptr;
  a.coef = (const Coef*)ctx->coef[dim].p;
  a.gamma = p->gamma;
  a.dt = p->dt;
  a.dt_device = p->dt_device;
  a.eta1 = p->eta1;
  a.eta2 = p->eta2;
  a.small_rho = p->small_rho;
  a.pmin = p->tiny_number;
  a.fallback = p->riemann_fallback;
  a.counters = (unsigned long long*)ctx->counters.p;

  // subgrid flux capture requests (Grid_xEulerSweep.C:313-377 and y/z siblings)
  std::vector<FluxCapture> reqs;
  std::vector<HostCapture> hreq;
  if (nsub > 0 && sub) {
    for (int s = 0; s < nsub; ++s) {
      const ppm_b200_fluxes& fx = sub[s];
      // flux-plane axes as the reference names them: (idim, jdim)
      int ia = (dim == 0) ? 1 : 0;
      int ja = (dim == 2) ? 1 : 2;
      long long fi0 = fx.right_start[dim][ia] - ggs[ia];
      long long fi1 = fx.right_end[dim][ia] - ggs[ia];
      long long fj0 = fx.right_start[dim][ja] - ggs[ja];
      long long fj1 = fx.right_end[dim][ja] - ggs[ja];
      long long nfi = fi1 - fi0 + 1;
      long long lface = fx.left_start[dim][dim] - ggs[dim];
      long long rface = fx.right_start[dim][dim] - ggs[dim] + 1;
      if (lface < a.is || rface > a.ie + 1) return PPM_B200_ERR_INVALID;
      for (long long cj = fj0; cj <= fj1; ++cj)
        for (long long ci = fi0; ci <= fi1; ++ci) {
          long long c[3];
          c[ia] = ci;
          c[ja] = cj;
          int64_t t1 = c[ax1], t2 = c[ax2];
          if (t1 < 0 || t1 >= a.n1 || t2 < 0 || t2 >= a.n2) return PPM_B200_ERR_INVALID;
          int64_t pencil = t2 * a.n1 + t1;
          long long offset = (ci - fi0) + (cj - fj0) * nfi;
          for (int side = 0; side < 2; ++side) {
            FluxCapture r;
            r.pencil = pencil;
            r.face = (int)(side == 0 ? lface : rface);
            r.pad = (int)hreq.size();
            r.dst = 0;
            reqs.push_back(r);
            hreq.push_back(HostCapture{s, side, offset});
          }
        }
    }
    std::sort(reqs.begin(), reqs.end(), [](const FluxCapture& x, const FluxCapture& y) {
      return x.pencil != y.pencil ? x.pencil < y.pencil : x.face < y.face;
    });
    for (size_t k = 0; k < reqs.size(); ++k) reqs[k].dst = (int64_t)k * 6;
    rc = ensure(ctx, ctx->captures, reqs.size() * sizeof(FluxCapture));
    if (rc) return rc;
    rc = ensure(ctx, ctx->capture_buf, reqs.size() * 6 * sizeof(double));
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->captures.p, reqs.data(), reqs.size() * sizeof(FluxCapture),
                       cudaMemcpyHostToDevice, ctx->stream));
    a.captures = (const FluxCapture*)ctx->captures.p;
    a.ncaptures = (int64_t)reqs.size();
    a.capture_buf = (double*)ctx->capture_buf.p;
  }

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (ctx->profiling) {
    while (ctx->ev_pool.size() < ctx->ev_used + 2) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      ctx->ev_pool.push_back(e);
    }
    ev0 = ctx->ev_pool[ctx->ev_used++];
    ev1 = ctx->ev_pool[ctx->ev_used++];
    CK(cudaEventRecord(ev0, ctx->stream));
  }
  a.plane = (int64_t)(a.ie - a.is + 2) * a.npencils;
  const size_t planes = (size_t)(ppm::kFaceVars + ppm::kFluxVars) * (size_t)a.plane;
  const size_t need = planes * sizeof(double) + (size_t)a.npencils * sizeof(int64_t);
  rc = ensure(ctx, ctx->face_scratch, need);
  if (rc) return rc;
  a.fstate = (double*)ctx->face_scratch.p;
  a.fflux = a.fstate + (size_t)ppm::kFaceVars * (size_t)a.plane;
  a.flagged = (int64_t*)(a.fstate + planes);
  ppm::launch_sweep_split(a, p->dual_energy != 0, p->gravity != 0, ctx->stream);
  ctx->launches += 5;
  CK(cudaGetLastError());
  if (ev1) CK(cudaEventRecord(ev1, ctx->stream));

  if (!reqs.empty()) {
    ctx->capture_host.resize(reqs.size() * 6);
    CK(cudaMemcpyAsync(ctx->capture_host.data(), ctx->capture_buf.p,
                       reqs.size() * 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    // active extents for the transverse-velocity rule (nxz/nyz/nzz > 1)
    long long nact[3];
    for (int d = 0; d < 3; ++d) nact[d] = d < g->rank ? g->end[d] - g->start[d] + 1 : 1;
    // capture slot order: df, ef, uf, vf, wf, gef -> BaryonField slots
    const int slot_of_role[3] = {2 + vu, 2 + vv, 2 + vw};
    for (size_t k = 0; k < reqs.size(); ++k) {
      const HostCapture& h = hreq[reqs[k].pad];
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
    }
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
  }
  int s = PPM_B200_OK;
  if (c[ppm::kCntFatal]) s = PPM_B200_ERR_NEGATIVE;
  else if (c[ppm::kCntNonFinite]) s = PPM_B200_ERR_NONFINITE;
  if (status) *status = s;
  return PPM_B200_OK;
}

}  // namespace

extern "C" {

int ppm_b200_version(void) { return PPM_B200_VERSION; }

const char* ppm_b200_error_string(int code) {
  switch (code) {
    case PPM_B200_OK: return "ok";
    case PPM_B200_ERR_UNSUPPORTED: return "configuration not supported by ppm_b200";
    case PPM_B200_ERR_INVALID: return "invalid argument";
    case PPM_B200_ERR_CUDA: return "CUDA runtime error";
    case PPM_B200_ERR_NEGATIVE: return "negative density or energy the reference aborts on";
    case PPM_B200_ERR_NONFINITE: return "non-finite value in the output";
    case PPM_B200_ERR_TOO_LARGE: return "size exceeds the fixed limit of this entry point";
    default: return "unknown error";
  }
}

int ppm_b200_create(int device, void* cuda_stream, ppm_b200_context** out) {
  if (!out) return PPM_B200_ERR_INVALID;
  *out = nullptr;
  ppm_b200_context* ctx = new ppm_b200_context();
  ctx->device = device;
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
  auto fr = [](DevBuf& b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
  };
  for (auto& s : ctx->field_set)
    for (auto& b : s) fr(b);
  for (auto& b : ctx->host_set) fr(b);
  for (auto& b : ctx->host_acc) fr(b);
  fr(ctx->pressure);
  for (auto& b : ctx->coef) fr(b);
  for (auto& b : ctx->cw_dev) fr(b);
  fr(ctx->counters);
  fr(ctx->misc);
  fr(ctx->captures);
  fr(ctx->capture_buf);
  fr(ctx->face_scratch);
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
  for (size_t k = 0; k + 1 < ctx->ev_used; k += 2) {
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, ctx->ev_pool[k], ctx->ev_pool[k + 1]));
    total += ms;
  }
  if (sweep_ms) *sweep_ms = total;
  if (sweep_launches) *sweep_launches = (long long)(ctx->ev_used / 2);
  ctx->ev_used = 0;
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

// Resolve the device field set of a call: device pointers as given, or the context's
// device copies of host fields (copied in here).
static int stage_in(ppm_b200_context* ctx, const ppm_b200_params* p, ppm_b200_grid* g, int memory,
                    FieldSet& fs, const double* acc[3]) {
  double* src[6] = {g->density, g->total_energy, g->velocity[0],
                    g->rank > 1 ? g->velocity[1] : nullptr,
                    g->rank > 2 ? g->velocity[2] : nullptr,
                    p->dual_energy ? g->gas_energy : nullptr};
  const size_t bytes = (size_t)grid_size(g) * sizeof(double);
  for (int k = 0; k < 3; ++k) acc[k] = nullptr;
  if (memory == PPM_B200_MEM_DEVICE) {
    for (int k = 0; k < 6; ++k) fs.f[k] = src[k];
    for (int k = 0; k < g->rank; ++k) acc[k] = p->gravity ? g->acceleration[k] : nullptr;
    return PPM_B200_OK;
  }
  if (memory != PPM_B200_MEM_HOST) return PPM_B200_ERR_INVALID;
  for (int k = 0; k < 6; ++k) {
    fs.f[k] = nullptr;
    if (!src[k]) continue;
    int rc = ensure(ctx, ctx->host_set[k], bytes);
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->host_set[k].p, src[k], bytes, cudaMemcpyHostToDevice, ctx->stream));
    fs.f[k] = (double*)ctx->host_set[k].p;
  }
  if (p->gravity) {
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

static int stage_out(ppm_b200_context* ctx, const ppm_b200_params* p, ppm_b200_grid* g,
                     const FieldSet& fs) {
  double* dst[6] = {g->density, g->total_energy, g->velocity[0],
                    g->rank > 1 ? g->velocity[1] : nullptr,
                    g->rank > 2 ? g->velocity[2] : nullptr,
                    p->dual_energy ? g->gas_energy : nullptr};
  const size_t bytes = (size_t)grid_size(g) * sizeof(double);
  for (int k = 0; k < 6; ++k)
    if (dst[k] && fs.f[k])
      CK(cudaMemcpyAsync(dst[k], fs.f[k], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return PPM_B200_OK;
}

static int scratch_sets(ppm_b200_context* ctx, const ppm_b200_params* p, const ppm_b200_grid* g,
                        const FieldSet& user, FieldSet out[2]) {
  const size_t bytes = (size_t)grid_size(g) * sizeof(double);
  for (int s = 0; s < 2; ++s)
    for (int k = 0; k < 6; ++k) {
      out[s].f[k] = nullptr;
      if (!user.f[k]) continue;
      int rc = ensure(ctx, ctx->field_set[s][k], bytes);
      if (rc) return rc;
      out[s].f[k] = (double*)ctx->field_set[s][k].p;
    }
  return PPM_B200_OK;
}

static int pressure_into(ppm_b200_context* ctx, const ppm_b200_params* p, const ppm_b200_grid* g,
                         const FieldSet& fs, double* pres) {
  ppm::launch_pressure_plain(fs.f[0], fs.f[1], fs.f[2], g->rank > 1 ? fs.f[3] : nullptr,
                             g->rank > 2 ? fs.f[4] : nullptr, p->dual_energy ? fs.f[5] : nullptr,
                             pres, grid_size(g), p->gamma, p->tiny_number, p->min_support,
                             ctx->sms, ctx->stream);
  ctx->launches += 1;
  CK(cudaGetLastError());
  return PPM_B200_OK;
}

int ppm_b200_solve_ppm_de(ppm_b200_context* ctx, const ppm_b200_params* p, int cycle_number,
                          ppm_b200_grid* g, int memory, int nsub, ppm_b200_fluxes* sub,
                          const long long ggs_in[3], ppm_b200_stats* stats) {
  if (!ctx || !p || !g) return PPM_B200_ERR_INVALID;
  int rc = check_supported(p);
  if (rc) return rc;
  rc = check_grid(g, p);
  if (rc) return rc;
  if (nsub > 0 && !sub) return PPM_B200_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  const long long zero3[3] = {0, 0, 0};
  const long long* ggs = ggs_in ? ggs_in : zero3;

  FieldSet user;
  const double* acc[3];
  rc = stage_in(ctx, p, g, memory, user, acc);
  if (rc) return rc;
  FieldSet ring[2];
  rc = scratch_sets(ctx, p, g, user, ring);
  if (rc) return rc;
  rc = ensure(ctx, ctx->pressure, (size_t)grid_size(g) * sizeof(double));
  if (rc) return rc;
  double* pres = (double*)ctx->pressure.p;
  rc = pressure_into(ctx, p, g, user, pres);
  if (rc) return rc;

  // sweep order rotation, Grid_SolvePPM_DE.C:53 and :86-146
  const int rank = g->rank;
  const int nact[3] = {g->end[0] - g->start[0] + 1, rank > 1 ? g->end[1] - g->start[1] + 1 : 1,
                       rank > 2 ? g->end[2] - g->start[2] + 1 : 1};
  int order[3], nsweeps = 0;
  const int ixyz = cycle_number % rank;
  for (int n = ixyz; n < ixyz + rank; ++n) {
    const int dim = n % rank;
    if (nact[dim] > 1) order[nsweeps++] = dim;
  }
  // out-of-place ring: user -> S0 [-> S1] -> user; the last of two or three sweeps
  // writes the caller's arrays directly, a single sweep is copied back.
  const FieldSet* cur = &user;
  for (int s = 0; s < nsweeps; ++s) {
    const FieldSet* dst;
    if (s == nsweeps - 1 && nsweeps >= 2) dst = &user;
    else dst = &ring[s % 2];
    rc = run_sweep(ctx, order[s], p, g, *cur, *dst, pres, acc, nsub, sub, ggs);
    if (rc) return rc;
    cur = dst;
  }
  if (cur != &user) {
    const size_t bytes = (size_t)grid_size(g) * sizeof(double);
    for (int k = 0; k < 6; ++k)
      if (user.f[k])
        CK(cudaMemcpyAsync(user.f[k], cur->f[k], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  if (memory == PPM_B200_MEM_HOST) {
    rc = stage_out(ctx, p, g, user);
    if (rc) return rc;
  }
  if (memory == PPM_B200_MEM_HOST || stats || nsub > 0) {
    int status = PPM_B200_OK;
    rc = read_counters(ctx, stats, &status);
    if (rc) return rc;
    return status;
  }
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
  CK(cudaSetDevice(ctx->device));
  const long long zero3[3] = {0, 0, 0};
  const long long* ggs = ggs_in ? ggs_in : zero3;
  FieldSet user;
  const double* acc[3];
  rc = stage_in(ctx, p, g, memory, user, acc);
  if (rc) return rc;
  FieldSet ring[2];
  rc = scratch_sets(ctx, p, g, user, ring);
  if (rc) return rc;
  const double* pres = pressure;
  if (memory == PPM_B200_MEM_HOST) {
    rc = ensure(ctx, ctx->pressure, (size_t)grid_size(g) * sizeof(double));
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->pressure.p, pressure, (size_t)grid_size(g) * sizeof(double),
                       cudaMemcpyHostToDevice, ctx->stream));
    pres = (const double*)ctx->pressure.p;
  }
  rc = run_sweep(ctx, dim, p, g, user, ring[0], pres, acc, nsub, sub, ggs);
  if (rc) return rc;
  const size_t bytes = (size_t)grid_size(g) * sizeof(double);
  for (int k = 0; k < 6; ++k)
    if (user.f[k])
      CK(cudaMemcpyAsync(user.f[k], ring[0].f[k], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  if (memory == PPM_B200_MEM_HOST) {
    rc = stage_out(ctx, p, g, user);
    if (rc) return rc;
  }
  if (memory == PPM_B200_MEM_HOST || stats || nsub > 0) {
    int status = PPM_B200_OK;
    rc = read_counters(ctx, stats, &status);
    if (rc) return rc;
    return status;
  }
  return PPM_B200_OK;
}

int ppm_b200_compute_pressure(ppm_b200_context* ctx, const ppm_b200_params* p, ppm_b200_grid* g,
                              double* pressure, int memory) {
  if (!ctx || !p || !g || !pressure) return PPM_B200_ERR_INVALID;
  int rc = check_grid(g, p);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  FieldSet user;
  const double* acc[3];
  rc = stage_in(ctx, p, g, memory, user, acc);
  if (rc) return rc;
  double* out = pressure;
  if (memory == PPM_B200_MEM_HOST) {
    rc = ensure(ctx, ctx->pressure, (size_t)grid_size(g) * sizeof(double));
    if (rc) return rc;
    out = (double*)ctx->pressure.p;
  }
  rc = pressure_into(ctx, p, g, user, out);
  if (rc) return rc;
  if (memory == PPM_B200_MEM_HOST) {
    CK(cudaMemcpyAsync(pressure, out, (size_t)grid_size(g) * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return PPM_B200_OK;
}

int ppm_b200_compute_timestep(ppm_b200_context* ctx, const ppm_b200_params* p, ppm_b200_grid* g,
                              int memory, double courant, double aye, const double vgrid_in[3],
                              double* dt_device, double* dt_host) {
  if (!ctx || !p || !g) return PPM_B200_ERR_INVALID;
  int rc = check_grid(g, p);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  FieldSet user;
  const double* acc[3];
  rc = stage_in(ctx, p, g, memory, user, acc);
  if (rc) return rc;
  const double* cw[3] = {nullptr, nullptr, nullptr};
  for (int d = 0; d < g->rank; ++d) {
    if (!g->cell_width[d]) return PPM_B200_ERR_INVALID;
    rc = upload_cw(ctx, d, g);
    if (rc) return rc;
    cw[d] = (const double*)ctx->cw_dev[d].p;
  }
  const double zero3[3] = {0.0, 0.0, 0.0};
  const double* vg = vgrid_in ? vgrid_in : zero3;
  unsigned long long* min_bits = (unsigned long long*)ctx->misc.p;
  double* dt_slot = dt_device ? dt_device : ((double*)ctx->misc.p) + 1;
  const double* vel[3] = {user.f[2], g->rank > 1 ? user.f[3] : nullptr,
                          g->rank > 2 ? user.f[4] : nullptr};
  ppm::launch_timestep_plain(user.f[0], user.f[1], vel, p->dual_energy ? user.f[5] : nullptr,
                             g->rank, g->dims, g->start, g->end, p->gamma, p->tiny_number,
                             p->min_support, aye, vg, cw, min_bits, courant, dt_slot, ctx->sms,
                             ctx->stream);
  ctx->launches += 2;
  CK(cudaGetLastError());
  if (dt_host) {
    CK(cudaMemcpyAsync(dt_host, dt_slot, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return PPM_B200_OK;
}

int ppm_b200_set_boundary(ppm_b200_context* ctx, ppm_b200_grid* g, int dual_energy,
                          const int bc_type[3]) {
  if (!ctx || !g || !bc_type) return PPM_B200_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  double* f[6];
  int nf = 0;
  f[nf++] = g->density;
  f[nf++] = g->total_energy;
  for (int d = 0; d < g->rank; ++d) f[nf++] = g->velocity[d];
  if (dual_energy) f[nf++] = g->gas_energy;
  for (int k = 0; k < nf; ++k)
    if (!f[k]) return PPM_B200_ERR_INVALID;
  for (int d = 0; d < 3; ++d)
    if (bc_type[d] != 0 && bc_type[d] != 1) return PPM_B200_ERR_INVALID;
  ppm::launch_boundary_plain(f, nf, g->dims, g->start, g->end, bc_type, ctx->sms, ctx->stream);
  ctx->launches += 1;
  CK(cudaGetLastError());
  return PPM_B200_OK;
}

}  // extern "C"
