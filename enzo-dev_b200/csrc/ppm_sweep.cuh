// ppm_sweep.cuh -- launch arguments shared by the sweep kernels and the host driver.
#pragma once

#include <cuda.h>  // CUtensorMap

#include <cstdint>
#include <vector>

namespace ppm {

// Per-cell coefficients along one sweep axis, precomputed by the host from the
// cell widths exactly as inteuler.F:140-158 computes them (same expressions, FP64).
struct Coef {
  double c1, c2, c3, c4, c5, c6, dx2i, dx;
};

// Subgrid-flux capture request for one pencil: flux of face `face` goes to
// `dst_offset` of capture slot `slot` (a contiguous range of the capture buffer).
struct FluxCapture {
  int64_t pencil;     // linear pencil id
  int32_t face;       // face index along the pencil (left face of cell `face`)
  int32_t pad;
  int64_t dst;        // base offset (in doubles) of this request in the capture buffer
};

enum { kMaxCounters = 32 };
// device counters (unsigned long long), see ppm_b200_stats
enum {
  kCntInterfaces = 0,
  kCntNewton = 1,
  kCntHist0 = 2,  // 2..9 : newton_hist[0..7]
  kCntFallbacks = 10,
  kCntFatal = 11,
  kCntGuessRejected = 12,
  kCntNonFinite = 13,
  kCntFlagged = 14,  // pencils handed to the fallback pass (index into BatchArgs::flagged)
  kCntTimeout = 15,  // bounded waits on asynchronous copies that gave up
  kCntWarpNewton = 16,  // sum over Riemann warps of the most Newton updates any lane took
  kCntWarps = 17,       // Riemann warps with at least one face
};

struct SweepArgs {
  // geometry: pencils are indexed p = t2 * n1 + t1; cell a of pencil (t1, t2)
  // sits at element t1 * s1 + t2 * s2 + a * sa of every field array.
  int n;                 // pencil length (GridDimension[dim])
  int is, ie;            // active range along the pencil, 0-based inclusive
  int n1, n2;            // pencils along the two transverse axes
  int64_t s1, s2, sa;    // element strides
  int64_t npencils;
  // fields: d, e, u(sweep velocity), v, w, ge -- input and output sets (distinct)
  const double* __restrict__ in_d;
  const double* __restrict__ in_e;
  const double* __restrict__ in_u;
  const double* __restrict__ in_v;   // may be null (rank < 3): read as 0, not written
  const double* __restrict__ in_w;
  const double* __restrict__ in_ge;  // may be null unless dual
  const double* __restrict__ pres;   // pressure of this SolvePPM_DE call (stale across sweeps)
  const double* __restrict__ grav;   // acceleration along the sweep axis (GRAV only)
  double* __restrict__ out_d;
  double* __restrict__ out_e;
  double* __restrict__ out_u;
  double* __restrict__ out_v;
  double* __restrict__ out_w;
  double* __restrict__ out_ge;
  const Coef* __restrict__ coef;     // n entries
  // physics
  double gamma, dt, eta1, eta2, small_rho, pmin;
  const double* dt_device;           // if non-null, *dt_device replaces dt
  int fallback;                      // RiemannSolverFallback
  // subgrid flux capture (optional)
  const FluxCapture* captures;       // sorted by pencil
  int64_t ncaptures;
  double* capture_buf;               // 6 doubles per request: df, ef, uf, vf, wf, gef
  // face scratch of the three-stage sweep: plane v holds one value per (face, pencil),
  // element fi * npencils + pencil with fi = face - is in [0, ie - is + 1]
  double* fstate;                    // kFaceVars planes: dl dr pl pr ul ur vl vr wl wr gel ger
  double* fflux;                     // kFluxVars planes: df ef uf vf wf gef ub
  int64_t plane;                     // elements per plane = (ie - is + 2) * npencils
  // learned Newton start (ppm_guess.cuh): packed BF16 weights, used by the LEARNED kernels
  const uint32_t* guess;
  // optional log of sampled faces of the plain solver: 8 doubles per record
  // (dl dr pl pr ul ur p* +-iterations, negative when Newton did not converge)
  double* log;
  unsigned long long* log_count;     // records claimed (may exceed log_cap)
  int64_t log_cap;
  int log_stride;                    // about one face in log_stride is logged; 0 = off
  // Courant time step of the updated fields (calc_dt.F), computed in the update kernel of
  // a solve's last sweep when cfl_min_bits is set: the minimum over the batch of dt1
  // goes to *cfl_min_bits (positive doubles order as integers)
  unsigned long long* cfl_min_bits;
  const double* cw1;                 // cell widths along the t1 and t2 axes (device)
  const double* cw2;
  int dim, rank;                     // the sweep axis and GridRank
  int ts1, te1, ts2, te2;            // active ranges along the t1 and t2 axes
  double aye, vg[3], min_support;    // calc_dt's a, grid velocity, ComputePressure's floor
  // slope corrections: calcdiss's flattening (type 1 or 3) of every variable and
  // inteuler's steepening of the density, as per-cell coefficients of cells is-1 .. ie+1
  // in planes [cell - (is-1)][pencil], written by the corrections kernel; null when off
  double* flat;
  double* steep;
  int flatten, steepen;              // PPMFlatteningParameter, PPMSteepeningParameter
  // colour fields (NumberOfColours > 0): advected in place by the colour kernel after the
  // sweep's update.  col: device array of ncolour field pointers; fcol: kColVars face
  // planes that the density reconstruction and the Riemann stage leave for it; fhll: one
  // byte per face, set where the HLL fallback replaced the face's fluxes;
  // col_capture: ncolour doubles per subgrid-flux capture request (request r = dst / 6)
  int ncolour;
  double* const* col;
  double* fcol;
  unsigned char* fhll;
  double* col_capture;
  // Riemann solver (Grid_xEulerSweep.C:223-283): 0 two-shock, 1 HLL, 2 HLLC.  For HLL and
  // HLLC the flux plane XUB holds the gas-energy source ges of the face's right cell
  // instead of the Godunov velocity.
  int solver;
  // PressureFree: sound speed tiny in the characteristics (inteuler.F:199) and the time
  // step (calc_dt.F:78-137), the face densities the uncorrected ones (inteuler.F:556-561),
  // the two-shock solve replaced by p* = pmin, u* = (ul + ur)/2 (twoshock.F:124-130)
  int presfree;
  // EOSType 3 (isothermal): the folded time step's pressure is rho * eos_cs^2
  int eos_type;
  double eos_cs;
};

enum { kFaceVars = 12, kFluxVars = 7 };
// colour face planes: dla dl0 dra dr0 (the density's characteristic averages), the
// corrected densities before the dual-energy override, the override flags (1 left,
// 2 right), the Godunov density db, and on faces the HLL fallback replaced its weights
// sl, bm0, sr, bp0 (written by the fallback pass only there)
enum { CDLA = 0, CDL0, CDRA, CDR0, CDLC, CDRC, COVR, CDB, CHSL, CHBM, CHSR, CHBP, kColVars };
enum { kMaxColours = 45 };  // MAX_COLOR (fortran.def:2)

// Threads per block of the marching stages and of the face-parallel Riemann stage.
// (Riemann blocks of 128 faces leave fewer idle lanes at the end of each face plane of
// the small grids of a level than 256: -18 % Riemann time on a 600-patch level, and
// slightly faster on 256^3.)
#ifndef PPM_RIEMANN_THREADS
#define PPM_RIEMANN_THREADS 128
#endif
#ifndef PPM_MARCH_THREADS
#define PPM_MARCH_THREADS 128
#endif
enum { kMarchThreads = PPM_MARCH_THREADS, kRiemannThreads = PPM_RIEMANN_THREADS };

// One launch over a batch of grids (an AMR level, or a single grid).  Every block
// belongs to one grid: grid g owns blocks [prefix[g], prefix[g+1]) of a stage; a
// block finds its grid by binary search over the prefix table.
//   marching stages: ceil(npencils / kMarchThreads) blocks per grid
//   Riemann stage:   (ie - is + 2) * ceil(npencils / kRiemannThreads) blocks per grid
struct BatchArgs {
  SweepArgs one;                     // the record itself when ngrids == 1 (read from the
                                     // kernel parameter space, like a plain launch)
  const SweepArgs* grids;            // device array, ngrids records
  int ngrids;
  const int64_t* march_prefix;       // ngrids + 1
  const int64_t* riemann_prefix;     // ngrids + 1
  unsigned long long* counters;      // kMaxCounters, shared by the batch
  int64_t* flagged;                  // pencils needing the fallback pass: (grid << 40) | pencil
  int corrections = 0;               // the batch's grids carry flattening / steepening
  // x sweep of a single grid: the update kernel reads its input cells as TMA tiles of
  // kXTileRows pencils x kXTileCells cells, through 2-D tensor maps (cells x pencils) of
  // d, e, u, v, w, ge (absent fields: unused).  x_tma = 0: plain loads.
  int x_tma = 0;
  // test hook (ppm_b200_debug_tma_stall): bytes every TMA chunk expects beyond its
  // copies, so that its barrier never completes and the bounded waits run out; 0
  unsigned x_tma_extra_tx = 0;
  // colours: the batch's NumberOfColours (every grid the same) and the fallback-face
  // flags of all its grids (one region, cleared at the start of each sweep)
  int ncolour = 0;
  unsigned char* hll_flags = nullptr;
  int64_t hll_bytes = 0;
  int solver = 0;                    // the batch's Riemann solver (SweepArgs::solver)
  int presfree = 0;                  // PressureFree (SweepArgs::presfree)
  // two-shock Riemann stage (plain start, no colours): faces per block (64, 128 or 256;
  // the Riemann prefix table counts blocks of this size) and a persistent launch that
  // walks riemann_total blocks with a grid of the resident blocks
  int riemann_threads = kRiemannThreads;
  int persistent = 0;
  int64_t riemann_total = 0;
  // fused sweep (two-shock with the plain start, no colours or slope corrections): one
  // kernel reconstructs the interface states and solves the Riemann problems of a
  // (group of kFaceWarps pencils, segment of kFaceSeg faces) per block; face_prefix is
  // its block prefix table
  int fused = 0;
  const int64_t* face_prefix = nullptr;
  int64_t face_blocks = 0;
  // learned start from a tensor-core guess pass (tcgen05, ppm_guess_tc.cu) over the
  // interface states before the Riemann kernel, instead of inside it
  int learned_pass = 0;
  int sms = 148;
  CUtensorMap xin[6];
};

// The fused face kernel: a warp takes one pencil and kFaceSeg consecutive faces, lane
// l >= 1 the face of cell f0 - 1 + l (lane 0 the cell left of the first face); a block
// takes kFaceWarps consecutive pencils.
#ifndef PPM_FACE_WARPS
#define PPM_FACE_WARPS 8
#endif
enum { kFaceWarps = PPM_FACE_WARPS, kFaceThreads = 32 * PPM_FACE_WARPS, kFaceSeg = 31 };
__host__ __device__ inline int64_t face_segments(int is, int ie) {
  return (ie - is + 2 + kFaceSeg - 1) / kFaceSeg;
}
__host__ __device__ inline int64_t face_blocks(int64_t npencils, int is, int ie) {
  return ((npencils + kFaceWarps - 1) / kFaceWarps) * face_segments(is, ie);
}

// TMA tiles of the x sweep's update kernel: a warp's 32 pencils x 4 cells (32 bytes a
// pencil), double-buffered per warp
#ifndef PPM_X_BUFFERS
#define PPM_X_BUFFERS 2
#endif
#ifndef PPM_X_TILE_CELLS
#define PPM_X_TILE_CELLS 4
#endif
enum { kXTileRows = 32, kXTileCells = PPM_X_TILE_CELLS, kXBuffers = PPM_X_BUFFERS };

// inteuler.F:140-158 on the host (same expressions; 1-based i mapped to entry i-1): the
// coefficient table of one sweep axis.  Every entry point builds its table here, so the
// library's paths cannot drift apart; host code is compiled with -ffp-contract=off.
inline void build_coef(const double* dxi_in, int n, int is0, int ie0, std::vector<Coef>& out) {
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

// Grid that owns block b of a stage, and the block's index inside that grid.
__device__ __forceinline__ int batch_locate(const int64_t* prefix, int ngrids, int64_t b,
                                            int64_t& local) {
  int lo = 0, hi = ngrids - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= b) lo = mid; else hi = mid - 1;
  }
  local = b - prefix[lo];
  return lo;
}

}  // namespace ppm
