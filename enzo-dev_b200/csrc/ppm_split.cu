// ppm_split.cu -- one directional sweep as three sm_100a kernels sharing a face scratch.
//
//   reconstruct_kernel  (thread per pencil, marching, two roles)  inteuler + intvar: the
//                       12 corrected interface states of every face -> fstate
//   riemann_kernel      (thread per face)               twoshock + flux_twoshock -> fflux
//   update_kernel       (thread per pencil, marching)  flux_twoshock's negative-state check
//                       with the per-cell flux_hll fallback, euler, pgas2d_dual
//
// Splitting the chain at the interface states keeps each kernel's live state small.
// The Riemann stage -- a divergent Newton iteration with a serial chain of divides and
// square roots per face -- runs face-parallel at full occupancy instead of inside a
// register-heavy marching pipeline.  The two marching stages keep the reference's
// sequential semantics along a pencil: the fallback of cell i rewrites faces i and
// i+1 before cell i+1 is checked and before cell i-1 is updated, and pgas2d_dual
// reads its already-updated left neighbour.
// Scratch planes are laid out face-major with the pencil index fastest, so every
// warp's scratch accesses are contiguous.
#include <cuda_runtime.h>

#include <type_traits>

#include <atomic>

#include "ppm_device.cuh"
#include "ppm_guess.cuh"
#include "ppm_sweep.cuh"

namespace ppm {
void launch_guess_pass(const BatchArgs& B, int sms, cudaStream_t st);
namespace split {

enum { VD = 0, VP = 1, VU = 2, VV = 3, VW = 4, VGE = 5 };
enum { SDL = 0, SDR, SPL, SPR, SUL, SUR, SVL, SVR, SWL, SWR, SGEL, SGER };
enum { XDF = 0, XEF, XUF, XVF, XWF, XGEF, XUB };

__device__ __forceinline__ double ldg0(const double* __restrict__ p, int64_t off) {
  return p ? __ldg(p + off) : 0.0;
}

// Every thread of a block works on the same grid.  A batch of one grid (ONE) reads its
// record from the kernel parameters, where the compiler uses the fields as constant
// operands; a larger batch copies the block's record from the device array into shared
// memory once per block.  (Reading the record through a reference into global memory
// or as a by-value copy measured slower: the marching loops then hold the fields in
// registers and spill.)
__device__ __forceinline__ void load_record(SweepArgs& dst, const SweepArgs* src) {
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(&dst);
  for (int i = threadIdx.x; i < (int)(sizeof(SweepArgs) / 8); i += blockDim.x) d[i] = __ldg(s + i);
}

template <bool ONE>
__device__ __forceinline__ int locate(const int64_t* prefix, int ngrids, int64_t& lb) {
  if (ONE) {
    lb = blockIdx.x;
    return 0;
  }
  return batch_locate(prefix, ngrids, blockIdx.x, lb);
}

#define PPM_BIND_RECORD(name, g)           \
  __shared__ SweepArgs s_rec_;             \
  if (!ONE) {                              \
    load_record(s_rec_, B.grids + (g));    \
    __syncthreads();                       \
  }                                        \
  const SweepArgs& name = ONE ? B.one : s_rec_;

__device__ __forceinline__ Phys make_phys(const SweepArgs& a) {
  Phys P;
  P.gamma = a.gamma;
  P.dt = a.dt_device ? *a.dt_device : a.dt;
  P.eta1 = a.eta1;
  P.eta2 = a.eta2;
  P.small_rho = a.small_rho;
  P.pmin = a.pmin;
  P.qa = (a.gamma + 1.0) / (2.0 * a.gamma);
  P.gp1 = a.gamma + 1.0;
  P.gm1 = a.gamma - 1.0;
  return P;
}

// ------------------------------------------------------------------ stage 0 (optional)
// Slope-correction coefficients of every cell is-1 .. ie+1 of a pencil: calcdiss's
// flattening (calcdiss.F:213-224 with type 1 :407-438 or type 3 :486-564) from the
// sweep's pressure, velocity, density and total energy, and inteuler's density
// steepening (inteuler.F:166-193).  Thread per pencil, marching; the flattening's
// flattemp values are computed once each and kept for the max of eq. A2.
template <bool ONE>
__global__ void __launch_bounds__(kMarchThreads) corrections_kernel(const __grid_constant__ BatchArgs B) {
  int64_t lb;
  const int g = locate<ONE>(B.march_prefix, B.ngrids, lb);
  PPM_BIND_RECORD(a, g)
  const int64_t pid = lb * kMarchThreads + threadIdx.x;
  if (pid >= a.npencils) return;
  const int64_t base = (pid % a.n1) * a.s1 + (pid / a.n1) * a.s2;
  const int64_t sa = a.sa, np = a.npencils;
  const int is = a.is, ie = a.ie;
  const double gamma = a.gamma;
  auto ld = [&](const double* f, int i) { return __ldg(f + base + (int64_t)i * sa); };
  // flattemp of cell j, j clamped to is-1 .. ie+1 (calcdiss.F:427-428, 563-564)
  auto ftemp = [&](int j) {
    j = j < is - 1 ? is - 1 : (j > ie + 1 ? ie + 1 : j);
    double p[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) p[k] = ld(a.pres, j - 2 + k);
    const double wf = cd_wflag(p[1], p[3], ld(a.in_u, j - 1), ld(a.in_u, j + 1));
    if (a.flatten == 1) return cd_ftemp1(p, wf);
    double d[5], e[5], u[5];
    if (a.flatten == 2) {
#pragma unroll
      for (int k = 0; k < 5; ++k) d[k] = ld(a.in_d, j - 2 + k);
      return cd_ftemp2(d, p, wf, gamma);
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      d[k] = ld(a.in_d, j - 2 + k);
      e[k] = ld(a.in_e, j - 2 + k);
      u[k] = ld(a.in_u, j - 2 + k);
    }
    return cd_ftemp3(d, e, u, p, wf, gamma);
  };
  double fm = 0.0, f0 = 0.0;
  if (a.flatten) {
    fm = ftemp(is - 2);
    f0 = ftemp(is - 1);
  }
  for (int c = is - 1; c <= ie + 1; ++c) {
    const int64_t o = (int64_t)(c - (is - 1)) * np + pid;
    if (a.flatten) {  // eq. A2: the max with the neighbour on the high-pressure side
      const double fp = ftemp(c + 1);
      if (a.flatten == 2)  // eq. A6: the max over both neighbours (calcdiss.F:480-483)
        a.flat[o] = dmax_g(dmax_g(fm, f0), fp);
      else
        a.flat[o] = (ld(a.pres, c + 1) - ld(a.pres, c - 1) < 0.0) ? dmax(f0, fp) : dmax(f0, fm);
      fm = f0;
      f0 = fp;
    }
    if (a.steepen) {
      double d[5], dx[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        d[k] = ld(a.in_d, c - 2 + k);
        dx[k] = a.coef[c - 2 + k].dx;
      }
      a.steep[o] = steepen_coef(d, dx, ld(a.pres, c - 1), ld(a.pres, c + 1), gamma);
    }
  }
}

// ------------------------------------------------------------------ stage 1
// Two roles march the same pencil independently: ROLE 0 reconstructs density,
// pressure and normal velocity and applies inteuler's characteristic corrections,
// dual-energy override and floors; ROLE 1 reconstructs the transverse velocities and
// the gas energy and selects their upwind states.  Each writes its own six planes.
// Splitting the face this way halves the live state of a marching thread.
// Four resident blocks per SM keep a 256^3 sweep's pencils in a single wave.
#ifndef PPM_RECON_MINBLOCKS
#define PPM_RECON_MINBLOCKS (4 * 128 / PPM_MARCH_THREADS)
#endif

#ifndef PPM_RECON0_MINBLOCKS
#define PPM_RECON0_MINBLOCKS PPM_RECON_MINBLOCKS
#endif
// PPM_RECON_PREFETCH: a steady step of the march loads the next cell's values while it
// computes with this one (v/w/ge march 0.55 -> 0.48 ms per 256^3 sweep)
#ifndef PPM_RECON_PREFETCH
#define PPM_RECON_PREFETCH 1
#endif
// COR: the batch carries slope corrections (the coefficients of the corrections kernel).
// One pencil's march (the body of the reconstruct kernels).
template <bool DUAL, bool GRAV, int ROLE, bool COR>
__device__ __forceinline__ void reconstruct_pencil(const SweepArgs& a, int64_t pid) {
  constexpr int NV = (ROLE == 0) ? 3 : (DUAL ? 3 : 2);
  const Phys P = make_phys(a);
  const int64_t base = (pid % a.n1) * a.s1 + (pid / a.n1) * a.s2;
  const int64_t sa = a.sa;
  const int is = a.is, ie = a.ie;
  const int64_t np = a.npencils, plane = a.plane;
  // the role's variables: ROLE 0 (d, p, u), ROLE 1 (v, w, ge)
  const double* q0p = ROLE == 0 ? a.in_d : a.in_v;
  const double* q1p = ROLE == 0 ? a.pres : a.in_w;
  const double* q2p = ROLE == 0 ? a.in_u : (DUAL ? a.in_ge : nullptr);

  double wq0[3], wq1[3], wq2[3];  // cells t-3, t-2, t-1
  double dqm1[3], qlm1[3];        // dq(t-2), ql(t-2)
  double dqm2 = 0.0;              // dq(t-3) of the density (COR, steepening)
#pragma unroll
  for (int v = 0; v < 3; ++v) wq0[v] = wq1[v] = wq2[v] = dqm1[v] = qlm1[v] = 0.0;
  double wu0 = 0.0, wu1 = 0.0, wu2 = 0.0;  // normal velocity of cells t-3, t-2, t-1
  double wg0 = 0.0, wg1 = 0.0, wg2 = 0.0;  // acceleration (ROLE 0, GRAV)
  Prep prA = {0, 0, 0, 0, 0}, prB = {0, 0, 0, 0, 0};  // cells t-2, t-1
  // ROLE 0: the left side of face t-2 (cell t-3's right edge), solved when that cell's
  // parabola was formed, with its raw density averages (colours, PressureFree)
  SideOut sLp = {0.0, 0.0, 0.0, 0.0, false};
  double lda = 0.0, ld0 = 0.0;
  AdvL aLp = {};   // left data of face t-2 (ROLE 1)

  const int tend = ie + 3;  // the last face, ie+1, is assembled at t = ie+3
  // the next cell's loads (PPM_RECON_PREFETCH)
  double xq[3] = {0.0, 0.0, 0.0}, xu = 0.0, xg = 0.0, xd = 0.0, xp = 0.0;
  auto fetch = [&](const int t) {
    const int64_t off = base + (int64_t)t * sa;
    xq[0] = ldg0(q0p, off);
    xq[1] = ldg0(q1p, off);
    xq[2] = ldg0(q2p, off);
    if (ROLE != 0) xu = ldg0(a.in_u, off);
    if (GRAV && ROLE == 0) xg = __ldg(a.grav + off);
    if (ROLE != 0) {
      xd = __ldg(a.in_d + off);
      xp = __ldg(a.pres + off);
    }
  };
  // One step of the march.  ST (steady): cells t-2 .. t all inside the range every stage
  // touches (t in [is+2, ie+1]), so the range tests drop out and the step is one block
  // of straight-line code the scheduler can interleave.
  auto step = [&](const int t, auto steady) {
    constexpr bool ST = decltype(steady)::value;
    constexpr bool PF = ST && PPM_RECON_PREFETCH;
    const int64_t off = base + (int64_t)t * sa;
    double nq[3];
    nq[0] = PF ? xq[0] : ldg0(q0p, off);
    nq[1] = PF ? xq[1] : ldg0(q1p, off);
    nq[2] = PF ? xq[2] : ldg0(q2p, off);
    const double nu = ROLE == 0 ? nq[2] : (PF ? xu : ldg0(a.in_u, off));
    const double ng = (GRAV && ROLE == 0) ? (PF ? xg : __ldg(a.grav + off)) : 0.0;
    const double pd = PF ? xd : 0.0, pp = PF ? xp : 0.0;
    if (PF) fetch(t + 1);  // t + 1 <= ie + 2: inside the pencil
    // characteristic distances of cell t (inteuler.F:197-208)
    Prep prC = prB;
    if (ST || (t >= is - 1 && t <= ie + 1)) {
      const double nd = ROLE == 0 ? nq[0] : (PF ? pd : __ldg(a.in_d + off));
      const double npr = ROLE == 0 ? nq[1] : (PF ? pp : __ldg(a.pres + off));
      prC = (COR && a.presfree) ? cell_prep<true>(nd, npr, nu, a.coef[t].dx2i, P)
                                : cell_prep(nd, npr, nu, a.coef[t].dx2i, P);
    }
    // slope and left edge of cell t-1 (intvar.F:82-102)
    double dqN[3], qlN[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) dqN[v] = qlN[v] = 0.0;
    {
      const int c = t - 1;
      if (ST || (c >= is - 2 && c <= ie + 2)) {
        const Coef cf = a.coef[c];
#pragma unroll
        for (int v = 0; v < NV; ++v) dqN[v] = pm_slope(wq1[v], wq2[v], nq[v], cf.c1, cf.c2);
        if (ST || c >= is - 1) {
#pragma unroll
          for (int v = 0; v < NV; ++v)
            qlN[v] = pm_edge(wq1[v], wq2[v], dqm1[v], dqN[v], cf.c3, cf.c4, cf.c5, cf.c6);
        }
      }
    }
    // parabola of cell t-2, its face contributions, and face t-2 (inteuler.F:304-551)
    SideOut sLn = sLp;
    double ldn = lda, ld0n = ld0;
    AdvL aLn = aLp;
    {
      const int c = t - 2;
      if (ST || (c >= is - 1 && c <= ie + 1)) {
        Para pa[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) pa[v] = Para{0.0, 0.0, 0.0, 0.0};
        if (COR) {
          const int64_t co = (int64_t)(c - (is - 1)) * np + pid;
          const bool fl_on = a.flatten != 0, st_on = ROLE == 0 && a.steepen != 0;
          const double fl = fl_on ? a.flat[co] : 0.0;
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            if (v == 0 && st_on) {
              const double st = a.steep[co];
              pa[v] = fl_on ? pm_parabola<true, true>(wq0[v], wq1[v], wq2[v], qlm1[v], qlN[v],
                                                      st, dqm2, dqN[v], fl)
                            : pm_parabola<true, false>(wq0[v], wq1[v], wq2[v], qlm1[v],
                                                       qlN[v], st, dqm2, dqN[v]);
            } else if (fl_on) {
              pa[v] = pm_parabola<false, true>(wq0[v], wq1[v], wq2[v], qlm1[v], qlN[v], 0.0,
                                               0.0, 0.0, fl);
            } else {
              pa[v] = pm_parabola(wq0[v], wq1[v], wq2[v], qlm1[v], qlN[v]);
            }
          }
        } else {
#pragma unroll
          for (int v = 0; v < NV; ++v) pa[v] = pm_parabola(wq0[v], wq1[v], wq2[v], qlm1[v], qlN[v]);
        }
        double* o = a.fstate + (int64_t)(c - is) * np + pid;
        if (ROLE == 0) {
          // cell c's left edge gives the right side of face c, its right edge the left
          // side of face c+1; each side is solved on its own (face_side), the left one
          // carried to the next step
          if (ST || c >= is) {
            const SideIn Rin{pm_C(pa[0], prA.char2), pm_B(pa[0], prA.c0),
                             pm_C(pa[1], prA.char2), pm_B(pa[1], prA.c0),
                             pm_B(pa[1], prA.cm),    pm_B(pa[1], prA.cp),
                             pm_C(pa[2], prA.char2), pm_B(pa[2], prA.c0),
                             pm_B(pa[2], prA.cm),    pm_B(pa[2], prA.cp),
                             prA.cm,                 prA.c0,
                             prA.cp};
            const SideOut r = face_side<DUAL, GRAV, false>(Rin, GRAV ? (wg0 + wg1) : 0.0, P);
            double dl = sLp.d, dr = r.d;
            if (COR && a.fcol) {  // colours: what their face states need (kColVars planes)
              double* oc = a.fcol + (int64_t)(c - is) * np + pid;
              oc[CDLA * plane] = lda;
              oc[CDL0 * plane] = ld0;
              oc[CDRA * plane] = Rin.da;
              oc[CDR0 * plane] = Rin.d0;
              oc[CDLC * plane] = sLp.dc;
              oc[CDRC * plane] = r.dc;
              oc[COVR * plane] = (sLp.ov ? 1.0 : 0.0) + (r.ov ? 2.0 : 0.0);
            }
            if (COR && a.presfree) {  // the uncorrected densities (inteuler.F:556-561)
              dl = lda;
              dr = Rin.da;
            }
            o[SDL * plane] = dl;
            o[SDR * plane] = dr;
            o[SPL * plane] = sLp.p;
            o[SPR * plane] = r.p;
            o[SUL * plane] = sLp.u;
            o[SUR * plane] = r.u;
          }
          if (ST || c <= ie) {
            const SideIn Lin{pm_A(pa[0], prA.char1), pm_A(pa[0], prA.c0),
                             pm_A(pa[1], prA.char1), pm_A(pa[1], prA.c0),
                             pm_A(pa[1], prA.cm),    pm_A(pa[1], prA.cp),
                             pm_A(pa[2], prA.char1), pm_A(pa[2], prA.c0),
                             pm_A(pa[2], prA.cm),    pm_A(pa[2], prA.cp),
                             prA.cm,                 prA.c0,
                             prA.cp};
            sLn = face_side<DUAL, GRAV, true>(Lin, GRAV ? (wg1 + wg2) : 0.0, P);
            ldn = Lin.da;
            ld0n = Lin.d0;
          }
        } else {
          if (ST || c >= is) {
            AdvR R;
            R.vra = pm_C(pa[0], prA.char2);
            R.vr0 = pm_B(pa[0], prA.c0);
            R.wra = pm_C(pa[1], prA.char2);
            R.wr0 = pm_B(pa[1], prA.c0);
            R.gera = DUAL ? pm_C(pa[2], prA.char2) : 0.0;
            R.ger0 = DUAL ? pm_B(pa[2], prA.c0) : 0.0;
            const AdvState s = face_advected(aLp, R, wu0, wu1);
            o[SVL * plane] = s.vl;
            o[SVR * plane] = s.vr;
            o[SWL * plane] = s.wl;
            o[SWR * plane] = s.wr;
            if (DUAL) {
              o[SGEL * plane] = s.gel;
              o[SGER * plane] = s.ger;
            }
          }
          if (ST || c <= ie) {
            aLn.vla = pm_A(pa[0], prA.char1);
            aLn.vl0 = pm_A(pa[0], prA.c0);
            aLn.wla = pm_A(pa[1], prA.char1);
            aLn.wl0 = pm_A(pa[1], prA.c0);
            aLn.gela = DUAL ? pm_A(pa[2], prA.char1) : 0.0;
            aLn.gel0 = DUAL ? pm_A(pa[2], prA.c0) : 0.0;
          }
        }
      }
    }
    if (COR) dqm2 = dqm1[0];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      wq0[v] = wq1[v];
      wq1[v] = wq2[v];
      wq2[v] = nq[v];
      dqm1[v] = dqN[v];
      qlm1[v] = qlN[v];
    }
    wu0 = wu1;
    wu1 = wu2;
    wu2 = nu;
    wg0 = wg1;
    wg1 = wg2;
    wg2 = ng;
    prA = prB;
    prB = prC;
    sLp = sLn;
    lda = ldn;
    ld0 = ld0n;
    aLp = aLn;
  };
  using Ramp = std::integral_constant<bool, false>;
  using Steady = std::integral_constant<bool, true>;
  const int t_steady0 = is + 2, t_steady1 = ie + 1;
#pragma unroll 1
  for (int t = 0; t < t_steady0 && t <= tend; ++t) step(t, Ramp{});
  if (PPM_RECON_PREFETCH && t_steady0 <= t_steady1) fetch(t_steady0);
#pragma unroll 1
  for (int t = t_steady0; t <= t_steady1; ++t) step(t, Steady{});
#pragma unroll 1
  for (int t = t_steady1 + 1 > t_steady0 ? t_steady1 + 1 : t_steady0; t <= tend; ++t)
    step(t, Ramp{});
}

// FLAG: only the pencils of the batch's flagged list (the fused sweep's fallback pass,
// which needs the interface states of those pencils): a fixed grid walks the list.
template <bool DUAL, bool GRAV, int ROLE, bool ONE, bool COR = false, bool FLAG = false>
__global__ void __launch_bounds__(kMarchThreads,
                                  ROLE == 0 ? PPM_RECON0_MINBLOCKS : PPM_RECON_MINBLOCKS)
    reconstruct_kernel(const __grid_constant__ BatchArgs B) {
  if (FLAG) {
    const unsigned long long nflag = *(volatile unsigned long long*)&B.counters[kCntFlagged];
    for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         k < nflag; k += (unsigned long long)gridDim.x * blockDim.x) {
      const int64_t code = B.flagged[k];
      const SweepArgs& a = ONE ? B.one : B.grids[(int)(code >> 40)];
      reconstruct_pencil<DUAL, GRAV, ROLE, COR>(a, code & ((int64_t(1) << 40) - 1));
    }
    return;
  }
  int64_t lb;
  const int g = locate<ONE>(B.march_prefix, B.ngrids, lb);
  PPM_BIND_RECORD(a, g)
  const int64_t pid = lb * kMarchThreads + threadIdx.x;
  if (pid >= a.npencils) return;
  reconstruct_pencil<DUAL, GRAV, ROLE, COR>(a, pid);
}

template <bool DUAL>
__device__ __forceinline__ FaceState load_face(const SweepArgs& a, int64_t idx) {
  const double* s = a.fstate + idx;
  const int64_t pl = a.plane;
  FaceState f;
  f.dl = s[SDL * pl];
  f.dr = s[SDR * pl];
  f.pl = s[SPL * pl];
  f.pr = s[SPR * pl];
  f.ul = s[SUL * pl];
  f.ur = s[SUR * pl];
  f.vl = s[SVL * pl];
  f.vr = s[SVR * pl];
  f.wl = s[SWL * pl];
  f.wr = s[SWR * pl];
  f.gel = DUAL ? s[SGEL * pl] : 0.0;
  f.ger = DUAL ? s[SGER * pl] : 0.0;
  return f;
}

// The advected states (v, w, ge) of a face, which only the flux needs: the Riemann
// kernel loads them after the Newton iteration, so they hold no registers during it.
template <bool DUAL>
__device__ __forceinline__ void load_face_advected(const SweepArgs& a, int64_t idx,
                                                   FaceState& f) {
  const double* s = a.fstate + idx;
  const int64_t pl = a.plane;
  f.vl = s[SVL * pl];
  f.vr = s[SVR * pl];
  f.wl = s[SWL * pl];
  f.wr = s[SWR * pl];
  f.gel = DUAL ? s[SGEL * pl] : 0.0;
  f.ger = DUAL ? s[SGER * pl] : 0.0;
}

// ------------------------------------------------------------------ stage 2
// per grid, blocks over (face plane fi = face - is) x (chunks of pencils)
// LEARNED: the Newton iteration starts from the MLP's pressure (ppm_guess.cuh) and falls
// back to the acoustic start, i.e. the plain solver, when it does not converge.
// Without LEARNED, a sample of the faces can be logged (states + converged p*) as
// training data for that net.
// 8 resident blocks of 128 faces per SM (64 registers, a few spilled): the Newton
// iteration's dependent FP64 chains want warps more than registers (256^3 sweep:
// 1.65 -> 1.53 ms against the unconstrained 80 registers; 7 blocks: 1.59 ms).  The
// learned start, with the net's fragments as well, gains the same way (3 blocks at 168
// registers: 3.94 ms; 8 blocks at 64: 2.71 ms).
#ifndef PPM_RIEMANN_MINBLOCKS
#define PPM_RIEMANN_MINBLOCKS (8 * 128 / PPM_RIEMANN_THREADS)
#endif
#ifndef PPM_RIEMANN_LEARNED_MINBLOCKS
#define PPM_RIEMANN_LEARNED_MINBLOCKS (8 * 128 / PPM_RIEMANN_THREADS)
#endif
// COL: also store the Godunov density of every face for the colour kernel.
// RT: threads (faces) per block; the batch's Riemann prefix table is built for it.
// PERSIST: a persistent launch -- a grid sized to the resident blocks walks the batch's
// block list (B.riemann_total entries) with a stride of the grid, keeping each grid's
// record in shared memory while consecutive blocks belong to it.  RT and PERSIST are the
// level autotuner's choices per size class (ppm_b200_autotune_level).
// PLANE (with LEARNED): the net's output and |x|^2 of each face come from the guess
// pass, in the face's slot of the XUB plane.
template <bool DUAL, bool ONE, bool LEARNED, bool COL = false, int RT = kRiemannThreads,
          bool PERSIST = false, bool PLANE = false>
__global__ void __launch_bounds__(RT, (LEARNED ? PPM_RIEMANN_LEARNED_MINBLOCKS
                                               : PPM_RIEMANN_MINBLOCKS) * kRiemannThreads / RT)
    riemann_kernel(const __grid_constant__ BatchArgs B) {
  __shared__ unsigned int s_hist[8];
  __shared__ unsigned int s_newton;
  __shared__ unsigned int s_rejected;
  __shared__ unsigned int s_wtrips, s_warps;
  __shared__ SweepArgs s_rec;
  if (threadIdx.x < 8) s_hist[threadIdx.x] = 0u;
  if (threadIdx.x == 0) {
    s_newton = 0u;
    s_rejected = 0u;
    s_wtrips = 0u;
    s_warps = 0u;
  }
  int cur = -1;
  for (int64_t blk = blockIdx.x; !PERSIST || blk < B.riemann_total; blk += gridDim.x) {
  int64_t lb = blk;
  const int g = ONE ? 0 : batch_locate(B.riemann_prefix, B.ngrids, blk, lb);
  if (!ONE && g != cur) {  // block-uniform: every thread takes this branch together
    __syncthreads();       // the previous grid's record is no longer read
    load_record(s_rec, B.grids + g);
    cur = g;
  }
  __syncthreads();
  const SweepArgs& a = ONE ? B.one : s_rec;
  const int64_t chunks = (a.npencils + RT - 1) / RT;
  const int fi = (int)(lb / chunks);
  const int64_t pid = (lb - (int64_t)fi * chunks) * RT + threadIdx.x;
  const bool valid = pid < a.npencils;
  const Phys P = make_phys(a);
  const int64_t idx = (int64_t)fi * a.npencils + pid;
  FaceState s = FaceState{1.0, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (valid) {  // d, p, u now; v, w, ge after the Newton iteration
    const double* f = a.fstate + idx;
    const int64_t pl = a.plane;
    s.dl = f[SDL * pl];
    s.dr = f[SDR * pl];
    s.pl = f[SPL * pl];
    s.pr = f[SPR * pl];
    s.ul = f[SUL * pl];
    s.ur = f[SUR * pl];
  }
  float y = 0.0f, d2 = 0.0f;
  if (LEARNED && PLANE) {
    if (valid) {
      const float2 v = *reinterpret_cast<const float2*>(a.fflux + XUB * a.plane + idx);
      y = v.x;
      d2 = v.y;
    }
  } else if (LEARNED) {
    float f[6];
    d2 = guess_features(s.dl, s.dr, s.pl, s.pr, s.ul, s.ur, P.gamma, f);
    if (!valid) d2 = 0.0f;
    // warp-collective (every lane takes part, with or without a face); a warp whose
    // jumps are all weak keeps the acoustic start, which is then within ~|x|^2 of p*
    if (__any_sync(0xffffffffu, d2 > kGuessMinJump)) y = guess_mlp_warp(a.guess, f);
  }
  unsigned trips = 0;  // Newton updates of this lane's face (both starts when rejected)
  if (valid) {
    const double cl = qsqrt(P.gamma * s.pl * s.dl);
    const double cr = qsqrt(P.gamma * s.pr * s.dr);
    const double ps = acoustic_guess(s, cl, cr, P);
    Riemann rs;
    unsigned spent = 0;
    if (LEARNED) {
      rs = twoshock_newton(s, cl, cr, guess_pressure(ps, y, d2, P.pmin), P);
      if (!rs.converged) {
        spent = (unsigned)rs.iters;
        rs = twoshock_newton(s, cl, cr, ps, P);
        atomicAdd(&s_rejected, 1u);
      }
    } else {
      rs = twoshock_newton(s, cl, cr, ps, P);
      if (a.log && a.log_stride > 0) {
        const unsigned long long h =
            ((unsigned long long)idx + 0x9E3779B97F4A7C15ull * (unsigned long long)(g + 1)) *
            0xD1B54A32D192ED03ull;
        if ((h >> 40) % (unsigned long long)a.log_stride == 0) {
          const unsigned long long slot = atomicAdd(a.log_count, 1ull);
          if (slot < (unsigned long long)a.log_cap) {
            double* r = a.log + slot * 8;
            r[0] = s.dl; r[1] = s.dr; r[2] = s.pl; r[3] = s.pr;
            r[4] = s.ul; r[5] = s.ur; r[6] = rs.pbar;
            r[7] = rs.converged ? (double)rs.iters : -(double)rs.iters;
          }
        }
      }
    }
    const double qc = qdiv(P.dt, a.coef[a.is + fi].dx);
    load_face_advected<DUAL>(a, idx, s);
    double db;
    const Flux F = flux_twoshock<DUAL>(s, rs.pbar, rs.ubar, qc, P, COL ? &db : nullptr);
    double* o = a.fflux + idx;
    const int64_t pl = a.plane;
    if (COL) a.fcol[CDB * pl + idx] = db;
    o[XDF * pl] = F.df;
    o[XEF * pl] = F.ef;
    o[XUF * pl] = F.uf;
    o[XVF * pl] = F.vf;
    o[XWF * pl] = F.wf;
    if (DUAL) o[XGEF * pl] = F.gef;
    o[XUB * pl] = F.ub;
    atomicAdd(&s_hist[rs.iters & 7], 1u);
    atomicAdd(&s_newton, (unsigned)rs.iters + spent);
    trips = (unsigned)rs.iters + spent;
  }
  {  // what the warp pays for its divergent Newton loop: the most updates of any lane
    const unsigned wmax = __reduce_max_sync(0xffffffffu, trips);
    const unsigned any = __ballot_sync(0xffffffffu, valid);
    if ((threadIdx.x & 31) == 0 && any) {
      atomicAdd(&s_wtrips, wmax);
      atomicAdd(&s_warps, 1u);
    }
  }
  if (!PERSIST) break;
  }
  __syncthreads();
  if (threadIdx.x < 8 && s_hist[threadIdx.x])
    atomicAdd(&B.counters[kCntHist0 + threadIdx.x], (unsigned long long)s_hist[threadIdx.x]);
  if (threadIdx.x == 8 && s_newton) {
    unsigned long long nif = 0;
    for (int h = 0; h < 8; ++h) nif += s_hist[h];
    atomicAdd(&B.counters[kCntInterfaces], nif);
    atomicAdd(&B.counters[kCntNewton], (unsigned long long)s_newton);
  }
  if (LEARNED && threadIdx.x == 9 && s_rejected)
    atomicAdd(&B.counters[kCntGuessRejected], (unsigned long long)s_rejected);
  if (threadIdx.x == 10 && s_warps) {
    atomicAdd(&B.counters[kCntWarpNewton], (unsigned long long)s_wtrips);
    atomicAdd(&B.counters[kCntWarps], (unsigned long long)s_warps);
  }
}

// ------------------------------------------------------------------ stages 1+2 fused
// The interface states and the two-shock solution of every face in one kernel (the plain
// path: two-shock solver, acoustic start, no colours or slope corrections), so the
// twelve state planes never leave the chip; only the seven flux planes are written.
// A warp takes one pencil and kFaceSeg consecutive faces f0 .. f0+30: lane l holds cell
// c = f0 - 1 + l, reconstructs its parabolas (the neighbours' cells, slopes and edges
// arrive by warp shuffles; lane 0 computes the slope left of its cell and lane 31 the
// slope and edge right of its cell itself) and the contributions of that cell to its two
// faces; lane l >= 1 then assembles face c from lane l-1's left-side data and its own,
// solves its Riemann problem and writes its fluxes.  Each cell's work is done once, plus
// one extra cell per 31 faces.  The per-point arithmetic is the split kernels', so the
// fluxes are the same bits.
#ifndef PPM_FACE_MINBLOCKS
#define PPM_FACE_MINBLOCKS 2
#endif

__device__ __forceinline__ double shfl_up1(double v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ double shfl_dn1(double v) { return __shfl_down_sync(0xffffffffu, v, 1); }

// Parabolas of one cell for three variables from the cell values of every lane's cell
// (q), the slope left of lane 0's cell and right of lane 31's cell, and the coefficients.
// Returns the parabolas; qm: the left neighbour's value (for the caller).
template <int NV>
__device__ __forceinline__ void face_parabolas(const double q[3], const double qm[3],
                                               const double qp[3], const double qmm[3],
                                               const double qpp[3], const Coef& cf,
                                               const Coef& cfm, const Coef& cfp, int lane,
                                               Para pa[3]) {
#pragma unroll
  for (int v = 0; v < 3; ++v) pa[v] = Para{0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double dq = pm_slope(qm[v], q[v], qp[v], cf.c1, cf.c2);
    double dqm = shfl_up1(dq);
    double dqp = shfl_dn1(dq);
    if (lane == 0) dqm = pm_slope(qmm[v], qm[v], q[v], cfm.c1, cfm.c2);
    if (lane == 31) dqp = pm_slope(q[v], qp[v], qpp[v], cfp.c1, cfp.c2);
    const double ql = pm_edge(qm[v], q[v], dqm, dq, cf.c3, cf.c4, cf.c5, cf.c6);
    double qr = shfl_dn1(ql);
    if (lane == 31) qr = pm_edge(q[v], qp[v], dq, dqp, cfp.c3, cfp.c4, cfp.c5, cfp.c6);
    pa[v] = pm_parabola(qm[v], q[v], qp[v], ql, qr);
  }
}

template <bool DUAL, bool GRAV, bool ONE>
__global__ void __launch_bounds__(kFaceThreads, PPM_FACE_MINBLOCKS)
    face_kernel(const __grid_constant__ BatchArgs B) {
  __shared__ unsigned int s_hist[8];
  __shared__ unsigned int s_newton, s_wtrips, s_warps;
  if (threadIdx.x < 8) s_hist[threadIdx.x] = 0u;
  if (threadIdx.x == 0) {
    s_newton = 0u;
    s_wtrips = 0u;
    s_warps = 0u;
  }
  int64_t lb;
  const int g = locate<ONE>(B.face_prefix, B.ngrids, lb);
  PPM_BIND_RECORD(a, g)
  if (ONE) __syncthreads();
  const int lane = threadIdx.x & 31;
  const int is = a.is, ie = a.ie, n = a.n;
  const int64_t nseg = face_segments(is, ie);
  const int64_t grp = lb / nseg;
  const int f0 = is + (int)(lb - grp * nseg) * kFaceSeg;
  const int64_t pid = grp * kFaceWarps + (threadIdx.x >> 5);
  const bool pencil_ok = pid < a.npencils;  // warp-uniform
  const Phys P = make_phys(a);
  const int64_t base = pencil_ok ? (pid % a.n1) * a.s1 + (pid / a.n1) * a.s2 : 0;
  const int c = f0 - 1 + lane;  // this lane's cell; lanes >= 1: also the face of that index
  // cells beyond the pencil (past the last face's neighbours) are clamped: their results
  // are never used
  auto cl = [&](int i) { return i < 0 ? 0 : (i > n - 1 ? n - 1 : i); };
  auto ld = [&](const double* f, int i) -> double {
    return (f && pencil_ok) ? __ldg(f + base + (int64_t)cl(i) * a.sa) : 0.0;
  };
  const Coef cf = a.coef[cl(c)];
  const Coef cfm = a.coef[cl(c - 1)];
  const Coef cfp = a.coef[cl(c + 1)];

  // ---- density, pressure, normal velocity: parabolas, characteristic corrections
  const double* vA[3] = {a.in_d, a.pres, a.in_u};
  double q[3], qm[3], qp[3], qmm[3], qpp[3];
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    q[v] = ld(vA[v], c);
    qm[v] = shfl_up1(q[v]);
    qp[v] = shfl_dn1(q[v]);
    qmm[v] = qpp[v] = 0.0;
    if (lane == 0) {
      qm[v] = ld(vA[v], c - 1);
      qmm[v] = ld(vA[v], c - 2);
    }
    if (lane == 31) {
      qp[v] = ld(vA[v], c + 1);
      qpp[v] = ld(vA[v], c + 2);
    }
  }
  const double u_c = q[2], u_m = qm[2];  // uslice(c), uslice(c-1) for the upwinding
  Para pa[3];
  face_parabolas<3>(q, qm, qp, qmm, qpp, cf, cfm, cfp, lane, pa);
  const Prep pr = cell_prep(q[0], q[1], q[2], cf.dx2i, P);
  // right-side data of face c, left-side data of face c+1 (inteuler.F:304-316)
  CoreR R;
  R.dra = pm_C(pa[0], pr.char2);
  R.dr0 = pm_B(pa[0], pr.c0);
  R.pra = pm_C(pa[1], pr.char2);
  R.pr0 = pm_B(pa[1], pr.c0);
  R.prm = pm_B(pa[1], pr.cm);
  R.prp = pm_B(pa[1], pr.cp);
  R.ura = pm_C(pa[2], pr.char2);
  R.ur0 = pm_B(pa[2], pr.c0);
  R.urm = pm_B(pa[2], pr.cm);
  R.urp = pm_B(pa[2], pr.cp);
  R.cm = pr.cm;
  R.c0 = pr.c0;
  R.cp = pr.cp;
  CoreL L;  // of this cell, then moved to the right neighbour lane
  L.dla = shfl_up1(pm_A(pa[0], pr.char1));
  L.dl0 = shfl_up1(pm_A(pa[0], pr.c0));
  L.pla = shfl_up1(pm_A(pa[1], pr.char1));
  L.pl0 = shfl_up1(pm_A(pa[1], pr.c0));
  L.plm = shfl_up1(pm_A(pa[1], pr.cm));
  L.plp = shfl_up1(pm_A(pa[1], pr.cp));
  L.ula = shfl_up1(pm_A(pa[2], pr.char1));
  L.ul0 = shfl_up1(pm_A(pa[2], pr.c0));
  L.ulm = shfl_up1(pm_A(pa[2], pr.cm));
  L.ulp = shfl_up1(pm_A(pa[2], pr.cp));
  L.cm = shfl_up1(pr.cm);
  L.c0 = shfl_up1(pr.c0);
  L.cp = shfl_up1(pr.cp);
  double gsum = 0.0;
  if (GRAV) {
    const double gc = ld(a.grav, c);
    gsum = shfl_up1(gc) + gc;  // grslice(c-1) + grslice(c)
  }
  const bool face_ok = pencil_ok && lane >= 1 && c <= ie + 1;
  const CoreState cs = face_core<DUAL, GRAV>(L, R, gsum, P);

  // ---- the two-shock solution (twoshock.F:156-254)
  FaceState st = FaceState{1.0, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (face_ok) {
    st.dl = cs.dl; st.dr = cs.dr; st.pl = cs.pl; st.pr = cs.pr; st.ul = cs.ul; st.ur = cs.ur;
  }
  Riemann rs = {0.0, 0.0, 0, true};
  const int64_t np = a.npencils, plane = a.plane;
  const int64_t idx = (int64_t)(c - is) * np + pid;
  unsigned trips = 0;
  if (face_ok) {
    const double clr = qsqrt(P.gamma * st.pl * st.dl);
    const double crr = qsqrt(P.gamma * st.pr * st.dr);
    rs = twoshock_newton(st, clr, crr, acoustic_guess(st, clr, crr, P), P);
    trips = (unsigned)rs.iters;
    if (a.log && a.log_stride > 0) {
      const unsigned long long h =
          ((unsigned long long)idx + 0x9E3779B97F4A7C15ull * (unsigned long long)(g + 1)) *
          0xD1B54A32D192ED03ull;
      if ((h >> 40) % (unsigned long long)a.log_stride == 0) {
        const unsigned long long slot = atomicAdd(a.log_count, 1ull);
        if (slot < (unsigned long long)a.log_cap) {
          double* r = a.log + slot * 8;
          r[0] = st.dl; r[1] = st.dr; r[2] = st.pl; r[3] = st.pr;
          r[4] = st.ul; r[5] = st.ur; r[6] = rs.pbar;
          r[7] = rs.converged ? (double)rs.iters : -(double)rs.iters;
        }
      }
    }
    atomicAdd(&s_hist[rs.iters & 7], 1u);
    atomicAdd(&s_newton, (unsigned)rs.iters);
  }
  {
    const unsigned wmax = __reduce_max_sync(0xffffffffu, trips);
    const unsigned any = __ballot_sync(0xffffffffu, face_ok);
    if (lane == 0 && any != 0u) {
      atomicAdd(&s_wtrips, wmax);
      atomicAdd(&s_warps, 1u);
    }
  }

  // ---- transverse velocities and gas energy: parabolas and upwinded states
  constexpr int NB = DUAL ? 3 : 2;
  const double* vB[3] = {a.in_v, a.in_w, DUAL ? a.in_ge : nullptr};
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    q[v] = ld(vB[v], c);
    qm[v] = shfl_up1(q[v]);
    qp[v] = shfl_dn1(q[v]);
    qmm[v] = qpp[v] = 0.0;
    if (lane == 0) {
      qm[v] = ld(vB[v], c - 1);
      qmm[v] = ld(vB[v], c - 2);
    }
    if (lane == 31) {
      qp[v] = ld(vB[v], c + 1);
      qpp[v] = ld(vB[v], c + 2);
    }
  }
  face_parabolas<NB>(q, qm, qp, qmm, qpp, cf, cfm, cfp, lane, pa);
  AdvR AR;
  AR.vra = pm_C(pa[0], pr.char2);
  AR.vr0 = pm_B(pa[0], pr.c0);
  AR.wra = pm_C(pa[1], pr.char2);
  AR.wr0 = pm_B(pa[1], pr.c0);
  AR.gera = DUAL ? pm_C(pa[2], pr.char2) : 0.0;
  AR.ger0 = DUAL ? pm_B(pa[2], pr.c0) : 0.0;
  AdvL AL;
  AL.vla = shfl_up1(pm_A(pa[0], pr.char1));
  AL.vl0 = shfl_up1(pm_A(pa[0], pr.c0));
  AL.wla = shfl_up1(pm_A(pa[1], pr.char1));
  AL.wl0 = shfl_up1(pm_A(pa[1], pr.c0));
  AL.gela = shfl_up1(DUAL ? pm_A(pa[2], pr.char1) : 0.0);
  AL.gel0 = shfl_up1(DUAL ? pm_A(pa[2], pr.c0) : 0.0);
  const AdvState as = face_advected(AL, AR, u_m, u_c);

  // ---- the Godunov flux (flux_twoshock.F:84-396)
  if (face_ok) {
    st.vl = as.vl; st.vr = as.vr; st.wl = as.wl; st.wr = as.wr;
    st.gel = DUAL ? as.gel : 0.0;
    st.ger = DUAL ? as.ger : 0.0;
    const double qc = qdiv(P.dt, cf.dx);
    const Flux F = flux_twoshock<DUAL>(st, rs.pbar, rs.ubar, qc, P);
    double* o = a.fflux + idx;
    o[XDF * plane] = F.df;
    o[XEF * plane] = F.ef;
    o[XUF * plane] = F.uf;
    o[XVF * plane] = F.vf;
    o[XWF * plane] = F.wf;
    if (DUAL) o[XGEF * plane] = F.gef;
    o[XUB * plane] = F.ub;
  }
  __syncthreads();
  if (threadIdx.x < 8 && s_hist[threadIdx.x])
    atomicAdd(&B.counters[kCntHist0 + threadIdx.x], (unsigned long long)s_hist[threadIdx.x]);
  if (threadIdx.x == 8 && s_newton) {
    unsigned long long nif = 0;
    for (int h = 0; h < 8; ++h) nif += s_hist[h];
    atomicAdd(&B.counters[kCntInterfaces], nif);
    atomicAdd(&B.counters[kCntNewton], (unsigned long long)s_newton);
  }
  if (threadIdx.x == 10 && s_warps) {
    atomicAdd(&B.counters[kCntWarpNewton], (unsigned long long)s_wtrips);
    atomicAdd(&B.counters[kCntWarps], (unsigned long long)s_warps);
  }
}

// PressureFree with the two-shock solver: no Riemann problem, p* = pmin, u* the mean of
// the face velocities, and the face pressures set to pmin before flux_twoshock
// (twoshock.F:124-130).  COL: the Godunov density for the colour kernel.
template <bool DUAL, bool ONE, bool COL>
__global__ void __launch_bounds__(kRiemannThreads) presfree_riemann_kernel(const __grid_constant__ BatchArgs B) {
  int64_t lb;
  const int g = locate<ONE>(B.riemann_prefix, B.ngrids, lb);
  PPM_BIND_RECORD(a, g)
  const int64_t chunks = (a.npencils + kRiemannThreads - 1) / kRiemannThreads;
  const int fi = (int)(lb / chunks);
  const int64_t pid = (lb - (int64_t)fi * chunks) * kRiemannThreads + threadIdx.x;
  if (pid >= a.npencils) return;
  const Phys P = make_phys(a);
  const int64_t pl = a.plane, idx = (int64_t)fi * a.npencils + pid;
  FaceState s = load_face<DUAL>(a, idx);
  const double pbar = P.pmin;
  const double ubar = 0.5 * (s.ul + s.ur);
  s.pl = P.pmin;
  s.pr = P.pmin;
  // the reference overwrites pls/prs in place: an HLL fallback reads these too
  a.fstate[SPL * pl + idx] = P.pmin;
  a.fstate[SPR * pl + idx] = P.pmin;
  const double qc = P.dt / a.coef[a.is + fi].dx;
  double db;
  const Flux F = flux_twoshock<DUAL>(s, pbar, ubar, qc, P, COL ? &db : nullptr);
  double* o = a.fflux + idx;
  o[XDF * pl] = F.df;
  o[XEF * pl] = F.ef;
  o[XUF * pl] = F.uf;
  o[XVF * pl] = F.vf;
  o[XWF * pl] = F.wf;
  if (DUAL) o[XGEF * pl] = F.gef;
  o[XUB * pl] = F.ub;
  if (COL) a.fcol[CDB * pl + idx] = db;
}

// RiemannSolver = HLL (flux_hll.F:6-415) or HLLC (flux_hllc.F:6-421) at every face, one
// thread per face: the fluxes times dt/dx, and in the XUB plane the gas-energy source of
// the face's right cell c, ges(c) = dt/dx * pcent(c) * (sl*gesl + sr*gesr of face c,
// minus those of face c+1, in the reference's order), which needs face c+1's weights:
// recomputed here from its states (bit-identical to its own thread's).  COL: the weights
// (sl, gesl, sr, gesr) of every face for the colour kernel.
template <bool DUAL, bool HLLC>
__device__ __forceinline__ HllFace hll_any(const FaceState& s, const Phys& P) {
  return HLLC ? hllc_face<DUAL>(s, P) : hll_face<DUAL>(s, P);
}

// 8 blocks of 128 threads per SM (64 registers): the Riemann stage 12 % faster than at the
// 6 blocks its 74 registers allowed (HLLC 0.95 -> 0.83 ms per 256^3 sweep)
#ifndef PPM_HLL_MINBLOCKS
#define PPM_HLL_MINBLOCKS (8 * 128 / PPM_RIEMANN_THREADS)
#endif
template <bool DUAL, bool ONE, bool HLLC, bool COL>
__global__ void __launch_bounds__(kRiemannThreads, PPM_HLL_MINBLOCKS)
    hll_riemann_kernel(const __grid_constant__ BatchArgs B) {
  int64_t lb;
  const int g = locate<ONE>(B.riemann_prefix, B.ngrids, lb);
  PPM_BIND_RECORD(a, g)
  const int64_t chunks = (a.npencils + kRiemannThreads - 1) / kRiemannThreads;
  const int fi = (int)(lb / chunks);
  const int64_t pid = (lb - (int64_t)fi * chunks) * kRiemannThreads + threadIdx.x;
  if (pid >= a.npencils) return;
  const Phys P = make_phys(a);
  const int64_t np = a.npencils, pl = a.plane;
  const int64_t idx = (int64_t)fi * np + pid;
  const int c = a.is + fi;  // the face's right cell
  const HllFace h = hll_any<DUAL, HLLC>(load_face<DUAL>(a, idx), P);
  const double qc = P.dt / a.coef[c].dx;
  double* o = a.fflux + idx;
  o[XDF * pl] = qc * h.df;
  o[XEF * pl] = qc * h.ef;
  o[XUF * pl] = qc * h.uf;
  o[XVF * pl] = qc * h.vf;
  o[XWF * pl] = qc * h.wf;
  if (DUAL) o[XGEF * pl] = P.dt / a.coef[c].dx * h.gef;
  double ges = 0.0;  // ges(ie+1) is not consumed
  if (DUAL && c <= a.ie) {
    const HllFace h1 = hll_any<DUAL, HLLC>(load_face<DUAL>(a, idx + np), P);
    const int64_t off = (pid % a.n1) * a.s1 + (pid / a.n1) * a.s2 + (int64_t)c * a.sa;
    const double pcent = dmax(P.gm1 * __ldg(a.in_ge + off) * __ldg(a.in_d + off), kTiny);
    ges = qc * pcent * (h.sl * h.gesl + h.sr * h.gesr - h1.sl * h1.gesl - h1.sr * h1.gesr);
  }
  o[XUB * pl] = ges;
  if (COL) {
    double* w = a.fcol + idx;
    w[CHSL * pl] = h.sl;
    w[CHBM * pl] = h.gesl;
    w[CHSR * pl] = h.sr;
    w[CHBP * pl] = h.gesr;
  }
}

// The flux planes are read once, with whole lines per warp: streaming loads (evicted
// first) keep them from displacing the cells the marching kernels reuse.
__device__ __forceinline__ Flux load_flux(const SweepArgs& a, int64_t idx) {
  const double* s = a.fflux + idx;
  const int64_t pl = a.plane;
  Flux f;
  f.df = __ldcs(s + XDF * pl);
  f.ef = __ldcs(s + XEF * pl);
  f.uf = __ldcs(s + XUF * pl);
  f.vf = __ldcs(s + XVF * pl);
  f.wf = __ldcs(s + XWF * pl);
  f.gef = __ldcs(s + XGEF * pl);
  f.ub = __ldcs(s + XUB * pl);
  return f;
}

// The x sweep's cells: each lane reads its pencil's line over 16 consecutive steps, so
// these lines are marked to be evicted last from L1.
__device__ __forceinline__ double ldg_keep(const double* p) {
  double v;
  asm volatile("ld.global.nc.L1::evict_last.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ldg_keep0(const double* p, int64_t off) {
  return p ? ldg_keep(p + off) : 0.0;
}

template <bool DUAL>
__device__ __forceinline__ Cell load_cell_keep(const SweepArgs& a, int64_t off) {
  Cell c;
  c.d = ldg_keep(a.in_d + off);
  c.e = ldg_keep(a.in_e + off);
  c.u = ldg_keep0(a.in_u, off);
  c.v = ldg_keep0(a.in_v, off);
  c.w = ldg_keep0(a.in_w, off);
  c.ge = DUAL ? ldg_keep(a.in_ge + off) : 0.0;
  return c;
}

template <bool DUAL>
__device__ __forceinline__ Cell load_cell(const SweepArgs& a, int64_t off) {
  Cell c;
  c.d = __ldg(a.in_d + off);
  c.e = __ldg(a.in_e + off);
  c.u = ldg0(a.in_u, off);
  c.v = ldg0(a.in_v, off);
  c.w = ldg0(a.in_w, off);
  c.ge = DUAL ? __ldg(a.in_ge + off) : 0.0;
  return c;
}

// Input pipeline of the y and z sweeps' update kernel.  A step of a pencil consumes one
// unit: cell s (6 fields) and, for is <= s <= ie, face s+1-is (7 flux planes).  Each
// thread copies its own units PD steps ahead with cp.async (8 bytes a lane, so a warp's
// 32 consecutive pencils fill whole sectors) into a private ring of PD+1 units in
// shared memory, laid out [slot][value][thread]; the bytes in flight do not occupy
// registers.  The ring has one slot more than the distance, so a slot is refilled one
// step after it was read.  No barrier is involved: every thread reads only what it
// copied itself, after its own cp.async.wait_group.
// Measured (y/z update at 256^3, 0.76 ms with the one-step register prefetch at 3
// blocks/SM): distance 1 at 4 blocks/SM (128 registers) 0.55 ms; distance 2 at 4
// blocks 0.60; distance 1 or 2 at 3 blocks 0.74 / 0.70; 5 blocks spill.  On the
// 600-patch level (many short pencils, records in shared memory) distance 2 at 3
// blocks is the fastest.  The x sweep's update measured slower through the ring (1.64
// -> 2.12 ms): its lanes read 32 different lines, which the evict-last loads keep in
// L1 better.
#ifndef PPM_UPDATE_PIPE_ONE
#define PPM_UPDATE_PIPE_ONE 1
#endif
#ifndef PPM_UPDATE_PIPE_BATCH
#define PPM_UPDATE_PIPE_BATCH 2
#endif
constexpr int kUnitVals = 6 + kFluxVars;
template <int PD>
__host__ __device__ constexpr int ring_doubles() {
  return PD > 0 ? (PD + 1) * kUnitVals * kMarchThreads : 0;
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ring: this thread's column of the block's ring (ring[v * kMarchThreads] is value v)
template <bool DUAL, int PD>
__device__ __forceinline__ void pipe_issue(const SweepArgs& a, double* ring, int64_t base,
                                           int64_t pid, int s) {
  if (s < a.n) {
    double* r = ring + (s % (PD + 1)) * (kUnitVals * kMarchThreads);
    const int64_t off = base + (int64_t)s * a.sa;
    cp_async8(r, a.in_d + off);
    cp_async8(r + kMarchThreads, a.in_e + off);
    if (a.in_u) cp_async8(r + 2 * kMarchThreads, a.in_u + off);
    if (a.in_v) cp_async8(r + 3 * kMarchThreads, a.in_v + off);
    if (a.in_w) cp_async8(r + 4 * kMarchThreads, a.in_w + off);
    if (DUAL) cp_async8(r + 5 * kMarchThreads, a.in_ge + off);
    if (s >= a.is && s <= a.ie) {
      const double* f = a.fflux + (int64_t)(s + 1 - a.is) * a.npencils + pid;
      const int64_t pl = a.plane;
      cp_async8(r + 6 * kMarchThreads, f + XDF * pl);
      cp_async8(r + 7 * kMarchThreads, f + XEF * pl);
      cp_async8(r + 8 * kMarchThreads, f + XUF * pl);
      cp_async8(r + 9 * kMarchThreads, f + XVF * pl);
      cp_async8(r + 10 * kMarchThreads, f + XWF * pl);
      cp_async8(r + 11 * kMarchThreads, f + XGEF * pl);
      cp_async8(r + 12 * kMarchThreads, f + XUB * pl);
    }
  }
  cp_async_commit();  // one group per unit, empty past the pencil's end
}

template <bool DUAL>
__device__ __forceinline__ Cell pipe_cell(const SweepArgs& a, const double* r) {
  Cell c;
  c.d = r[0];
  c.e = r[kMarchThreads];
  c.u = a.in_u ? r[2 * kMarchThreads] : 0.0;
  c.v = a.in_v ? r[3 * kMarchThreads] : 0.0;
  c.w = a.in_w ? r[4 * kMarchThreads] : 0.0;
  c.ge = DUAL ? r[5 * kMarchThreads] : 0.0;
  return c;
}

// ------------------------------------------------ TMA tiles of the x sweep's update
// The x sweep's pencils run along the contiguous axis: a warp's 32 pencils are 32 rows
// of every field.  Plain loads fetch one sector per lane per cell; instead lane 0 of
// each warp has the tensor-memory accelerator copy the warp's [32 pencils x 2 cells]
// tile of every input field into shared memory, two chunks ahead, completing on an
// mbarrier per buffer (no multicast; the tensor maps cover this GPU's own fields).
// Every lane waits on the chunk's barrier (bounded: after ~1 s the warp records a
// timeout, stops copying and drains what is in flight) and reads its own row.
#ifndef PPM_X_TMA
#define PPM_X_TMA 1
#endif
constexpr int kXTile = kXTileRows * kXTileCells;       // doubles per field and buffer
constexpr int kXWarp = kXBuffers * 6 * kXTile;         // doubles per warp
constexpr long long kXWaitCycles = 2000000000ll;       // ~1 s at the B200's clocks

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kXWaitCycles) return false;
  return true;
}
__device__ __forceinline__ void tma_load_2d(double* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

struct XTiles {
  double* buf;                  // this warp's kXBuffers x 6 tiles [field][pencil][cell]
  uint64_t* bar;                // this warp's kXBuffers mbarriers
  const CUtensorMap* map;       // the six tensor maps (kernel parameter space)
  unsigned long long* timeouts; // the batch's kCntTimeout counter
  unsigned fields;              // bit f: input field f present
  unsigned bytes;               // bytes of one chunk (all present fields)
  int row0;                     // the warp's first pencil
  int last;                     // last chunk issued, -1: none
  bool broken;                  // a wait gave up: no further copies
};

__device__ __forceinline__ void x_issue(XTiles& x, int q) {
  const int b = q % kXBuffers;
  if ((threadIdx.x & 31) == 0) {
    mbar_expect_tx(x.bar + b, x.bytes);
#pragma unroll
    for (int f = 0; f < 6; ++f)
      if (x.fields & (1u << f))
        tma_load_2d(x.buf + (b * 6 + f) * kXTile, x.map + f, q * kXTileCells, x.row0, x.bar + b);
  }
  x.last = q;
}

// warp-uniform: called by every lane at the first step of chunk q (t = q * kXTileCells)
__device__ __forceinline__ void x_chunk(XTiles& x, int q, int n) {
  __syncwarp();  // every lane has read chunk q-1, whose buffer the next copy reuses
  if (x.broken) return;
  const int next = q + kXBuffers - 1;
  if (next * kXTileCells < n) x_issue(x, next);
  const bool ok = mbar_wait_bounded(x.bar + q % kXBuffers, (unsigned)(q / kXBuffers) & 1u);
  if (__any_sync(0xffffffffu, !ok)) {
    x.broken = true;
    if ((threadIdx.x & 31) == 0) atomicAdd(x.timeouts, 1ull);
  }
}

// after a timeout: wait (bounded) for the last copy issued into every buffer
__device__ __forceinline__ void x_drain(XTiles& x) {
  if (!x.broken) return;
  for (int b = 0; b < kXBuffers; ++b) {
    int q = x.last - ((x.last - b) % kXBuffers + kXBuffers) % kXBuffers;
    if (q >= 0) mbar_wait_bounded(x.bar + b, (unsigned)(q / kXBuffers) & 1u);
  }
}

template <bool DUAL>
__device__ __forceinline__ Cell x_cell(const XTiles& x, const SweepArgs& a, int t) {
  const double* r = x.buf + ((t / kXTileCells) % kXBuffers) * (6 * kXTile) +
                    (threadIdx.x & 31) * kXTileCells + t % kXTileCells;
  Cell c;
  c.d = r[0];
  c.e = r[kXTile];
  c.u = a.in_u ? r[2 * kXTile] : 0.0;
  c.v = a.in_v ? r[3 * kXTile] : 0.0;
  c.w = a.in_w ? r[4 * kXTile] : 0.0;
  c.ge = DUAL ? r[5 * kXTile] : 0.0;
  return c;
}

__device__ __forceinline__ Flux pipe_flux(const double* r) {
  Flux f;
  f.df = r[6 * kMarchThreads];
  f.ef = r[7 * kMarchThreads];
  f.uf = r[8 * kMarchThreads];
  f.vf = r[9 * kMarchThreads];
  f.wf = r[10 * kMarchThreads];
  f.gef = r[11 * kMarchThreads];
  f.ub = r[12 * kMarchThreads];
  return f;
}

// flux_hll for cell c (flux_hll.F with i1 = i2 = c): replaces the fluxes of faces c and
// c+1 and returns ges(c); ges(c+1), which the single-cell call leaves to its unset
// locals at index c+2, is defined from the HLL state of face c+2 when that face exists.
template <bool DUAL>
__device__ __noinline__ void hll_fallback(const SweepArgs& a, int64_t pid, int64_t base, int c,
                                          const Cell& cell, const Phys& P, Flux& F0, Flux& F1,
                                          double& ges_c, double& ges_c1, bool& fatal) {
  const int is = a.is, ie = a.ie;
  const int64_t np = a.npencils;
  const FaceState s0 = load_face<DUAL>(a, (int64_t)(c - is) * np + pid);
  const FaceState s1 = load_face<DUAL>(a, (int64_t)(c + 1 - is) * np + pid);
  const HllFace h0 = hll_face<DUAL>(s0, P);
  const HllFace h1 = hll_face<DUAL>(s1, P);
  if (a.fcol) {  // the colour kernel's HLL weights of faces c and c+1 (flux_hll.F:236-262)
    const int64_t plane = a.plane;
    double* w0 = a.fcol + (int64_t)(c - is) * np + pid;
    double* w1 = w0 + np;
    w0[CHSL * plane] = h0.sl; w0[CHBM * plane] = h0.gesl;
    w0[CHSR * plane] = h0.sr; w0[CHBP * plane] = h0.gesr;
    w1[CHSL * plane] = h1.sl; w1[CHBM * plane] = h1.gesl;
    w1[CHSR * plane] = h1.sr; w1[CHBP * plane] = h1.gesr;
  }
  HllFace h2 = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (c + 2 <= ie + 1) h2 = hll_face<DUAL>(load_face<DUAL>(a, (int64_t)(c + 2 - is) * np + pid), P);
  const double qcc = P.dt / a.coef[c].dx;
  const double qc1 = P.dt / a.coef[c + 1].dx;
  if (DUAL) {
    const int64_t off1 = base + (int64_t)(c + 1) * a.sa;
    const double pc0 = dmax(P.gm1 * cell.ge * cell.d, kTiny);
    const double pc1 = dmax(P.gm1 * __ldg(a.in_ge + off1) * __ldg(a.in_d + off1), kTiny);
    ges_c = qcc * pc0 * (h0.sl * h0.gesl + h0.sr * h0.gesr - h1.sl * h1.gesl - h1.sr * h1.gesr);
    ges_c1 = qc1 * pc1 * (h1.sl * h1.gesl + h1.sr * h1.gesr - h2.sl * h2.gesl - h2.sr * h2.gesr);
  }
  F0.df = qcc * h0.df;
  F0.uf = qcc * h0.uf;
  F0.vf = qcc * h0.vf;
  F0.wf = qcc * h0.wf;
  F0.ef = qcc * h0.ef;
  F0.gef = DUAL ? P.dt / a.coef[c].dx * h0.gef : 0.0;
  F1.df = qc1 * h1.df;
  F1.uf = qc1 * h1.uf;
  F1.vf = qc1 * h1.vf;
  F1.wf = qc1 * h1.wf;
  F1.ef = qc1 * h1.ef;
  F1.gef = DUAL ? P.dt / a.coef[c + 1].dx * h1.gef : 0.0;
  if (cell.d + F0.df - F1.df <= 0.0) fatal = true;  // flux_hll.F:336-383
}

// ------------------------------------------------------------------ stage 3
// Marching order per step t: (1) check cell t (flux_twoshock.F:401-456) and apply its
// fallback, which may rewrite faces t and t+1; face t is then final; (2) conservative
// update of cell t-1 from faces t-1 and t (euler.F); (3) dual-energy select of cell
// t-2 (pgas2d_dual.F, which needs the post-euler state of t-1) and store.  This is
// the reference's order: all checks and fallbacks of a pencil precede its update, and
// a fallback of cell i changes the right face of cell i-1.
//
// FALLBACK = false is the hot pass: it stops at the first cell that fails its check
// and flags the pencil; FALLBACK = true re-runs flagged pencils with the per-cell HLL
// fallback.  Sweeps are out of place, so the re-run reads untouched inputs and
// rewrites every output (and subgrid-flux capture) of the pencil.
struct UpdateCounts {
  unsigned int fallbacks, fatal, nonfinite;
  double dtmin;  // smallest calc_dt dt1 of the pencil's active cells (cfl_min_bits set)
};

// calc_dt.F:136-153 for one updated cell (the cell of pencil position c), with the
// pressure of grid::ComputePressure at the new time (Grid_ComputePressure.C:96-164):
// the time step of the next cycle, computed where the final state is first known.
// Roles -> axes: the sweep velocity u is v[dim], v is v[dim+1], w is v[dim+2].
template <bool DUAL>
__device__ __forceinline__ double cell_dt1(const SweepArgs& a, const Cell& o, double dx_sweep,
                                           int64_t t1, int64_t t2, const Phys& P) {
  // axis x, y, z of the sweep's (u, v, w) and cell widths: (sweep, t1, t2) axes are
  // (x, y, z), (y, x, z) and (z, x, y) -- as selects, not a dynamically indexed array
  const int dim = a.dim;
  const double w1 = a.cw1 ? a.cw1[t1] : 1.0, w2 = a.cw2 ? a.cw2[t2] : 1.0;
  const double dx[3] = {dim == 0 ? dx_sweep : w1, dim == 1 ? dx_sweep : (dim == 0 ? w1 : w2),
                        dim == 2 ? dx_sweep : w2};
  const double vx = dim == 0 ? o.u : (dim == 1 ? o.w : o.v);
  const double vy = dim == 0 ? o.v : (dim == 1 ? o.u : o.w);
  const double vz = dim == 0 ? o.w : (dim == 1 ? o.v : o.u);
  const double velocity1 = vx;
  const double velocity2 = a.rank > 1 ? vy : 0.0;
  const double velocity3 = a.rank > 2 ? vz : 0.0;
  double gas_energy;
  if (DUAL) {
    gas_energy = o.ge;
  } else {
    gas_energy = o.e - 0.5 * (velocity1 * velocity1 + velocity2 * velocity2 +
                              velocity3 * velocity3);
  }
  double p = P.gm1 * o.d * gas_energy;
  if (p < P.pmin) p = P.pmin;
  const double min_pressure = a.min_support * P.gm1 * o.d * o.d;
  if (p < min_pressure) p = min_pressure;
  if (a.eos_type == 3) p = o.d * a.eos_cs * a.eos_cs;  // EOS.h type 3
  const double cs = a.presfree ? kTiny : dmax(sqrt(P.gamma * p / o.d), kTiny);
  if (a.rank == 1) return dx[0] * a.aye / (cs + fabs(velocity1 - a.vg[0]));
  if (a.rank == 2)
    return a.aye / ((cs + fabs(velocity1 - a.vg[0])) / dx[0] +
                    (cs + fabs(velocity2 - a.vg[1])) / dx[1]);
  return a.aye / ((cs + fabs(velocity1 - a.vg[0])) / dx[0] +
                  (cs + fabs(velocity2 - a.vg[1])) / dx[1] +
                  (cs + fabs(velocity3 - a.vg[2])) / dx[2]);
}

// Output staging of the x sweep.  Its pencils run along the contiguous axis, so a warp
// storing one cell per pencil writes 32 separate sectors; instead every thread stores
// its cells into shared memory, and every kStageCells cells each warp writes out its
// 32 pencils' cells with consecutive lanes on consecutive cells of a pencil (warp-local:
// no block barrier).  Layout per warp [field][cell][lane], the cell row padded
// (kStageLd) so that the flush reads hit distinct banks.
#ifndef PPM_X_STAGE_STORES
#define PPM_X_STAGE_STORES 1
#endif
#ifndef PPM_STAGE_LD
#define PPM_STAGE_LD (32 + 8)
#endif
#ifndef PPM_STAGE_CELLS
#define PPM_STAGE_CELLS 4
#endif
enum { kStageCells = PPM_STAGE_CELLS, kStageLd = PPM_STAGE_LD };
constexpr int kStageField = kStageCells * kStageLd;
constexpr int kStageWarp = 6 * kStageField;  // doubles per warp

// stage: this warp's buffer; pid0: the warp's first pencil
template <bool DUAL>
__device__ __forceinline__ void flush_stage(const SweepArgs& a, const double* stage,
                                            int64_t pid0, int c0, int ncells) {
  __syncwarp();  // every lane has staged its cells
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int r = 0; r < kStageCells; ++r) {
    const int q = lane + 32 * r;
    const int j = q % kStageCells, p = q / kStageCells;
    const int64_t pid = pid0 + p;
    if (j < ncells && pid < a.npencils) {
      const int64_t off = (pid % a.n1) * a.s1 + (pid / a.n1) * a.s2 + (c0 + j);  // sa == 1
      const double* sp = stage + j * kStageLd + p;
      a.out_d[off] = sp[0];
      a.out_e[off] = sp[kStageField];
      if (a.out_u) a.out_u[off] = sp[2 * kStageField];
      if (a.out_v) a.out_v[off] = sp[3 * kStageField];
      if (a.out_w) a.out_w[off] = sp[4 * kStageField];
      if (DUAL) a.out_ge[off] = sp[5 * kStageField];
    }
  }
  __syncwarp();  // the buffer may be refilled
}

//
// STAGED (x sweep, hot pass only): every lane of a warp runs the same steps, including
// lanes without a pencil (valid = false) and lanes whose pencil was flagged, since the
// warp flushes the staged outputs together; those lanes skip all loads and computation.  A flagged pencil's partial outputs are rewritten by the
// fallback pass.
//
// PD > 0 (y and z sweeps, hot pass): the inputs arrive through the cp.async ring at
// distance PD (ring: this thread's column of it) instead of a one-step register
// prefetch.
//
// XT (x sweep of a single grid, with STAGED): the input cells arrive as TMA tiles (xt).
template <bool DUAL, bool GRAV, bool FALLBACK, bool STAGED = false, int PD = 0, bool XT = false,
          bool RS = false>
__device__ __forceinline__ bool update_pencil(const SweepArgs& a, int64_t pid, const Phys& P,
                                              UpdateCounts& cnt, bool valid = true,
                                              double* stage = nullptr, int64_t pid0 = 0,
                                              double* ring = nullptr, XTiles* xt = nullptr) {
  bool live = valid, flagged = false;
  const int64_t base = live ? (pid % a.n1) * a.s1 + (pid / a.n1) * a.s2 : 0;
  const int64_t t1 = pid % a.n1, t2 = pid / a.n1;
  // the pencil's cells are active across the sweep (calc_dt covers active cells only)
  const bool cfl = a.cfl_min_bits && t1 >= a.ts1 && t1 <= a.te1 && t2 >= a.ts2 && t2 <= a.te2;
  double dtmin = 1.0e20;
  const int64_t sa = a.sa, np = a.npencils;
  const int n = a.n, is = a.is, ie = a.ie;

  int64_t cap = 0, cap_end = 0;
  if (a.ncaptures > 0) {
    int64_t lo = 0, hi = a.ncaptures;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (a.captures[mid].pencil < pid) lo = mid + 1; else hi = mid;
    }
    cap = cap_end = lo;
    while (cap_end < a.ncaptures && a.captures[cap_end].pencil == pid) ++cap_end;
  }

  Flux Fm = {0, 0, 0, 0, 0, 0, 0};  // final flux at face t-1
  Flux F0 = Fm;                     // flux at face t (face is while t <= is)
  if (live) F0 = load_flux(a, pid);
  Cell Cm = {0, 0, 0, 0, 0, 0};     // input state of cell t-1
  double ges_m = 0.0;               // final ges of cell t-1
  bool gov = false;                 // ges(t) was set by the fallback of cell t-1
  double govv = 0.0;
  Cell PEm = {0, 0, 0, 0, 0, 0};    // post-euler state of cell t-2
  double dep = 0.0;                 // post-pgas d*e of cell t-3
  unsigned int nonfin = 0;
  // one-step prefetch of cell t and face t+1
  Cell Cpf = Cm;
  Flux Fpf = F0;
  constexpr bool PIPE = PD > 0;
  if (live) {
    if (PIPE) {
#pragma unroll
      for (int u = 0; u < PD; ++u) pipe_issue<DUAL, PD>(a, ring, base, pid, u);
    } else {
      if (!XT) Cpf = STAGED ? load_cell_keep<DUAL>(a, base) : load_cell<DUAL>(a, base);
      if (0 >= is && 0 <= ie) Fpf = load_flux(a, (int64_t)(1 - is) * np + pid);
    }
  }
  if (XT) {  // warp-wide, live or not: the first chunks
    for (int q = 0; q < kXBuffers - 1 && q * kXTileCells < n; ++q) x_issue(*xt, q);
  }

  // One step of the march.  ST (steady): t in [is+2, ie-1], where cell t, face t+1 and
  // cells t-1, t-2 are all inside the ranges every stage tests, so the tests drop out.
  bool handed = false;  // the pencil went to the fallback pass
  auto step = [&](const int t, auto steady) {
    constexpr bool ST = decltype(steady)::value;
    if (XT && (ST || t < n) && t % kXTileCells == 0) x_chunk(*xt, t / kXTileCells, n);
    Cell Cn = Cm;
    double ges_n = 0.0;
    Flux F1 = F0;
    bool gov_next = false;
    double govv_next = 0.0;
    // (1) check of cell t
    if (live && (ST || t < n)) {
      if (PIPE) {
        cp_async_wait<(PD > 0 ? PD - 1 : 0)>();  // unit t has landed, t+1 .. t+PD-1 may not
        const double* r = ring + (t % (PD + 1)) * (kUnitVals * kMarchThreads);
        Cn = pipe_cell<DUAL>(a, r);
        if (ST || (t >= is && t <= ie)) F1 = pipe_flux(r);
        pipe_issue<DUAL, PD>(a, ring, base, pid, t + PD);  // into the slot read at t-1
      } else {
        Cn = XT ? x_cell<DUAL>(*xt, a, t) : Cpf;
        if (ST || (t >= is && t <= ie)) F1 = Fpf;
        if (ST || t + 1 < n) {
          if (!XT)
            Cpf = STAGED ? load_cell_keep<DUAL>(a, base + (int64_t)(t + 1) * sa)
                         : load_cell<DUAL>(a, base + (int64_t)(t + 1) * sa);
          if (ST || (t + 1 >= is && t + 1 <= ie)) Fpf = load_flux(a, (int64_t)(t + 2 - is) * np + pid);
        }
      }
      if (ST || (t >= is && t <= ie)) {
        if (DUAL) {
          const double pcent = dmax(P.gm1 * Cn.ge * Cn.d, kTiny);
          ges_n = gov ? govv : (RS ? F0.ub : P.dt / a.coef[t].dx * pcent * (F0.ub - F1.ub));
        }
        // RS (HLL, HLLC): flux_hll.F:336 / flux_hllc.F:332 test the density alone
        const bool bad = RS ? (Cn.d + F0.df - F1.df <= 0.0)
                            : (Cn.d + (F0.df - F1.df) <= 0.0 || Cn.e < 0.0);
        if (bad) {
          if (!FALLBACK && !STAGED) {  // hand the pencil to the fallback pass
            if (PIPE) cp_async_wait<0>();
            handed = true;
            return;
          }
          if (!FALLBACK) {  // STAGED: stop computing, keep joining the block's flushes
            live = false;
            flagged = true;
          }
        }
        if (live && bad) {
          if (a.fallback == 0) {
            cnt.fatal += 1;
          } else {
            bool fatal = false;
            cnt.fallbacks += 1;
            hll_fallback<DUAL>(a, pid, base, t, Cn, P, F0, F1, ges_n, govv_next, fatal);
            if (a.fhll) {  // these faces' colour fluxes are HLL's (weights in fcol)
              a.fhll[(int64_t)(t - is) * np + pid] = 1;
              a.fhll[(int64_t)(t + 1 - is) * np + pid] = 1;
            }
            gov_next = DUAL;
            if (fatal) cnt.fatal += 1;
          }
        }
        // subgrid flux capture: faces t (and ie+1 after the last check) are final
        while (cap < cap_end && a.captures[cap].face <= t + (t == ie ? 1 : 0)) {
          const FluxCapture& rq = a.captures[cap];
          const Flux& F = (rq.face == t) ? F0 : F1;
          double* dst = a.capture_buf + rq.dst;
          dst[0] = F.df; dst[1] = F.ef; dst[2] = F.uf;
          dst[3] = F.vf; dst[4] = F.wf; dst[5] = DUAL ? F.gef : 0.0;
          ++cap;
        }
      }
    }
    // (2) conservative update of cell t-1
    Cell PEn = Cm;
    if (live) {
      const int c = t - 1;
      if (ST || (c >= is && c <= ie)) {
        bool fatal = false;
        PEn = euler_update<DUAL, GRAV>(Cm, Fm, F0, ges_m,
                                       GRAV ? __ldg(a.grav + base + (int64_t)c * sa) : 0.0, P,
                                       fatal);
        if (fatal) cnt.fatal += 1;
      }
    }
    // (3) dual-energy select of cell t-2 and store
    {
      const int c = t - 2;
      if (live && (ST || c >= 0)) {
        Cell o = PEm;
        if (DUAL) {
          const double own = o.d * o.e;
          const double de_m = (!ST && c == 0) ? own : dep;
          const double de_p = (!ST && c == n - 1) ? own : PEn.d * PEn.e;
          pgas2d_dual(o, de_m, de_p, P);
          dep = o.d * o.e;
        }
        if (!isfinite(o.d) || !isfinite(o.e)) nonfin += 1;
        if (cfl && (ST || (c >= is && c <= ie)))
          dtmin = dmin(dtmin, cell_dt1<DUAL>(a, o, a.coef[c].dx, t1, t2, P));
        if (STAGED && PPM_X_STAGE_STORES) {
          double* sp = stage + (c % kStageCells) * kStageLd + (threadIdx.x & 31);
          sp[0] = o.d;
          sp[kStageField] = o.e;
          sp[2 * kStageField] = o.u;
          sp[3 * kStageField] = o.v;
          sp[4 * kStageField] = o.w;
          if (DUAL) sp[5 * kStageField] = o.ge;
        } else {
          const int64_t off = base + (int64_t)c * sa;
          a.out_d[off] = o.d;
          a.out_e[off] = o.e;
          if (a.out_u) a.out_u[off] = o.u;
          if (a.out_v) a.out_v[off] = o.v;
          if (a.out_w) a.out_w[off] = o.w;
          if (DUAL) a.out_ge[off] = o.ge;
        }
      }
      // warp-wide: the same steps on every lane
      if (STAGED && PPM_X_STAGE_STORES && (ST || c >= 0) && c % kStageCells == kStageCells - 1)
        flush_stage<DUAL>(a, stage, pid0, c - (kStageCells - 1), kStageCells);
    }
    Fm = F0;
    F0 = F1;
    Cm = Cn;
    ges_m = ges_n;
    gov = gov_next;
    govv = govv_next;
    PEm = PEn;
  };
  using Ramp = std::integral_constant<bool, false>;
  using Steady = std::integral_constant<bool, true>;
  // the x sweep's update (TMA tiles) gains from the steady block; the y/z update, with
  // its cp.async ring, measured slower with it (more registers than its 128)
  const int t_steady0 = XT ? is + 2 : n + 1, t_steady1 = XT ? ie - 1 : n;
#pragma unroll 1
  for (int t = 0; t < t_steady0 && t <= n; ++t) {
    step(t, Ramp{});
    if (handed) return true;
  }
  if constexpr (XT) {
#pragma unroll 1
    for (int t = t_steady0; t <= t_steady1; ++t) step(t, Steady{});
#pragma unroll 1
    for (int t = t_steady1 + 1 > t_steady0 ? t_steady1 + 1 : t_steady0; t <= n; ++t)
      step(t, Ramp{});
  }
  // the last step (t = n) leaves cell n-1 unstored; it is a ghost cell, whose
  // post-euler state is its input, selected against itself and its left neighbour
  {
    const int c = n - 1;
    if (live) {
      Cell o = PEm;
      if (DUAL) {
        const double own = o.d * o.e;
        pgas2d_dual(o, (c == 0) ? own : dep, own, P);
      }
      if (!isfinite(o.d) || !isfinite(o.e)) nonfin += 1;
      if (STAGED && PPM_X_STAGE_STORES) {
        double* sp = stage + (c % kStageCells) * kStageLd + (threadIdx.x & 31);
        sp[0] = o.d;
        sp[kStageField] = o.e;
        sp[2 * kStageField] = o.u;
        sp[3 * kStageField] = o.v;
        sp[4 * kStageField] = o.w;
        if (DUAL) sp[5 * kStageField] = o.ge;
      } else {
        const int64_t off = base + (int64_t)c * sa;
        a.out_d[off] = o.d;
        a.out_e[off] = o.e;
        if (a.out_u) a.out_u[off] = o.u;
        if (a.out_v) a.out_v[off] = o.v;
        if (a.out_w) a.out_w[off] = o.w;
        if (DUAL) a.out_ge[off] = o.ge;
      }
    }
    if (STAGED && PPM_X_STAGE_STORES) {  // the partial last chunk, cells c0 .. n-1
      const int c0 = c - c % kStageCells;
      flush_stage<DUAL>(a, stage, pid0, c0, c - c0 + 1);
    }
  }
  if (PIPE) cp_async_wait<0>();  // only empty groups remain
  if (XT) x_drain(*xt);
  cnt.nonfinite += nonfin;
  cnt.dtmin = dtmin;
  return flagged;
}

#ifndef PPM_UPDATE_MINBLOCKS
#define PPM_UPDATE_MINBLOCKS (3 * 128 / PPM_MARCH_THREADS)
#endif
// y and z sweeps: a single grid at 4 blocks/SM (the ring frees the prefetch registers),
// a batch of grids at 3
#ifndef PPM_UPDATE_YZ_MINBLOCKS
#define PPM_UPDATE_YZ_MINBLOCKS (4 * 128 / PPM_MARCH_THREADS)
#endif
// x sweep with TMA tiles: 2 blocks/SM (78 KB of shared memory a block; at 3 blocks the
// shared memory leaves too little L1)
#ifndef PPM_UPDATE_XT_MINBLOCKS
#define PPM_UPDATE_XT_MINBLOCKS (2 * 128 / PPM_MARCH_THREADS)
#endif
#ifndef PPM_UPDATE_YZ_BATCH_MINBLOCKS
#define PPM_UPDATE_YZ_BATCH_MINBLOCKS PPM_UPDATE_MINBLOCKS
#endif

// the input ring's distance: none for the x sweep
template <bool ONE, bool STAGED>
__host__ __device__ constexpr int update_pipe() {
  return STAGED ? 0 : (ONE ? PPM_UPDATE_PIPE_ONE : PPM_UPDATE_PIPE_BATCH);
}
constexpr int kStageBlock = (kMarchThreads / 32) * kStageWarp;
constexpr int kXBlock = (kMarchThreads / 32) * kXWarp;
// dynamic shared memory of the update kernel: the x sweep's TMA tiles (XT) and output
// staging, one of each per warp, or the y and z sweeps' input ring
template <bool ONE, bool STAGED, bool XT>
constexpr size_t update_smem_bytes() {
  return sizeof(double) * ((XT ? kXBlock : 0) + (STAGED ? kStageBlock : 0) +
                           ring_doubles<update_pipe<ONE, STAGED>()>());
}

// STAGED: the x sweep (pencils along the contiguous axis) with staged outputs; XT: its
// input cells as TMA tiles (a single grid with B.x_tma set).
// RS: HLL or HLLC fluxes (ges precomputed in the XUB plane, the density-only check)
template <bool DUAL, bool GRAV, bool ONE, bool STAGED, bool XT, bool RS = false>
__global__ void __launch_bounds__(kMarchThreads,
                                  STAGED ? (XT ? PPM_UPDATE_XT_MINBLOCKS : PPM_UPDATE_MINBLOCKS)
                                         : (ONE ? PPM_UPDATE_YZ_MINBLOCKS
                                                : PPM_UPDATE_YZ_BATCH_MINBLOCKS))
    update_kernel(const __grid_constant__ BatchArgs B) {
  static_assert(!XT || (ONE && STAGED), "TMA tiles serve the x sweep of a single grid");
  __shared__ unsigned long long s_cnt[2];
  __shared__ uint64_t s_xbar[XT ? (kMarchThreads / 32) * kXBuffers : 1];
  extern __shared__ __align__(128) double s_dyn[];
  double* const s_xtile = s_dyn;                                // XT: kXWarp per warp
  double* const s_stage = s_dyn + (XT ? kXBlock : 0);           // STAGED: kStageWarp per warp
  double* const s_ring = s_dyn;                                 // y, z: the input ring
  if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0ull;
  int64_t lb;
  const int g = locate<ONE>(B.march_prefix, B.ngrids, lb);
  PPM_BIND_RECORD(a, g)
  const int64_t pid = lb * kMarchThreads + threadIdx.x;
  const int64_t wpid0 = pid - (threadIdx.x & 31);  // first pencil of this warp
  const int warp = threadIdx.x >> 5;
  XTiles xt;
  if (XT) {
    xt.buf = s_xtile + warp * kXWarp;
    xt.bar = s_xbar + warp * kXBuffers;
    xt.map = B.xin;
    xt.timeouts = B.counters + kCntTimeout;
    xt.fields = 3u | (a.in_u ? 4u : 0u) | (a.in_v ? 8u : 0u) | (a.in_w ? 16u : 0u) |
                ((DUAL && a.in_ge) ? 32u : 0u);
    xt.bytes = (unsigned)__popc(xt.fields) * kXTile * (unsigned)sizeof(double) +
               B.x_tma_extra_tx;
    xt.row0 = (int)wpid0;
    xt.last = -1;
    xt.broken = false;
    if ((threadIdx.x & 31) == 0) {
      for (int b = 0; b < kXBuffers; ++b) mbar_init(xt.bar + b, 1);
      // the barriers' initialisation is visible to the tensor-memory accelerator
      asm volatile("fence.mbarrier_init.release.cluster;\n\tfence.proxy.async.shared::cta;" ::
                       : "memory");
    }
  }
  if (ONE) __syncthreads();
  double my_dt = 1.0e20;
  const bool valid = pid < a.npencils;
  if (STAGED || valid) {
    const Phys P = make_phys(a);
    UpdateCounts cnt = {0, 0, 0, 1.0e20};
    if (update_pencil<DUAL, GRAV, false, STAGED, update_pipe<ONE, STAGED>(), XT, RS>(
            a, pid, P, cnt, valid, s_stage + warp * kStageWarp, wpid0, s_ring + threadIdx.x,
            &xt)) {
      const unsigned long long slot = atomicAdd(&B.counters[kCntFlagged], 1ull);
      B.flagged[slot] = ((int64_t)g << 40) | pid;
    } else {
      if (cnt.fatal) atomicAdd(&s_cnt[0], (unsigned long long)cnt.fatal);
      if (cnt.nonfinite) atomicAdd(&s_cnt[1], (unsigned long long)cnt.nonfinite);
      my_dt = cnt.dtmin;  // a flagged pencil's time step comes from the fallback pass
    }
  }
  if (a.cfl_min_bits) {  // warp minimum, one atomic per warp (every lane reaches this)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) my_dt = dmin(my_dt, __shfl_xor_sync(0xffffffffu, my_dt, o));
    if ((threadIdx.x & 31) == 0 && my_dt < 1.0e20)
      atomicMin(a.cfl_min_bits, (unsigned long long)__double_as_longlong(my_dt));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_cnt[0]) atomicAdd(&B.counters[kCntFatal], s_cnt[0]);
    if (s_cnt[1]) atomicAdd(&B.counters[kCntNonFinite], s_cnt[1]);
  }
}

// The fallback pass: a fixed grid that walks the list of flagged pencils.
template <bool DUAL, bool GRAV, bool ONE, bool RS = false>
__global__ void __launch_bounds__(128) fallback_kernel(const __grid_constant__ BatchArgs B) {
  const unsigned long long nflag = *(volatile unsigned long long*)&B.counters[kCntFlagged];
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
       k < nflag; k += (unsigned long long)gridDim.x * blockDim.x) {
    const int64_t code = B.flagged[k];
    const SweepArgs& a = ONE ? B.one : B.grids[(int)(code >> 40)];
    const Phys P = make_phys(a);
    UpdateCounts cnt = {0, 0, 0, 1.0e20};
    update_pencil<DUAL, GRAV, true, false, 0, false, RS>(a, code & ((int64_t(1) << 40) - 1), P,
                                                        cnt);
    if (a.cfl_min_bits && cnt.dtmin < 1.0e20)
      atomicMin(a.cfl_min_bits, (unsigned long long)__double_as_longlong(cnt.dtmin));
    if (cnt.fallbacks) atomicAdd(&B.counters[kCntFallbacks], (unsigned long long)cnt.fallbacks);
    if (cnt.fatal) atomicAdd(&B.counters[kCntFatal], (unsigned long long)cnt.fatal);
    if (cnt.nonfinite) atomicAdd(&B.counters[kCntNonFinite], (unsigned long long)cnt.nonfinite);
  }
}

// ------------------------------------------------------------------ stage 5 (colours)
// The colour fields of the sweep (NumberOfColours > 0), one thread per (pencil, chunk of
// colours), marching like the reconstruction: each colour's PPM parabola (intvar with the
// slice's flattening and no steepening, inteuler.F:276-282), its face states scaled by
// the corrected density and undone with the dual-energy override (inteuler.F:436-450,
// :500-515) and floored (:546-551), the flux at the Godunov state
// (flux_twoshock.F:251-259, :375-380) or, on faces the HLL fallback replaced, HLL's
// (flux_hll.F:236-262, :328-332), divided by dx (euler.F:173-176), the subgrid-flux
// capture of that quotient (Grid_xEulerSweep.C:361-371), and the update with its floor
// (euler.F:178-186), written in place: a cell is read three steps before it is written
// and never read again.
// Blocks: (march block, colour chunk) with the chunk fastest, so that the blocks of one
// pencil block run together and share their density, pressure, velocity and face reads
// through L2; within a thread the colours of a chunk share them outright.
#ifndef PPM_COLOUR_MINBLOCKS
#define PPM_COLOUR_MINBLOCKS 4
#endif
#ifndef PPM_COLOURS_PER_THREAD
#define PPM_COLOURS_PER_THREAD 2
#endif
// below this many (pencil block, colour) pairs a sweep runs one colour per thread: two
// would leave too few warps to hide the march's load latency (128^3 with 4 colours: 7.5
// of 16 warps active per SM)
#ifndef PPM_COLOUR_WIDE_BLOCKS
#define PPM_COLOUR_WIDE_BLOCKS (148 * 8)
#endif
constexpr double kColourFloor = 1.0e-35;        // color_floor, fortran.def:8
constexpr double kMinColour = 1.0e-5 * kTiny;   // min_color, euler.F:104-105

// CPT colours per thread: each thread marches one pencil for colours c0 .. c0+CPT-1 of
// its block's chunk, sharing the cell and face data between them.
template <bool DUAL, bool ONE, int CPT>
__global__ void __launch_bounds__(kMarchThreads, PPM_COLOUR_MINBLOCKS)
    colour_kernel(const __grid_constant__ BatchArgs B) {
  const int nc = B.ncolour;
  const int nchunk = (nc + CPT - 1) / CPT;
  const int64_t mb = blockIdx.x / nchunk;
  const int chunk = (int)(blockIdx.x - mb * nchunk);
  int64_t lb = mb;
  const int g = ONE ? 0 : batch_locate(B.march_prefix, B.ngrids, mb, lb);
  PPM_BIND_RECORD(a, g)
  const int64_t pid = lb * kMarchThreads + threadIdx.x;
  if (pid >= a.npencils) return;
  const Phys P = make_phys(a);
  const int64_t base = (pid % a.n1) * a.s1 + (pid / a.n1) * a.s2;
  const int64_t sa = a.sa;
  const int is = a.is, ie = a.ie;
  const int64_t np = a.npencils, plane = a.plane;
  const int c0 = chunk * CPT;
  const int ncol = nc - c0 < CPT ? nc - c0 : CPT;  // colours of this chunk
  double* q[CPT];
#pragma unroll
  for (int u = 0; u < CPT; ++u) q[u] = u < ncol ? a.col[c0 + u] : nullptr;

  int64_t cap = 0, cap_end = 0;
  if (a.ncaptures > 0) {
    int64_t lo = 0, hi = a.ncaptures;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (a.captures[mid].pencil < pid) lo = mid + 1; else hi = mid;
    }
    cap = cap_end = lo;
    while (cap_end < a.ncaptures && a.captures[cap_end].pencil == pid) ++cap_end;
  }

  double wq0[CPT], wq1[CPT], wq2[CPT];  // colour of cells t-3, t-2, t-1
  double dqm1[CPT], qlm1[CPT];          // dq(t-2), ql(t-2)
  double colla[CPT], coll0[CPT];        // left data of face t-2
  double fm[CPT];                       // colf / dx of face t-3
#pragma unroll
  for (int u = 0; u < CPT; ++u)
    wq0[u] = wq1[u] = wq2[u] = dqm1[u] = qlm1[u] = colla[u] = coll0[u] = fm[u] = 0.0;
  double wu0 = 0.0, wu1 = 0.0, wu2 = 0.0;  // normal velocity of cells t-3, t-2, t-1
  Prep prA = {0, 0, 0, 0, 0}, prB = {0, 0, 0, 0, 0};  // cells t-2, t-1
  const int tend = ie + 3;
#pragma unroll 1
  for (int t = 0; t <= tend; ++t) {
    const int64_t off = base + (int64_t)t * sa;
    double nq[CPT];
#pragma unroll
    for (int u = 0; u < CPT; ++u) nq[u] = u < ncol ? q[u][off] : 0.0;
    const double nu = ldg0(a.in_u, off);
    Prep prC = prB;
    if (t >= is - 1 && t <= ie + 1)
      prC = a.presfree ? cell_prep<true>(__ldg(a.in_d + off), __ldg(a.pres + off), nu,
                                         a.coef[t].dx2i, P)
                       : cell_prep(__ldg(a.in_d + off), __ldg(a.pres + off), nu,
                                   a.coef[t].dx2i, P);
    double dqN[CPT], qlN[CPT];  // slope and left edge of cell t-1
#pragma unroll
    for (int u = 0; u < CPT; ++u) dqN[u] = qlN[u] = 0.0;
    {
      const int c = t - 1;
      if (c >= is - 2 && c <= ie + 2) {
        const Coef cf = a.coef[c];
#pragma unroll
        for (int u = 0; u < CPT; ++u) {
          dqN[u] = pm_slope(wq1[u], wq2[u], nq[u], cf.c1, cf.c2);
          if (c >= is - 1) qlN[u] = pm_edge(wq1[u], wq2[u], dqm1[u], dqN[u], cf.c3, cf.c4, cf.c5, cf.c6);
        }
      }
    }
    {
      const int c = t - 2;  // parabola of cell c; face c
      if (c >= is - 1 && c <= ie + 1) {
        const double fl = a.flatten != 0 ? a.flat[(int64_t)(c - (is - 1)) * np + pid] : 0.0;
        Para pa[CPT];
#pragma unroll
        for (int u = 0; u < CPT; ++u)
          pa[u] = a.flatten != 0
                      ? pm_parabola<false, true>(wq0[u], wq1[u], wq2[u], qlm1[u], qlN[u], 0.0,
                                                 0.0, 0.0, fl)
                      : pm_parabola(wq0[u], wq1[u], wq2[u], qlm1[u], qlN[u]);
        if (c >= is) {
          const int64_t fidx = (int64_t)(c - is) * np + pid;
          const double* fc = a.fcol + fidx;
          const double dla = fc[CDLA * plane], dl0 = fc[CDL0 * plane];
          const double dra = fc[CDRA * plane], dr0 = fc[CDR0 * plane];
          const double dlc = fc[CDLC * plane], drc = fc[CDRC * plane];
          const double ov = fc[COVR * plane];
          const bool ovl = ov == 1.0 || ov == 3.0, ovr = ov >= 2.0;
          const bool hll = a.solver != 0 || a.fhll[fidx] != 0;
          double w[4] = {0.0, 0.0, 0.0, 0.0};
          double ub = 0.0, db = 0.0, dsl = 1.0, dsr = 1.0;
          if (hll) {  // the HLL weights the fallback pass left (sl, bm0, sr, bp0)
            w[0] = fc[CHSL * plane];
            w[1] = fc[CHBM * plane];
            w[2] = fc[CHSR * plane];
            w[3] = fc[CHBP * plane];
          } else {
            ub = a.fflux[XUB * plane + fidx];
            db = fc[CDB * plane];
            if (ub > 0.0) dsl = a.fstate[SDL * plane + fidx];
            else dsr = a.fstate[SDR * plane + fidx];
          }
          const double dx = a.coef[c].dx;
          int64_t cq = cap;  // this face's capture requests (the same for every colour)
#pragma unroll
          for (int u = 0; u < CPT; ++u) {
            if (u >= ncol) break;
            const double colra = pm_C(pa[u], prA.char2), colr0 = pm_B(pa[u], prA.c0);
            double cls = (wu0 <= 0.0) ? colla[u] * dlc / dla : coll0[u] * dlc / dl0;
            double crs = (wu1 >= 0.0) ? colra * drc / dra : colr0 * drc / dr0;
            if (ovl) cls = cls * dla / dlc;
            if (ovr) crs = crs * dra / drc;
            cls = dmax(cls, kColourFloor);
            crs = dmax(crs, kColourFloor);
            double cf;
            if (hll) {
              cf = w[0] * (w[1] * cls) + w[2] * (w[3] * crs);
              cf = P.dt * cf;
            } else {
              const double colb = ub > 0.0 ? cls * db / dsl : crs * db / dsr;
              cf = P.dt * ub * colb;
            }
            cf = cf / dx;
            for (cq = cap; cq < cap_end && a.captures[cq].face <= c; ++cq) {
              const FluxCapture& rq = a.captures[cq];
              if (rq.face == c) a.col_capture[(rq.dst / 6) * nc + c0 + u] = cf;
            }
            if (c - 1 >= is && c - 1 <= ie) {
              const double v = wq0[u] + (fm[u] - cf);
              q[u][base + (int64_t)(c - 1) * sa] = dmax(v, kMinColour);
            }
            fm[u] = cf;
          }
          cap = cq;
        }
        if (c <= ie) {
#pragma unroll
          for (int u = 0; u < CPT; ++u) {
            colla[u] = pm_A(pa[u], prA.char1);
            coll0[u] = pm_A(pa[u], prA.c0);
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < CPT; ++u) {
      wq0[u] = wq1[u];
      wq1[u] = wq2[u];
      wq2[u] = nq[u];
      dqm1[u] = dqN[u];
      qlm1[u] = qlN[u];
    }
    wu0 = wu1;
    wu1 = wu2;
    wu2 = nu;
    prA = prB;
    prB = prC;
  }
}

// Above 48 KB of dynamic shared memory a kernel needs the opt-in attribute, set once
// per device (a function attribute is not a stream operation, so this is also legal
// while a stream is being captured).
template <bool DUAL, bool GRAV, bool ONE, bool STAGED, bool XT, bool RS = false>
void launch_update(const BatchArgs& B, int64_t march_blocks, cudaStream_t st) {
  constexpr size_t bytes = update_smem_bytes<ONE, STAGED, XT>();
  if (bytes > 48 * 1024) {
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(done.load(std::memory_order_acquire) & bit)) {
      cudaFuncSetAttribute(update_kernel<DUAL, GRAV, ONE, STAGED, XT, RS>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
      done.fetch_or(bit, std::memory_order_release);
    }
  }
  update_kernel<DUAL, GRAV, ONE, STAGED, XT, RS>
      <<<(unsigned)march_blocks, kMarchThreads, bytes, st>>>(B);
}

// The two-shock stage with the plain start: the block size and persistence the batch
// asks for.  riemann_blocks: the launch's grid (the resident blocks when persistent).
template <bool DUAL, bool ONE, int RT>
void launch_riemann_rt(const BatchArgs& B, unsigned rb, cudaStream_t st) {
  if (B.persistent)
    riemann_kernel<DUAL, ONE, false, false, RT, true><<<rb, RT, 0, st>>>(B);
  else
    riemann_kernel<DUAL, ONE, false, false, RT, false><<<rb, RT, 0, st>>>(B);
}

template <bool DUAL, bool ONE>
void launch_riemann_plain(const BatchArgs& B, unsigned rb, cudaStream_t st) {
  if (B.riemann_threads == 64)
    launch_riemann_rt<DUAL, ONE, 64>(B, rb, st);
  else if (B.riemann_threads == 256)
    launch_riemann_rt<DUAL, ONE, 256>(B, rb, st);
  else
    launch_riemann_rt<DUAL, ONE, kRiemannThreads>(B, rb, st);
}

template <bool DUAL, bool GRAV, bool ONE>
void launch_stages(const BatchArgs& B, int64_t march_blocks, int64_t riemann_blocks,
                   cudaStream_t st, cudaEvent_t* ev, bool learned, bool staged) {
  auto mark = [&](int k) {
    if (ev) cudaEventRecord(ev[k], st);
  };
  mark(0);
  cudaMemsetAsync(B.counters + kCntFlagged, 0, sizeof(unsigned long long), st);
  if (B.fused) {  // the plain path with the fused face kernel
    face_kernel<DUAL, GRAV, ONE><<<(unsigned)B.face_blocks, kFaceThreads, 0, st>>>(B);
    mark(1);
    mark(2);
    mark(3);
    if (PPM_X_TMA && staged && ONE && B.x_tma)
      launch_update<DUAL, GRAV, ONE, true, ONE>(B, march_blocks, st);
    else if (staged)
      launch_update<DUAL, GRAV, ONE, true, false>(B, march_blocks, st);
    else
      launch_update<DUAL, GRAV, ONE, false, false>(B, march_blocks, st);
    mark(4);
    // the flagged pencils' interface states, then their per-cell HLL fallback
    reconstruct_kernel<DUAL, GRAV, 0, ONE, false, true><<<64, kMarchThreads, 0, st>>>(B);
    reconstruct_kernel<DUAL, GRAV, 1, ONE, false, true><<<64, kMarchThreads, 0, st>>>(B);
    fallback_kernel<DUAL, GRAV, ONE><<<64, 128, 0, st>>>(B);
    mark(5);
    return;
  }
  if (B.ncolour > 0) cudaMemsetAsync(B.hll_flags, 0, (size_t)B.hll_bytes, st);
  if (B.corrections || B.ncolour > 0 || B.presfree) {  // colours, PressureFree: COR too
    if (B.corrections)
      corrections_kernel<ONE><<<(unsigned)march_blocks, kMarchThreads, 0, st>>>(B);
    reconstruct_kernel<DUAL, GRAV, 0, ONE, true><<<(unsigned)march_blocks, kMarchThreads, 0, st>>>(B);
    mark(1);
    reconstruct_kernel<DUAL, GRAV, 1, ONE, true><<<(unsigned)march_blocks, kMarchThreads, 0, st>>>(B);
  } else {
    reconstruct_kernel<DUAL, GRAV, 0, ONE><<<(unsigned)march_blocks, kMarchThreads, 0, st>>>(B);
    mark(1);
    reconstruct_kernel<DUAL, GRAV, 1, ONE><<<(unsigned)march_blocks, kMarchThreads, 0, st>>>(B);
  }
  mark(2);
  const unsigned rb = (unsigned)riemann_blocks;
  const bool col = B.ncolour > 0;
  if (B.solver == 0 && B.presfree && col)
    presfree_riemann_kernel<DUAL, ONE, true><<<rb, kRiemannThreads, 0, st>>>(B);
  else if (B.solver == 0 && B.presfree)
    presfree_riemann_kernel<DUAL, ONE, false><<<rb, kRiemannThreads, 0, st>>>(B);
  else if (B.solver == 1 && col)
    hll_riemann_kernel<DUAL, ONE, false, true><<<rb, kRiemannThreads, 0, st>>>(B);
  else if (B.solver == 1)
    hll_riemann_kernel<DUAL, ONE, false, false><<<rb, kRiemannThreads, 0, st>>>(B);
  else if (B.solver == 2 && col)
    hll_riemann_kernel<DUAL, ONE, true, true><<<rb, kRiemannThreads, 0, st>>>(B);
  else if (B.solver == 2)
    hll_riemann_kernel<DUAL, ONE, true, false><<<rb, kRiemannThreads, 0, st>>>(B);
  else if (learned && B.ncolour > 0)
    riemann_kernel<DUAL, ONE, true, true><<<rb, kRiemannThreads, 0, st>>>(B);
  else if (learned && B.learned_pass) {
    launch_guess_pass(B, B.sms, st);
    riemann_kernel<DUAL, ONE, true, false, kRiemannThreads, false, true>
        <<<rb, kRiemannThreads, 0, st>>>(B);
  } else if (learned)
    riemann_kernel<DUAL, ONE, true><<<rb, kRiemannThreads, 0, st>>>(B);
  else if (B.ncolour > 0)
    riemann_kernel<DUAL, ONE, false, true><<<rb, kRiemannThreads, 0, st>>>(B);
  else
    launch_riemann_plain<DUAL, ONE>(B, rb, st);
  mark(3);
  if (B.solver != 0) {  // HLL / HLLC
    if (PPM_X_TMA && staged && ONE && B.x_tma)
      launch_update<DUAL, GRAV, ONE, true, ONE, true>(B, march_blocks, st);
    else if (staged)
      launch_update<DUAL, GRAV, ONE, true, false, true>(B, march_blocks, st);
    else
      launch_update<DUAL, GRAV, ONE, false, false, true>(B, march_blocks, st);
    mark(4);
    fallback_kernel<DUAL, GRAV, ONE, true><<<64, 128, 0, st>>>(B);
  } else {
    if (PPM_X_TMA && staged && ONE && B.x_tma)
      launch_update<DUAL, GRAV, ONE, true, ONE>(B, march_blocks, st);
    else if (staged)
      launch_update<DUAL, GRAV, ONE, true, false>(B, march_blocks, st);
    else
      launch_update<DUAL, GRAV, ONE, false, false>(B, march_blocks, st);
    mark(4);
    fallback_kernel<DUAL, GRAV, ONE><<<64, 128, 0, st>>>(B);
  }
  if (B.ncolour > 0) {
    constexpr int cpt = PPM_COLOURS_PER_THREAD;
    const int64_t chunks = (B.ncolour + cpt - 1) / cpt;
    if (march_blocks * B.ncolour < PPM_COLOUR_WIDE_BLOCKS)
      colour_kernel<DUAL, ONE, 1>
          <<<(unsigned)(march_blocks * B.ncolour), kMarchThreads, 0, st>>>(B);
    else
      colour_kernel<DUAL, ONE, cpt><<<(unsigned)(march_blocks * chunks), kMarchThreads, 0, st>>>(B);
  }
  mark(5);
}

template <bool DUAL, bool GRAV>
void launch_any(const BatchArgs& B, int64_t march_blocks, int64_t riemann_blocks,
                cudaStream_t st, cudaEvent_t* ev, bool learned, bool staged) {
  if (B.ngrids == 1)
    launch_stages<DUAL, GRAV, true>(B, march_blocks, riemann_blocks, st, ev, learned, staged);
  else
    launch_stages<DUAL, GRAV, false>(B, march_blocks, riemann_blocks, st, ev, learned, staged);
}

}  // namespace split

// One directional sweep of every grid of a batch: five launches (six with slope
// corrections, one more with colours; the Riemann stage by B.solver and B.presfree,
// the reconstruction's corrections variant whenever corrections, colours or
// PressureFree need it).  The caller provides
// each grid's fstate / fflux / plane, the prefix tables and the flagged list, and for a
// batch of one grid also B.one (a copy of that grid's record).  ev (optional): six
// events recorded before each kernel and after the last.  learned: start the Newton
// iteration from the MLP guess (every record's `guess` must point at packed weights).
// contiguous: every grid's pencils run along the contiguous axis (sa == 1, the x
// sweep); the update kernel then stages its stores.
// Resident blocks per SM of the persistent two-shock stage for a block size (the grid of
// a persistent launch is this times the SM count).
int riemann_resident_blocks(bool dual, bool one, int threads) {
  int n = 0;
  auto occ = [&](auto kern, int rt) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, rt, 0);
  };
  if (threads == 64) {
    if (dual) one ? occ(split::riemann_kernel<true, true, false, false, 64, true>, 64)
              : occ(split::riemann_kernel<true, false, false, false, 64, true>, 64);
    else one ? occ(split::riemann_kernel<false, true, false, false, 64, true>, 64)
             : occ(split::riemann_kernel<false, false, false, false, 64, true>, 64);
  } else if (threads == 256) {
    if (dual) one ? occ(split::riemann_kernel<true, true, false, false, 256, true>, 256)
              : occ(split::riemann_kernel<true, false, false, false, 256, true>, 256);
    else one ? occ(split::riemann_kernel<false, true, false, false, 256, true>, 256)
             : occ(split::riemann_kernel<false, false, false, false, 256, true>, 256);
  } else {
    constexpr int rt = kRiemannThreads;
    if (dual) one ? occ(split::riemann_kernel<true, true, false, false, rt, true>, rt)
              : occ(split::riemann_kernel<true, false, false, false, rt, true>, rt);
    else one ? occ(split::riemann_kernel<false, true, false, false, rt, true>, rt)
             : occ(split::riemann_kernel<false, false, false, false, rt, true>, rt);
  }
  return n > 0 ? n : 1;
}

void launch_sweep_batch(const BatchArgs& B, int64_t march_blocks, int64_t riemann_blocks,
                        bool dual, bool grav, cudaStream_t st, cudaEvent_t* ev, bool learned,
                        bool contiguous) {
  const int64_t mb = march_blocks, rb = riemann_blocks;
  if (dual && grav) split::launch_any<true, true>(B, mb, rb, st, ev, learned, contiguous);
  else if (dual) split::launch_any<true, false>(B, mb, rb, st, ev, learned, contiguous);
  else if (grav) split::launch_any<false, true>(B, mb, rb, st, ev, learned, contiguous);
  else split::launch_any<false, false>(B, mb, rb, st, ev, learned, contiguous);
}

}  // namespace ppm
