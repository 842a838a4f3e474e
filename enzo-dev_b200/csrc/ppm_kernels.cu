// ppm_kernels.cu -- sm_100a kernels of the PPM-DE hot path.
//
//   sweep_kernel<DUAL,GRAV>   one directional sweep (inteuler + twoshock + flux_twoshock
//                             [+ per-cell flux_hll fallback] + euler + pgas2d_dual), fused
//   pressure_kernel           grid::ComputePressure (time == Time)
//   timestep_kernel           calc_dt (ihydro = 0) min-reduction + Courant factor
//   boundary_kernel           outflow / periodic ghost-zone fill of one grid
//
// Sweep schedule: one thread owns one pencil and marches along it; the values that
// the reference keeps in its 1-D `ijkn` temporaries live in a short register pipeline
// instead.  Marching keeps the reference's sequential semantics along a pencil exactly
// (pgas2d_dual reads the already-updated left neighbour; the HLL fallback of cell i
// rewrites face i+1 before cell i+1 is checked) with no redundant stencil work and no
// intra-block synchronisation.  Pencils of the y and z sweeps are adjacent in x, so a
// warp's loads and stores are contiguous 256-byte rows: no global transposes.
// Sweeps are out of place (input set -> output set), so the fallback can rebuild face
// states from untouched inputs.
#include <cuda_runtime.h>

#include "ppm_device.cuh"
#include "ppm_sweep.cuh"

namespace ppm {

enum { VD = 0, VP = 1, VU = 2, VV = 3, VW = 4, VGE = 5 };

__device__ __forceinline__ double ldg0(const double* __restrict__ p, int64_t off) {
  return p ? __ldg(p + off) : 0.0;
}

template <bool DUAL>
__device__ __forceinline__ void load_cell(const SweepArgs& a, int64_t off, double (&q)[6],
                                          double& e) {
  q[VD] = __ldg(a.in_d + off);
  q[VP] = __ldg(a.pres + off);
  q[VU] = ldg0(a.in_u, off);
  q[VV] = ldg0(a.in_v, off);
  q[VW] = ldg0(a.in_w, off);
  q[VGE] = DUAL ? __ldg(a.in_ge + off) : 0.0;
  e = __ldg(a.in_e + off);
}

// Left-of-face data contributed by cell c (inteuler.F:304-316 and intvar.F:162-174, the
// i-1 terms) and right-of-face data contributed by cell c (the i terms).
template <bool DUAL>
__device__ __forceinline__ Lside make_left(const Para (&pa)[6], const Prep& pr) {
  Lside L;
  L.dla = pm_A(pa[VD], pr.char1);
  L.dl0 = pm_A(pa[VD], pr.c0);
  L.pla = pm_A(pa[VP], pr.char1);
  L.pl0 = pm_A(pa[VP], pr.c0);
  L.plm = pm_A(pa[VP], pr.cm);
  L.plp = pm_A(pa[VP], pr.cp);
  L.ula = pm_A(pa[VU], pr.char1);
  L.ul0 = pm_A(pa[VU], pr.c0);
  L.ulm = pm_A(pa[VU], pr.cm);
  L.ulp = pm_A(pa[VU], pr.cp);
  L.vla = pm_A(pa[VV], pr.char1);
  L.vl0 = pm_A(pa[VV], pr.c0);
  L.wla = pm_A(pa[VW], pr.char1);
  L.wl0 = pm_A(pa[VW], pr.c0);
  if (DUAL) {
    L.gela = pm_A(pa[VGE], pr.char1);
    L.gel0 = pm_A(pa[VGE], pr.c0);
  } else {
    L.gela = 0.0;
    L.gel0 = 0.0;
  }
  L.cm = pr.cm;
  L.c0 = pr.c0;
  L.cp = pr.cp;
  return L;
}

template <bool DUAL>
__device__ __forceinline__ Rside make_right(const Para (&pa)[6], const Prep& pr) {
  Rside R;
  R.dra = pm_C(pa[VD], pr.char2);
  R.dr0 = pm_B(pa[VD], pr.c0);
  R.pra = pm_C(pa[VP], pr.char2);
  R.pr0 = pm_B(pa[VP], pr.c0);
  R.prm = pm_B(pa[VP], pr.cm);
  R.prp = pm_B(pa[VP], pr.cp);
  R.ura = pm_C(pa[VU], pr.char2);
  R.ur0 = pm_B(pa[VU], pr.c0);
  R.urm = pm_B(pa[VU], pr.cm);
  R.urp = pm_B(pa[VU], pr.cp);
  R.vra = pm_C(pa[VV], pr.char2);
  R.vr0 = pm_B(pa[VV], pr.c0);
  R.wra = pm_C(pa[VW], pr.char2);
  R.wr0 = pm_B(pa[VW], pr.c0);
  if (DUAL) {
    R.gera = pm_C(pa[VGE], pr.char2);
    R.ger0 = pm_B(pa[VGE], pr.c0);
  } else {
    R.gera = 0.0;
    R.ger0 = 0.0;
  }
  R.cm = pr.cm;
  R.c0 = pr.c0;
  R.cp = pr.cp;
  return R;
}

// Rebuild the Riemann input state of face f from the untouched input arrays (cells
// f-3 .. f+2).  Only the HLL fallback calls this; it evaluates exactly the same
// per-point functions as the marching pipeline.
template <bool DUAL, bool GRAV>
__device__ __noinline__ FaceState rebuild_face(const SweepArgs& a, int64_t base, int f,
                                               const Phys& P) {
  constexpr int NV = DUAL ? 6 : 5;
  double q[6][6];  // q[k][v], cells f-3+k
  double e;
  for (int k = 0; k < 6; ++k) load_cell<DUAL>(a, base + (int64_t)(f - 3 + k) * a.sa, q[k], e);
  double dq[4][6];  // cells f-2 .. f+1
  for (int k = 0; k < 4; ++k) {
    const Coef cf = a.coef[f - 2 + k];
#pragma unroll
    for (int v = 0; v < NV; ++v) dq[k][v] = pm_slope(q[k][v], q[k + 1][v], q[k + 2][v], cf.c1, cf.c2);
  }
  double ql[3][6];  // cells f-1 .. f+1
  for (int k = 0; k < 3; ++k) {
    const Coef cf = a.coef[f - 1 + k];
#pragma unroll
    for (int v = 0; v < NV; ++v)
      ql[k][v] = pm_edge(q[k + 1][v], q[k + 2][v], dq[k][v], dq[k + 1][v], cf.c3, cf.c4, cf.c5, cf.c6);
  }
  Para pl[6], pr[6];
#pragma unroll
  for (int v = 0; v < 6; ++v) {
    pl[v] = Para{0.0, 0.0, 0.0, 0.0};
    pr[v] = Para{0.0, 0.0, 0.0, 0.0};
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    pl[v] = pm_parabola(q[1][v], q[2][v], q[3][v], ql[0][v], ql[1][v]);  // cell f-1
    pr[v] = pm_parabola(q[2][v], q[3][v], q[4][v], ql[1][v], ql[2][v]);  // cell f
  }
  Prep ppl = cell_prep(q[2][VD], q[2][VP], q[2][VU], a.coef[f - 1].dx2i, P);
  Prep ppr = cell_prep(q[3][VD], q[3][VP], q[3][VU], a.coef[f].dx2i, P);
  Lside L = make_left<DUAL>(pl, ppl);
  Rside R = make_right<DUAL>(pr, ppr);
  double gsum = 0.0;
  if (GRAV) gsum = __ldg(a.grav + base + (int64_t)(f - 1) * a.sa) + __ldg(a.grav + base + (int64_t)f * a.sa);
  return face_assemble<DUAL, GRAV>(L, R, q[2][VU], q[3][VU], gsum, P);
}

template <bool DUAL, bool GRAV>
__global__ void __launch_bounds__(128) sweep_kernel(const __grid_constant__ SweepArgs a) {
  constexpr int NV = DUAL ? 6 : 5;
  __shared__ unsigned long long s_cnt[kMaxCounters];
  if (threadIdx.x < kMaxCounters) s_cnt[threadIdx.x] = 0ull;
  __syncthreads();

  const int64_t pid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (pid < a.npencils) {
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

    const int64_t t1 = pid % a.n1, t2 = pid / a.n1;
    const int64_t base = t1 * a.s1 + t2 * a.s2;
    const int64_t sa = a.sa;
    const int n = a.n, is = a.is, ie = a.ie;

    // capture requests of this pencil (sorted by pencil, then face)
    int64_t cap = 0, cap_end = 0;
    if (a.ncaptures > 0) {
      int64_t lo = 0, hi = a.ncaptures;
      while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (a.captures[mid].pencil < pid) lo = mid + 1; else hi = mid;
      }
      cap = lo;
      cap_end = lo;
      while (cap_end < a.ncaptures && a.captures[cap_end].pencil == pid) ++cap_end;
    }

    // ---- pipeline state, as of the top of iteration t
    double wq0[6], wq1[6], wq2[6];  // cells t-3, t-2, t-1
    double we0 = 0.0, we1 = 0.0, we2 = 0.0;
    double wg0 = 0.0, wg1 = 0.0, wg2 = 0.0;
    double dqm1[6], qlm1[6];        // dq(t-2), ql(t-2)
#pragma unroll
    for (int v = 0; v < 6; ++v) {
      wq0[v] = wq1[v] = wq2[v] = 0.0;
      dqm1[v] = qlm1[v] = 0.0;
    }
    Prep prA = {0, 0, 0, 0, 0}, prB = {0, 0, 0, 0, 0};  // prep of cells t-2, t-1
    Lside Lp = {};                   // left data of face t-2 (from cell t-3)
    Flux Fp = {0, 0, 0, 0, 0, 0, 0}; // flux at face t-3
    bool gov = false;                // ges(t-3) was set by a fallback at cell t-4
    double govv = 0.0;
    Cell PEp = {0, 0, 0, 0, 0, 0};   // post-euler state of cell t-4
    double dep = 0.0;                // post-pgas d*e of cell t-5
    unsigned int c_if = 0, c_newton = 0, c_fb = 0, c_fatal = 0, c_nonfin = 0;
    unsigned int c_hist[8] = {0, 0, 0, 0, 0, 0, 0, 0};

#pragma unroll 1
    for (int t = 0; t < n + 4; ++t) {
      // 1. load cell t
      double nq[6] = {0, 0, 0, 0, 0, 0};
      double ne = 0.0, ng = 0.0;
      if (t < n) {
        load_cell<DUAL>(a, base + (int64_t)t * sa, nq, ne);
        if (GRAV) ng = __ldg(a.grav + base + (int64_t)t * sa);
      }
      // 2. characteristic distances of cell t (inteuler.F:197-208)
      Prep prC = prB;
      if (t >= is - 1 && t <= ie + 1) prC = cell_prep(nq[VD], nq[VP], nq[VU], a.coef[t].dx2i, P);
      // 3-4. slope and left edge of cell t-1 (intvar.F:82-102)
      double dqN[6], qlN[6];
#pragma unroll
      for (int v = 0; v < 6; ++v) dqN[v] = qlN[v] = 0.0;
      {
        const int c = t - 1;
        if (c >= is - 2 && c <= ie + 2) {
          const Coef cf = a.coef[c];
#pragma unroll
          for (int v = 0; v < NV; ++v) dqN[v] = pm_slope(wq1[v], wq2[v], nq[v], cf.c1, cf.c2);
          if (c >= is - 1) {
#pragma unroll
            for (int v = 0; v < NV; ++v)
              qlN[v] = pm_edge(wq1[v], wq2[v], dqm1[v], dqN[v], cf.c3, cf.c4, cf.c5, cf.c6);
          }
        }
      }
      // 5. parabola of cell t-2 and its face contributions
      Lside Ln = Lp;
      Rside Rc = {};
      bool have_R = false;
      {
        const int c = t - 2;
        if (c >= is - 1 && c <= ie + 1) {
          Para pa[6];
#pragma unroll
          for (int v = 0; v < 6; ++v) pa[v] = Para{0.0, 0.0, 0.0, 0.0};
#pragma unroll
          for (int v = 0; v < NV; ++v) pa[v] = pm_parabola(wq0[v], wq1[v], wq2[v], qlm1[v], qlN[v]);
          if (c <= ie) Ln = make_left<DUAL>(pa, prA);
          if (c >= is) {
            Rc = make_right<DUAL>(pa, prA);
            have_R = true;
          }
        }
      }
      // 6. face f = t-2: corrected states, Riemann problem, Godunov flux
      Flux Fn = Fp;
      {
        const int f = t - 2;
        if (have_R && f <= ie + 1) {
          const double gsum = GRAV ? (wg0 + wg1) : 0.0;
          FaceState s = face_assemble<DUAL, GRAV>(Lp, Rc, wq0[VU], wq1[VU], gsum, P);
          double cl = sqrt(P.gamma * s.pl * s.dl);
          double cr = sqrt(P.gamma * s.pr * s.dr);
          double ps = acoustic_guess(s, cl, cr, P);
          Riemann rs = twoshock_newton(s, cl, cr, ps, P);
          c_if += 1;
          c_newton += rs.iters;
          c_hist[rs.iters & 7] += 1;
          const double qc = P.dt / a.coef[f].dx;
          Fn = flux_twoshock<DUAL>(s, rs.pbar, rs.ubar, qc, P);
        }
      }
      // 7. cell c = t-3: negative-state check, HLL fallback, conservative update
      Cell PEn = PEp;
      bool gov_next = false;
      double govv_next = 0.0;
      {
        const int c = t - 3;
        if (c >= 0 && c < n) {
          Cell cell;
          cell.d = wq0[VD];
          cell.e = we0;
          cell.u = wq0[VU];
          cell.v = wq0[VV];
          cell.w = wq0[VW];
          cell.ge = DUAL ? wq0[VGE] : 0.0;
          if (c >= is && c <= ie) {
            const double qcc = P.dt / a.coef[c].dx;
            double ges = 0.0;
            if (DUAL) {
              double pcent = dmax(P.gm1 * cell.ge * cell.d, kTiny);
              ges = gov ? govv : qcc * pcent * (Fp.ub - Fn.ub);
            }
            bool fatal = false;
            if (cell.d + (Fp.df - Fn.df) <= 0.0 || cell.e < 0.0) {
              if (a.fallback == 0) {
                fatal = true;
              } else {
                // flux_hll for this cell (faces c, c+1; face c+2 feeds ges(c+1))
                c_fb += 1;
                FaceState s0 = rebuild_face<DUAL, GRAV>(a, base, c, P);
                FaceState s1 = rebuild_face<DUAL, GRAV>(a, base, c + 1, P);
                HllFace h0 = hll_face<DUAL>(s0, P);
                HllFace h1 = hll_face<DUAL>(s1, P);
                HllFace h2 = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
                if (c + 2 <= ie + 1) {
                  FaceState s2 = rebuild_face<DUAL, GRAV>(a, base, c + 2, P);
                  h2 = hll_face<DUAL>(s2, P);
                }
                const double qc1 = P.dt / a.coef[c + 1].dx;
                if (DUAL) {
                  double pc0 = dmax(P.gm1 * cell.ge * cell.d, kTiny);
                  double pc1 = dmax(P.gm1 * wq1[VGE] * wq1[VD], kTiny);
                  ges = qcc * pc0 * (h0.sl * h0.gesl + h0.sr * h0.gesr - h1.sl * h1.gesl - h1.sr * h1.gesr);
                  gov_next = true;
                  govv_next = qc1 * pc1 * (h1.sl * h1.gesl + h1.sr * h1.gesr - h2.sl * h2.gesl - h2.sr * h2.gesr);
                }
                Fp.df = qcc * h0.df; Fp.uf = qcc * h0.uf; Fp.vf = qcc * h0.vf;
                Fp.wf = qcc * h0.wf; Fp.ef = qcc * h0.ef;
                Fp.gef = DUAL ? P.dt / a.coef[c].dx * h0.gef : 0.0;
                Fn.df = qc1 * h1.df; Fn.uf = qc1 * h1.uf; Fn.vf = qc1 * h1.vf;
                Fn.wf = qc1 * h1.wf; Fn.ef = qc1 * h1.ef;
                Fn.gef = DUAL ? P.dt / a.coef[c + 1].dx * h1.gef : 0.0;
                if (cell.d + Fp.df - Fn.df <= 0.0) fatal = true;
              }
            }
            PEn = euler_update<DUAL, GRAV>(cell, Fp, Fn, ges, wg0, P, fatal);
            if (fatal) c_fatal += 1;
            // subgrid flux capture: faces are final once their right cell is checked
            while (cap < cap_end && a.captures[cap].face <= c + (c == ie ? 1 : 0)) {
              const FluxCapture& rq = a.captures[cap];
              const Flux& F = (rq.face == c) ? Fp : Fn;
              double* dst = a.capture_buf + rq.dst;
              dst[0] = F.df; dst[1] = F.ef; dst[2] = F.uf;
              dst[3] = F.vf; dst[4] = F.wf; dst[5] = F.gef;
              ++cap;
            }
          } else {
            PEn = cell;
          }
        }
      }
      // 8. cell c' = t-4: dual-energy select (pgas2d_dual) and store
      double dep_next = dep;
      {
        const int c = t - 4;
        if (c >= 0) {
          Cell o = PEp;
          if (DUAL) {
            const double own = o.d * o.e;
            const double de_m = (c == 0) ? own : dep;
            const double de_p = (c == n - 1) ? own : PEn.d * PEn.e;
            pgas2d_dual(o, de_m, de_p, P);
            dep_next = o.d * o.e;
          }
          if (!isfinite(o.d) || !isfinite(o.e)) c_nonfin += 1;
          const int64_t off = base + (int64_t)c * sa;
          a.out_d[off] = o.d;
          a.out_e[off] = o.e;
          if (a.out_u) a.out_u[off] = o.u;
          if (a.out_v) a.out_v[off] = o.v;
          if (a.out_w) a.out_w[off] = o.w;
          if (DUAL) a.out_ge[off] = o.ge;
        }
      }
      // 9. advance the pipeline
#pragma unroll
      for (int v = 0; v < 6; ++v) {
        wq0[v] = wq1[v];
        wq1[v] = wq2[v];
        wq2[v] = nq[v];
        dqm1[v] = dqN[v];
        qlm1[v] = qlN[v];
      }
      we0 = we1; we1 = we2; we2 = ne;
      wg0 = wg1; wg1 = wg2; wg2 = ng;
      prA = prB;
      prB = prC;
      Lp = Ln;
      Fp = Fn;
      gov = gov_next;
      govv = govv_next;
      PEp = PEn;
      dep = dep_next;
    }
    atomicAdd(&s_cnt[kCntInterfaces], (unsigned long long)c_if);
    atomicAdd(&s_cnt[kCntNewton], (unsigned long long)c_newton);
#pragma unroll
    for (int h = 0; h < 8; ++h)
      if (c_hist[h]) atomicAdd(&s_cnt[kCntHist0 + h], (unsigned long long)c_hist[h]);
    if (c_fb) atomicAdd(&s_cnt[kCntFallbacks], (unsigned long long)c_fb);
    if (c_fatal) atomicAdd(&s_cnt[kCntFatal], (unsigned long long)c_fatal);
    if (c_nonfin) atomicAdd(&s_cnt[kCntNonFinite], (unsigned long long)c_nonfin);
  }
  __syncthreads();
  if (threadIdx.x < kMaxCounters && s_cnt[threadIdx.x] != 0ull)
    atomicAdd(&a.counters[threadIdx.x], s_cnt[threadIdx.x]);
}

// ------------------------------------------------------------------ ComputePressure
struct PressureArgs {
  const double* d;
  const double* te;
  const double* v1;
  const double* v2;   // null when MaxVelocityIndex < 2
  const double* v3;   // null when MaxVelocityIndex < 3
  const double* ge;   // non-null selects the dual-energy branch
  double* p;
  int64_t size;
  double gamma, tiny_number, min_support;
};

__global__ void __launch_bounds__(256) pressure_kernel(const __grid_constant__ PressureArgs a) {
  const double gm1 = a.gamma - 1.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.size;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double density = __ldg(a.d + i);
    double gas_energy;
    if (a.ge) {
      gas_energy = __ldg(a.ge + i);
    } else {
      const double velocity1 = __ldg(a.v1 + i);
      const double velocity2 = a.v2 ? __ldg(a.v2 + i) : 0.0;
      const double velocity3 = a.v3 ? __ldg(a.v3 + i) : 0.0;
      gas_energy = __ldg(a.te + i) -
                   0.5 * (velocity1 * velocity1 + velocity2 * velocity2 + velocity3 * velocity3);
    }
    double p = gm1 * density * gas_energy;
    if (p < a.tiny_number) p = a.tiny_number;
    const double min_pressure = a.min_support * gm1 * density * density;
    if (p < min_pressure) p = min_pressure;
    a.p[i] = p;
  }
}

// ------------------------------------------------------------------ calc_dt (ihydro 0)
struct TimestepArgs {
  const double* d;
  const double* te;
  const double* v[3];
  const double* ge;
  int rank;
  int dims[3], start[3], end[3];
  double gamma, tiny_number, min_support;
  double aye, vg[3];
  const double* cw[3];                  // device copies of the cell widths
  unsigned long long* min_bits;         // running minimum of dt1 (positive doubles order as integers)
};

__global__ void __launch_bounds__(256) timestep_kernel(const __grid_constant__ TimestepArgs a) {
  const int nx = a.end[0] - a.start[0] + 1;
  const int ny = a.rank > 1 ? a.end[1] - a.start[1] + 1 : 1;
  const int nz = a.rank > 2 ? a.end[2] - a.start[2] + 1 : 1;
  const int64_t total = (int64_t)nx * ny * nz;
  const double gm1 = a.gamma - 1.0;
  double best = 1.0e20;  // calc_dt.F:71 (huge)
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < total;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int i = a.start[0] + (int)(c % nx);
    const int j = (a.rank > 1 ? a.start[1] : 0) + (int)((c / nx) % ny);
    const int k = (a.rank > 2 ? a.start[2] : 0) + (int)(c / ((int64_t)nx * ny));
    const int64_t g = ((int64_t)k * a.dims[1] + j) * a.dims[0] + i;
    // grid::ComputePressure (Grid_ComputePressure.C:96-164)
    const double density = __ldg(a.d + g);
    const double u = __ldg(a.v[0] + g);
    const double v = a.v[1] ? __ldg(a.v[1] + g) : 0.0;
    const double w = a.v[2] ? __ldg(a.v[2] + g) : 0.0;
    double gas_energy;
    if (a.ge) gas_energy = __ldg(a.ge + g);
    else gas_energy = __ldg(a.te + g) - 0.5 * (u * u + v * v + w * w);
    double p = gm1 * density * gas_energy;
    if (p < a.tiny_number) p = a.tiny_number;
    const double min_pressure = a.min_support * gm1 * density * density;
    if (p < min_pressure) p = min_pressure;
    // calc_dt.F:136-153
    const double cs = dmax(sqrt(a.gamma * p / density), kTiny);
    double dt1;
    if (a.rank == 1) {
      dt1 = a.cw[0][i] * a.aye / (cs + fabs(u - a.vg[0]));
    } else if (a.rank == 2) {
      dt1 = a.aye / ((cs + fabs(u - a.vg[0])) / a.cw[0][i] + (cs + fabs(v - a.vg[1])) / a.cw[1][j]);
    } else {
      dt1 = a.aye / ((cs + fabs(u - a.vg[0])) / a.cw[0][i] + (cs + fabs(v - a.vg[1])) / a.cw[1][j] +
                     (cs + fabs(w - a.vg[2])) / a.cw[2][k]);
    }
    best = dmin(best, dt1);
  }
  // warp then block min
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = dmin(best, __shfl_xor_sync(0xffffffffu, best, o));
  __shared__ double s_min[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) s_min[wid] = best;
  __syncthreads();
  if (wid == 0) {
    best = lane < (int)(blockDim.x >> 5) ? s_min[lane] : 1.0e20;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = dmin(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) atomicMin(a.min_bits, (unsigned long long)__double_as_longlong(best));
  }
}

// min_bits starts as all ones (set by a memset); every block has folded in a value <= huge.
__global__ void timestep_finalize_kernel(const unsigned long long* min_bits, double courant,
                                         double* dt_out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const unsigned long long b = *min_bits;
    double dt = (b == ~0ull) ? 1.0e20 : __longlong_as_double((long long)b);
    dt_out[0] = dt * courant;  // dtBaryons *= CourantSafetyNumber (Grid_ComputeTimeStep.C:209)
  }
}

// ------------------------------------------------------------------ ghost-zone fill
struct BoundaryArgs {
  double* f[8];
  int nf;
  int dims[3], start[3], end[3];
  int bc[3];  // 0 periodic, 1 outflow
  int64_t nghost_cells;
};

__device__ __forceinline__ int bc_map(int i, int s, int e, int bc) {
  if (i >= s && i <= e) return i;
  if (bc == 0) {
    const int nn = e - s + 1;
    int r = (i - s) % nn;
    if (r < 0) r += nn;
    return s + r;
  }
  return i < s ? s : e;
}

// One thread per cell of the padded grid; active cells return immediately.
__global__ void __launch_bounds__(256) boundary_kernel(const __grid_constant__ BoundaryArgs a) {
  const int64_t total = (int64_t)a.dims[0] * a.dims[1] * a.dims[2];
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(g % a.dims[0]);
    const int j = (int)((g / a.dims[0]) % a.dims[1]);
    const int k = (int)(g / ((int64_t)a.dims[0] * a.dims[1]));
    const int si = a.dims[0] > 1 ? bc_map(i, a.start[0], a.end[0], a.bc[0]) : i;
    const int sj = a.dims[1] > 1 ? bc_map(j, a.start[1], a.end[1], a.bc[1]) : j;
    const int sk = a.dims[2] > 1 ? bc_map(k, a.start[2], a.end[2], a.bc[2]) : k;
    if (si == i && sj == j && sk == k) continue;
    const int64_t src = ((int64_t)sk * a.dims[1] + sj) * a.dims[0] + si;
    for (int n = 0; n < a.nf; ++n) a.f[n][g] = a.f[n][src];
  }
}

// ------------------------------------------------------------------ launchers
void launch_sweep(const SweepArgs& a, bool dual, bool grav, cudaStream_t st) {
  const int threads = 128;
  const int64_t blocks = (a.npencils + threads - 1) / threads;
  if (dual && grav) sweep_kernel<true, true><<<(unsigned)blocks, threads, 0, st>>>(a);
  else if (dual) sweep_kernel<true, false><<<(unsigned)blocks, threads, 0, st>>>(a);
  else if (grav) sweep_kernel<false, true><<<(unsigned)blocks, threads, 0, st>>>(a);
  else sweep_kernel<false, false><<<(unsigned)blocks, threads, 0, st>>>(a);
}

static unsigned grid_for(int64_t n, int threads, int sms) {
  int64_t b = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)sms * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

void launch_pressure(const PressureArgs& a, int sms, cudaStream_t st) {
  pressure_kernel<<<grid_for(a.size, 256, sms), 256, 0, st>>>(a);
}

void launch_timestep(const TimestepArgs& a, double courant, double* dt_out, int sms,
                     cudaStream_t st) {
  const int64_t nx = a.end[0] - a.start[0] + 1;
  const int64_t ny = a.rank > 1 ? a.end[1] - a.start[1] + 1 : 1;
  const int64_t nz = a.rank > 2 ? a.end[2] - a.start[2] + 1 : 1;
  timestep_kernel<<<grid_for(nx * ny * nz, 256, sms), 256, 0, st>>>(a);
  timestep_finalize_kernel<<<1, 32, 0, st>>>(a.min_bits, courant, dt_out);
}

void launch_boundary(const BoundaryArgs& a, int sms, cudaStream_t st) {
  const int64_t total = (int64_t)a.dims[0] * a.dims[1] * a.dims[2];
  boundary_kernel<<<grid_for(total, 256, sms), 256, 0, st>>>(a);
}


// Plain-parameter entry points used by the C ABI layer.
void launch_pressure_plain(const double* d, const double* te, const double* v1, const double* v2,
                           const double* v3, const double* ge, double* p, int64_t size,
                           double gamma, double tiny_number, double min_support, int sms,
                           cudaStream_t st) {
  PressureArgs a;
  a.d = d; a.te = te; a.v1 = v1; a.v2 = v2; a.v3 = v3; a.ge = ge; a.p = p; a.size = size;
  a.gamma = gamma; a.tiny_number = tiny_number; a.min_support = min_support;
  launch_pressure(a, sms, st);
}

void launch_timestep_plain(const double* d, const double* te, const double* const v[3],
                           const double* ge, int rank, const int dims[3], const int start[3],
                           const int end[3], double gamma, double tiny_number, double min_support,
                           double aye, const double vg[3], const double* const cw[3],
                           unsigned long long* min_bits, double courant, double* dt_out, int sms,
                           cudaStream_t st) {
  TimestepArgs a;
  a.d = d; a.te = te; a.ge = ge; a.rank = rank;
  for (int k = 0; k < 3; ++k) {
    a.v[k] = v[k]; a.dims[k] = dims[k]; a.start[k] = start[k]; a.end[k] = end[k];
    a.vg[k] = vg[k]; a.cw[k] = cw[k];
  }
  a.gamma = gamma; a.tiny_number = tiny_number; a.min_support = min_support; a.aye = aye;
  a.min_bits = min_bits;
  cudaMemsetAsync(min_bits, 0xFF, sizeof(unsigned long long), st);
  launch_timestep(a, courant, dt_out, sms, st);
}

void launch_boundary_plain(double* const* f, int nf, const int dims[3], const int start[3],
                           const int end[3], const int bc[3], int sms, cudaStream_t st) {
  BoundaryArgs a;
  a.nf = nf;
  for (int k = 0; k < 8; ++k) a.f[k] = k < nf ? f[k] : nullptr;
  for (int k = 0; k < 3; ++k) {
    a.dims[k] = dims[k]; a.start[k] = start[k]; a.end[k] = end[k]; a.bc[k] = bc[k];
  }
  a.nghost_cells = 0;
  launch_boundary(a, sms, st);
}

}  // namespace ppm
