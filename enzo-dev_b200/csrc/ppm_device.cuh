// ppm_device.cuh -- per-point FP64 physics of the PPM-DE sweep, as device functions.
//
// Each function is one stencil point of a reference Fortran loop, written with the
// reference's operand order (left-to-right association, x**2 = x*x, x**3 = (x*x)*x,
// MAX/MIN as a compare-select).  The exact build of the library is compiled with
// -fmad=false, so every product and sum is rounded separately, and CUDA's FP64 '/' and
// sqrt are IEEE correctly rounded: the results are bit-identical to a plain x86-64
// build of the same expressions.  The tolerance-mode build (-fmad=true,
// PPM_FAST_ALGEBRA) fuses multiply-adds and shares a few divisions; its results are
// held to the oracle within a stated tolerance instead.  The sweep kernels
// (ppm_split.cu) only schedule these points.
#pragma once

#include <cstdint>

#include "ppm_fastmath.cuh"

// PPM_NEWTON_RSQRT: the tolerance build's Newton update from 1/sqrt of the shock factors
// (one reciprocal square root each instead of a square root plus a shared reciprocal;
// Riemann stage 0.77 -> 0.74 ms per 256^3 sweep)
#ifndef PPM_NEWTON_RSQRT
#define PPM_NEWTON_RSQRT 1
#endif

// PPM_FAST_ALGEBRA (the tolerance-mode build): a few quotients with a shared divisor
// are formed from one reciprocal, and the divisions and square roots of the
// reconstruction, the Riemann solvers and the update (not calc_dt's) go through qrcp /
// qdiv / qsqrt / qrsqrt (ppm_fastmath.cuh; the IEEE operations in the exact build);
// everything else is the reference's expression.

namespace ppm {

constexpr double kTiny = 1.0e-20;        // fortran_types.def: tiny (CONFIG_PFLOAT_8)
constexpr double kFt = 4.0 / 3.0;        // intvar.F:62, inteuler.F:127
constexpr double kTolerance = 1.0e-14;   // twoshock.F:97-100 (CONFIG_BFLOAT_8)
constexpr int kNumIter = 8;              // twoshock.F:105-106

__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
// Fortran MAX/MIN as gfortran lowers them without -ffinite-math-only: the first argument
// unless a later one compares greater (smaller) or the first is NaN, so a NaN argument
// after the first is ignored.  Used where a NaN is routine: calcdiss type 2's
// (p(i+1)-p(i-1))/(p(i+2)-p(i-2)) is 0/0 wherever the pressure is uniform.
__device__ __forceinline__ double dmax_g(double a, double b) { return (b > a || isnan(a)) ? b : a; }
__device__ __forceinline__ double dmin_g(double a, double b) { return (b < a || isnan(a)) ? b : a; }

struct Phys {
  double gamma, dt, eta1, eta2, small_rho, pmin;
  double qa;      // (gamma + 1)/(2 gamma)   twoshock.F:115, flux_twoshock.F:73
  double gp1;     // gamma + 1
  double gm1;     // gamma - 1
};

// ---------------------------------------------------------------- inteuler.F:197-208
struct Prep {
  double char1, char2, cm, c0, cp;
};

// PF: PressureFree, the sound speed set to tiny (inteuler.F:199)
template <bool PF = false>
__device__ __forceinline__ Prep cell_prep(double d, double p, double u, double dx2i,
                                          const Phys& P) {
  Prep r;
  double cs = qsqrt(qdiv(P.gamma * p, d));
  if (PF) cs = kTiny;
  r.char1 = dmax(0.0, P.dt * (u + cs)) * dx2i;
  r.char2 = dmax(0.0, -(P.dt * (u - cs))) * dx2i;
  r.cm = P.dt * (u - cs) * dx2i;
  r.c0 = P.dt * (u) * dx2i;
  r.cp = P.dt * (u + cs) * dx2i;
  return r;
}

// ---------------------------------------------------------------- intvar.F:82-94
__device__ __forceinline__ double pm_slope(double qm, double q0, double qp, double c1, double c2) {
  double qplus = qp - q0;
  double qmnus = q0 - qm;
  double qcent = c1 * qplus + c2 * qmnus;
  double qvanl = qdiv(2.0 * qplus * qmnus, qmnus + qplus);
  double temp1 = dmin(dmin(dmin(fabs(qcent), fabs(qvanl)), 2.0 * fabs(qmnus)), 2.0 * fabs(qplus));
  double r = temp1 * copysign(1.0, qcent);
  return (qplus * qmnus > 0.0) ? r : 0.0;
}

// ---------------------------------------------------------------- intvar.F:98-102
__device__ __forceinline__ double pm_edge(double qm, double q0, double dqm, double dq0, double c3,
                                          double c4, double c5, double c6) {
  return c3 * qm + c4 * q0 + c5 * dqm + c6 * dq0;
}

// ------------------------------------------------ calcdiss.F: flattening coefficients
// Per cell j of a pencil, from the cells j-2 .. j+2 (index 2 = cell j); the sweep's
// pressure, velocity, density and total energy.
constexpr double kCdEpsilon = 0.33, kCdKappa1 = 2.0, kCdKappa2 = 0.01, kCdOmega1 = 0.75,
                 kCdOmega2 = 10.0, kCdSigma1 = 0.5, kCdSigma2 = 1.0;  // calcdiss.F:143-149

// eq. A1, calcdiss.F:213-224: a shock at j (pressure jump above epsilon, compression)
__device__ __forceinline__ double cd_wflag(double pm1, double pp1, double um1, double up1) {
  const double qb = fabs(pp1 - pm1) / dmin(pp1, pm1);
  return (qb > kCdEpsilon && um1 > up1) ? 1.0 : 0.0;
}

// type 1, calcdiss.F:409-424 (before the max of eq. A2)
__device__ __forceinline__ double cd_ftemp1(const double p[5], double wflag) {
  double qa;
  if (fabs(p[4] - p[0]) / dmin(p[4], p[0]) < kCdEpsilon)
    qa = 1.0;
  else
    qa = (p[3] - p[1]) / (p[4] - p[0]);
  const double f = dmin(1.0, (qa - kCdOmega1) * kCdOmega2 * wflag);
  return dmax(0.0, f);
}

// type 2, calcdiss.F:447-478 (before the max of eq. A6): d, p at j-2 .. j+2
__device__ __forceinline__ double cd_ftemp2(const double d[5], const double p[5], double wflag,
                                            double gamma) {
  const double dp1 = p[3] - p[1];
  // is = j + sign(2, dp1)
  const bool neg = signbit(dp1);
  const double p_is = neg ? p[0] : p[4], d_is = neg ? d[0] : d[4];
  const double omega = dmax_g(0.0, kCdOmega1 * (kCdOmega2 - dp1 / (p[4] - p[0])));
  const double di2p = 1.0 / d[4], di2m = 1.0 / d[0];
  const double Z = sqrt((dmax_g(p[4], p[0]) + 0.5 * (p[4] + p[0]) * (gamma - 1.0)) /
                        dmax_g(di2p, di2m));
  const double kappa_tilde = (Z + sqrt(gamma * p_is * d_is)) / Z;
  const double kappa = dmax_g(0.0, (kappa_tilde - kCdKappa1) / (kappa_tilde + kCdKappa2));
  return dmin_g(wflag * omega, kappa);
}

// type 3, calcdiss.F:486-555 (before the max of eq. A2): d, e, u, p at j-2 .. j+2
__device__ __forceinline__ double cd_ftemp3(const double d[5], const double e[5],
                                            const double u[5], const double p[5], double wflag,
                                            double gamma) {
  const double dp1 = p[3] - p[1];
  const double dp2 = p[4] - p[0];
  const double de1 = e[3] - e[1];
  const double de2 = e[4] - e[0];
  double dpp = 0.0, dee = 0.0;
  if (dp2 != 0.0) dpp = dp1 / dp2;
  if (de2 != 0.0) dee = de1 / de2;
  const double omega_tilde = dmax(dpp, dee);
  // ism = j + sign(2, dp1) (post-shock), isp = j - sign(2, dp1) (upstream)
  const bool neg = signbit(dp1);
  const double d_ism = neg ? d[0] : d[4], u_ism = neg ? u[0] : u[4];
  const double d_isp = neg ? d[4] : d[0], u_isp = neg ? u[4] : u[0], p_isp = neg ? p[4] : p[0];
  double s = -copysign(1.0, dp1);
  if (dp1 == 0.0) s = 0.0;
  const double sigma_tilde = wflag * fabs(dp2) / dmin(p[4], p[0]);
  const double sigma = dmax(0.0, (sigma_tilde - kCdSigma1) / (sigma_tilde + kCdSigma2));
  const double omega = dmax(0.0, kCdOmega2 * (omega_tilde - kCdOmega1));
  const double di2p = 1.0 / d[4], di2m = 1.0 / d[0];
  const double Z = sqrt((dmax(p[4], p[0]) + 0.5 * (p[4] + p[0]) * (gamma - 1.0)) /
                        dmax(di2p, di2m));
  const double ZE = s * Z / d_ism + u_ism + kTiny;
  const double cj2s = sqrt(gamma * p_isp / d_isp);
  const double kappa_tilde = fabs((ZE - u_isp + s * cj2s) / ZE);
  const double kappa = dmax(0.0, (kappa_tilde - kCdKappa1) / (kappa_tilde + kCdKappa2));
  return dmin(dmin(kappa, wflag * omega), wflag * sigma);
}

// inteuler.F:166-193: the density steepening coefficient of cell j from d and the cell
// widths at j-2 .. j+2 (index 2 = cell j) and p at j-1, j+1
__device__ __forceinline__ double st_d2d(const double* d, const double* dx) {
  // d2d of the middle one of three consecutive cells
  const double qa = dx[0] + dx[1] + dx[2];
  double r = (d[2] - d[1]) / (dx[2] + dx[1]);
  r = (r - (d[1] - d[0]) / (dx[1] + dx[0])) / qa;
  return r;
}
__device__ __forceinline__ double steepen_coef(const double d[5], const double dx[5], double pm1,
                                               double pp1, double gamma) {
  const double d2m = st_d2d(d, dx);          // d2d(j-1)
  const double d2p = st_d2d(d + 2, dx + 2);  // d2d(j+1)
  const double bm = 0.5 * (dx[1] + dx[2]);   // dxb(j-1)
  const double b0 = 0.5 * (dx[2] + dx[3]);   // dxb(j)
  const double qc = fabs(d[3] - d[1]) - 0.01 * dmin(fabs(d[3]), fabs(d[1]));
  double s1 = (d2m - d2p) * (bm * bm * bm + b0 * b0 * b0) / ((b0 + bm) * (d[3] - d[1] + kTiny));
  if (d2p * d2m > 0.0) s1 = 0.0;
  if (qc <= 0.0) s1 = 0.0;
  const double s2 = dmax(0.0, dmin(20.0 * (s1 - 0.05), 1.0));
  const double qa = fabs(d[3] - d[1]) / dmin(d[3], d[1]);
  const double qb = fabs(pp1 - pm1) / dmin(pp1, pm1);
  return (gamma * 0.1 * qa >= qb) ? s2 : 0.0;
}

// ---------------------------------------------------------------- intvar.F:106-160
// The parabola of one cell from its edge values.  STEEP (density only): steepening
// toward the neighbours' linear profiles with coefficient st (intvar.F:106-113; dqm, dqp:
// the neighbours' slopes); FLAT: flattening toward the cell value with coefficient fl
// (intvar.F:135-140).  Without them this is the plain PPM parabola.
struct Para {
  double ql, qr, q6, dq;
};

template <bool STEEP = false, bool FLAT = false>
__device__ __forceinline__ Para pm_parabola(double qm, double q0, double qp, double ql, double qr,
                                            double st = 0.0, double dqm = 0.0,
                                            double dqp = 0.0, double fl = 0.0) {
  if (STEEP) {
    ql = (1.0 - st) * ql + st * (qm + 0.5 * dqm);
    qr = (1.0 - st) * qr + st * (qp - 0.5 * dqp);
  }
  double temp1 = (qr - q0) * (q0 - ql);
  double temp2 = qr - ql;
  double temp3 = 6.0 * (q0 - 0.5 * (qr + ql));
  if (temp1 <= 0.0) {
    ql = q0;
    qr = q0;
  }
  double temp22 = temp2 * temp2;
  double temp23 = temp2 * temp3;
  if (temp22 < temp23) ql = 3.0 * q0 - 2.0 * qr;
  if (temp22 < -temp23) qr = 3.0 * q0 - 2.0 * ql;
  if (FLAT) {
    ql = q0 * fl + ql * (1.0 - fl);
    qr = q0 * fl + qr * (1.0 - fl);
  }
  // CHECK_LR, intvar.F:145-153
  ql = dmax(dmin(q0, qm), ql);
  ql = dmin(dmax(q0, qm), ql);
  qr = dmax(dmin(q0, qp), qr);
  qr = dmin(dmax(q0, qp), qr);
  Para r;
  r.q6 = 6.0 * (q0 - 0.5 * (ql + qr));
  r.dq = qr - ql;
  r.ql = ql;
  r.qr = qr;
  return r;
}

// characteristic averages, intvar.F:162-174 and inteuler.F:304-316
// A: qla (x = char1), ql0 (c0), plm/ulm (cm), plp/ulp (cp) from the cell left of a face
__device__ __forceinline__ double pm_A(const Para& a, double x) {
  return a.qr - x * (a.dq - (1.0 - kFt * x) * a.q6);
}
// B: qr0 (c0), prm/urm (cm), prp/urp (cp) from the cell right of a face
__device__ __forceinline__ double pm_B(const Para& a, double x) {
  return a.ql - x * (a.dq + (1.0 + kFt * x) * a.q6);
}
// C: qra (x = char2)
__device__ __forceinline__ double pm_C(const Para& a, double x) {
  return a.ql + x * (a.dq + (1.0 - kFt * x) * a.q6);
}

struct FaceState {
  double dl, dr, pl, pr, ul, ur, vl, vr, wl, wr, gel, ger;
};

// ------------------------------------------------------- inteuler.F:320-551 for one face
// The corrected states of one face split into two independent groups: density,
// pressure and normal velocity (characteristic corrections, dual-energy override,
// floors) and the advected transverse velocities and gas energy (upwind selection).
struct CoreL {
  double dla, dl0, pla, pl0, plm, plp, ula, ul0, ulm, ulp, cm, c0, cp;
};
struct CoreR {
  double dra, dr0, pra, pr0, prm, prp, ura, ur0, urm, urp, cm, c0, cp;
};
struct CoreState {
  double dl, dr, pl, pr, ul, ur;
};
struct AdvL {
  double vla, vl0, wla, wl0, gela, gel0;
};
struct AdvR {
  double vra, vr0, wra, wr0, gera, ger0;
};
struct AdvState {
  double vl, vr, wl, wr, gel, ger;
};

// What the colour states of a face need from its density states (inteuler.F:436-450,
// :500-515): the corrected densities before the dual-energy override and whether the
// override replaced each side.
struct ColFace {
  double dlc, drc;
  bool ovl, ovr;
};

// One side of a face's d, p, u states (inteuler.F:320-410 for the left side, :493-551
// for the right; the two sides share nothing but gsum = grslice(i-1) + grslice(i)).
// qa, q0, qm, qp: the parabola averages over the domains of dependence (char, the
// zero, minus and plus characteristics) of density (a, 0 only), pressure and velocity
// of the cell on this side; cm, c0, cp: the characteristic speeds.  LEFT: a wave enters
// the face from the left where its speed is positive.
struct SideIn {
  double da, d0, pa, p0, pm, pp, ua, u0, um, up, cm, c0, cp;
};
struct SideOut {
  double p, u, d;  // the face state on this side
  double dc;       // the corrected density before the dual-energy override (colours)
  bool ov;         // the override replaced this side
};

template <bool DUAL, bool GRAV, bool LEFT>
__device__ __forceinline__ SideOut face_side(const SideIn& S, double gsum, const Phys& P) {
  SideOut o;
  const double c = qsqrt(dmax(P.gamma * S.pa * S.da, 0.0));
  // 0.5/c is computed as 0.5*(1/c): equal, since c is 0, inf, NaN or a square root of
  // a double (|c| <= 2^512), so 1/c never reaches the subnormal range
  double f1 = qrcp(c);
  const double hc = 0.5 * f1;
  const double yd = qrcp(S.da);
  double bp = (S.ua - S.up) + (S.pa - S.pp) * f1;
  double bm = (S.ua - S.um) - (S.pa - S.pm) * f1;
  double b0 = (S.pa - S.p0) * (f1 * f1) + yd - qrcp(S.d0);
  if (GRAV) {
    const double gterm = 0.25 * P.dt * gsum;
    bp = bp - gterm;
    bm = bm - gterm;
  }
  f1 = hc;
  bp = -(bp * f1);
  bm = +bm * f1;
  if (LEFT ? S.cp <= 0.0 : S.cp >= 0.0) bp = 0.0;
  if (LEFT ? S.cm <= 0.0 : S.cm >= 0.0) bm = 0.0;
  if (LEFT ? S.c0 <= 0.0 : S.c0 >= 0.0) b0 = 0.0;
  o.p = S.pa + (bp + bm) * (c * c);
  o.u = S.ua + (bp - bm) * c;
  o.d = qrcp(yd - (b0 + bp + bm));
  o.dc = o.d;
  o.ov = false;
  if (DUAL) {
    const double m = dmax(dmax(fabs(S.cm), fabs(S.c0)), fabs(S.cp));
#if PPM_FAST_ALGEBRA  // tolerance mode: the quotient by da from its reciprocal
    const bool ov = P.gamma * S.pa * yd < P.eta2 * (S.ua * S.ua) || m < 1.0e-3 ||
                    o.d * yd > 5.0;
#else
    const bool ov = P.gamma * S.pa / S.da < P.eta2 * (S.ua * S.ua) || m < 1.0e-3 ||
                    o.d / S.da > 5.0;
#endif
    if (ov) {
      o.p = S.pa;
      o.u = S.ua;
      o.d = S.da;
      o.ov = true;
    }
  }
  o.p = dmax(o.p, kTiny);
  o.d = dmax(o.d, kTiny);
  return o;
}

__device__ __forceinline__ SideIn side_in(const CoreL& L) {
  return SideIn{L.dla, L.dl0, L.pla, L.pl0, L.plm, L.plp, L.ula, L.ul0, L.ulm, L.ulp,
                L.cm, L.c0, L.cp};
}
__device__ __forceinline__ SideIn side_in(const CoreR& R) {
  return SideIn{R.dra, R.dr0, R.pra, R.pr0, R.prm, R.prp, R.ura, R.ur0, R.urm, R.urp,
                R.cm, R.c0, R.cp};
}

// inteuler.F:320-410, 493-551 (d, p, u) for both sides of a face; gsum = grslice(i-1) +
// grslice(i) (GRAV only).  CX: also report the colour data of the face in *cx.
template <bool DUAL, bool GRAV, bool CX = false>
__device__ __forceinline__ CoreState face_core(const CoreL& L, const CoreR& R, double gsum,
                                               const Phys& P, ColFace* cx = nullptr) {
  const SideOut l = face_side<DUAL, GRAV, true>(side_in(L), gsum, P);
  const SideOut r = face_side<DUAL, GRAV, false>(side_in(R), gsum, P);
  if (CX) {
    cx->dlc = l.dc;
    cx->drc = r.dc;
    cx->ovl = l.ov;
    cx->ovr = r.ov;
  }
  CoreState s;
  s.pl = l.p;
  s.pr = r.p;
  s.ul = l.u;
  s.ur = r.u;
  s.dl = l.d;
  s.dr = r.d;
  return s;
}

// inteuler.F:414-434: ul_cell / ur_cell = uslice(i-1) / uslice(i)
__device__ __forceinline__ AdvState face_advected(const AdvL& L, const AdvR& R, double ul_cell,
                                                  double ur_cell) {
  AdvState s;
  if (ul_cell <= 0.0) {
    s.vl = L.vla; s.wl = L.wla; s.gel = L.gela;
  } else {
    s.vl = L.vl0; s.wl = L.wl0; s.gel = L.gel0;
  }
  if (ur_cell >= 0.0) {
    s.vr = R.vra; s.wr = R.wra; s.ger = R.gera;
  } else {
    s.vr = R.vr0; s.wr = R.wr0; s.ger = R.ger0;
  }
  return s;
}

// ---------------------------------------------- twoshock.F:156-254 for one interface
// The acoustic starting pressure of twoshock.F:156-170, or `guess` when guess > 0.
struct Riemann {
  double pbar, ubar;
  int iters;      // Newton updates performed (1..7)
  bool converged; // reached |dp/p| < tolerance within numiter - 1 updates
};

__device__ __forceinline__ double acoustic_guess(const FaceState& s, double cl, double cr,
                                                 const Phys& P) {
  double ps = qdiv(cr * s.pl + cl * s.pr + cr * cl * (s.ul - s.ur), cr + cl);
  if (ps < P.pmin) ps = P.pmin;
  return ps;
}

__device__ __forceinline__ Riemann twoshock_newton(const FaceState& s, double cl, double cr,
                                                   double ps, const Phys& P) {
  double old_ps = ps, ubl = 0.0, ubr = 0.0, dpdul = 0.0, dpdur = 0.0;
  int it = 0;
  bool active = true;
#if PPM_FAST_ALGEBRA
  // Tolerance-mode build: the same Newton update with the face's reciprocals 1/pl, 1/pr,
  // 1/dl, 1/dr formed once, each pair of quotients with different divisors sharing one
  // division (a/x, b/y = a*y*q, b*x*q with q = 1/(x*y)), and the convergence test as
  // |dp| < tolerance * ps: three divisions per update instead of twelve.
  const double ipl = qrcp(s.pl), ipr = qrcp(s.pr), idl = qrcp(s.dl), idr = qrcp(s.dr);
#if PPM_NEWTON_RSQRT
  // zl = cl sqrt(Xl) from yl = 1/sqrt(Xl): zl = cl Xl yl, 1/zl = yl / cl, zl^2 = cl^2 Xl
  const double icl = qrcp(cl), icr = qrcp(cr), cl2 = cl * cl, cr2 = cr * cr;
#pragma unroll 1
  for (int n = 2; n <= kNumIter; n++) {
    if (active) {
      const double Xl = 1.0 + P.qa * (ps * ipl - 1.0), Xr = 1.0 + P.qa * (ps * ipr - 1.0);
      const double yl = qrsqrt(Xl), yr = qrsqrt(Xr);
      const double zl = cl * (Xl * yl), zr = cr * (Xr * yr);
      ubl = s.ul - (ps - s.pl) * (yl * icl);
      ubr = s.ur + (ps - s.pr) * (yr * icr);
      const double al = 4.0 * (cl2 * Xl) * idl, ar = 4.0 * (cr2 * Xr) * idr;
      const double dl = al - P.gp1 * (ps - s.pl), dr = ar - P.gp1 * (ps - s.pr);
      const double qd = qrcp(dl * dr);
      dpdul = -(zl * al * (dr * qd));
      dpdur = zr * ar * (dl * qd);
      ps = ps + qdiv((ubr - ubl) * dpdur * dpdul, dpdur - dpdul);
      if (ps < P.pmin) ps = P.pmin;
      const double delta_ps = ps - old_ps;
      old_ps = ps;
      it++;
      if (fabs(delta_ps) < kTolerance * ps) active = false;
    }
  }
#else
#pragma unroll 1
  for (int n = 2; n <= kNumIter; n++) {
    if (active) {
      const double zl = cl * qsqrt((1.0 + P.qa * (ps * ipl - 1.0)));
      const double zr = cr * qsqrt((1.0 + P.qa * (ps * ipr - 1.0)));
      const double qz = qrcp(zl * zr);
      ubl = s.ul - (ps - s.pl) * (zr * qz);
      ubr = s.ur + (ps - s.pr) * (zl * qz);
      const double al = 4.0 * (zl * zl) * idl, ar = 4.0 * (zr * zr) * idr;
      const double dl = al - P.gp1 * (ps - s.pl), dr = ar - P.gp1 * (ps - s.pr);
      const double qd = qrcp(dl * dr);
      dpdul = -(zl * al * (dr * qd));
      dpdur = zr * ar * (dl * qd);
      ps = ps + qdiv((ubr - ubl) * dpdur * dpdul, dpdur - dpdul);
      if (ps < P.pmin) ps = P.pmin;
      const double delta_ps = ps - old_ps;
      old_ps = ps;
      it++;
      if (fabs(delta_ps) < kTolerance * ps) active = false;
    }
  }
#endif
#else
#pragma unroll 1
  for (int n = 2; n <= kNumIter; n++) {
    if (active) {
      double zl = cl * sqrt((1.0 + P.qa * (ps / s.pl - 1.0)));
      double zr = cr * sqrt((1.0 + P.qa * (ps / s.pr - 1.0)));
      ubl = s.ul - (ps - s.pl) / zl;
      ubr = s.ur + (ps - s.pr) / zr;
      dpdul = -(4.0 * (zl * zl * zl) / s.dl / (4.0 * (zl * zl) / s.dl - P.gp1 * (ps - s.pl)));
      dpdur = 4.0 * (zr * zr * zr) / s.dr / (4.0 * (zr * zr) / s.dr - P.gp1 * (ps - s.pr));
      ps = ps + (ubr - ubl) * dpdur * dpdul / (dpdur - dpdul);
      if (ps < P.pmin) ps = P.pmin;
      double delta_ps = ps - old_ps;
      old_ps = ps;
      it++;
      if (fabs(delta_ps / ps) < kTolerance) active = false;
    }
  }
#endif
  Riemann r;
  if (ps < P.pmin) ps = dmin(s.pl, s.pr);
  r.pbar = ps;
  r.ubar = ubl + qdiv((ubr - ubl) * dpdur, dpdur - dpdul);
  r.iters = it;
  r.converged = !active;
  return r;
}

// ------------------------------------ flux_twoshock.F:84-396 for one face (RAREFACTION2)
struct Flux {
  double df, ef, uf, vf, wf, gef, ub;
};

// db_out (optional): the Godunov density db, which the colour fluxes scale by
// (flux_twoshock.F:251-259)
template <bool DUAL>
__device__ __forceinline__ Flux flux_twoshock(const FaceState& s, double pbar, double ubar,
                                              double qc, const Phys& P,
                                              double* db_out = nullptr) {
  const double gamma = P.gamma;
  double sn = copysign(1.0, -ubar);
  double u0, p0, d0;
  if (sn < 0.0) {
    u0 = s.ul; p0 = s.pl; d0 = s.dl;
  } else {
    u0 = s.ur; p0 = s.pr; d0 = s.dr;
  }
#if PPM_FAST_ALGEBRA
  // tolerance mode: 1/d0 once, and gamma*pbar/dbar as gamma*pbar*(1/dbar)
  const double id0 = qrcp(d0);
  double c0 = qsqrt(dmax(gamma * p0 * id0, kTiny));
  double z0 = c0 * d0 * qsqrt(dmax(1.0 + P.qa * (qdiv(pbar, p0) - 1.0), kTiny));
  const double idbar = id0 - qdiv(pbar - p0, dmax(z0 * z0, kTiny));
  double dbar = qrcp(idbar);
  double cbar = qsqrt(dmax(gamma * pbar * idbar, kTiny));
  double l0, lbar;
  if (pbar < p0) {
    l0 = u0 * sn + c0;
    lbar = sn * ubar + cbar;
  } else {
    l0 = u0 * sn + z0 * id0;
    lbar = l0;
  }
#else
  double c0 = sqrt(dmax(gamma * p0 / d0, kTiny));
  double z0 = c0 * d0 * sqrt(dmax(1.0 + P.qa * (pbar / p0 - 1.0), kTiny));
  double dbar = 1.0 / (1.0 / d0 - (pbar - p0) / dmax(z0 * z0, kTiny));
  double cbar = sqrt(dmax(gamma * pbar / dbar, kTiny));
  double l0, lbar;
  if (pbar < p0) {
    l0 = u0 * sn + c0;
    lbar = sn * ubar + cbar;
  } else {
    l0 = u0 * sn + z0 / d0;
    lbar = l0;
  }
#endif
  double frac = l0 - lbar;
  if (frac < kTiny) frac = kTiny;
  frac = qdiv(0.0 - lbar, frac);
  frac = dmin(dmax(frac, 0.0), 1.0);
  double pb = p0 * frac + pbar * (1.0 - frac);
  double db = d0 * frac + dbar * (1.0 - frac);
  double ub = u0 * frac + ubar * (1.0 - frac);
  if (lbar >= 0.0) {
    pb = pbar; db = dbar; ub = ubar;
  }
  if (l0 < 0.0) {
    pb = p0; db = d0; ub = u0;
  }
  if (db_out) *db_out = db;
  double vb, wb, geb;
  if (ub > 0.0) {
    vb = s.vl; wb = s.wl; geb = s.gel;
  } else {
    vb = s.vr; wb = s.wr; geb = s.ger;
  }
  double eb = qdiv(pb, P.gm1 * db) + 0.5 * (ub * ub + vb * vb + wb * wb);
  double upb = pb * ub;
  double dub = ub * db;
  double duub = dub * ub;
  double duvb = dub * vb;
  double duwb = dub * wb;
  double dueb = dub * eb;
  Flux f;
  f.df = qc * dub;
  f.ef = qc * (dueb + upb);
  f.uf = qc * (duub + pb);
  f.vf = qc * duvb;
  f.wf = qc * duwb;
  f.gef = DUAL ? qc * (dub * geb) : 0.0;
  f.ub = ub;
  return f;
}

// ------------------------------------------ flux_hll.F:111-258 for one face (no diffusion)
struct HllFace {
  double sl, sr, gesl, gesr;
  double df, uf, vf, wf, ef, gef;  // before the dt/dx factor
};

template <bool DUAL>
__device__ __forceinline__ HllFace hll_face(const FaceState& s, const Phys& P) {
  const double gamma = P.gamma;
  const double gamma1 = gamma - 1.0;
  const double gamma1i = qrcp(gamma1);
  double sqrtdl = qsqrt(s.dl);
  double sqrtdr = qsqrt(s.dr);
  double isdlpdr = qrcp(sqrtdl + sqrtdr);
  double vroe1 = (sqrtdl * s.ul + sqrtdr * s.ur) * isdlpdr;
  double vroe2 = (sqrtdl * s.vl + sqrtdr * s.vr) * isdlpdr;
  double vroe3 = (sqrtdl * s.wl + sqrtdr * s.wr) * isdlpdr;
  double v2 = vroe1 * vroe1 + vroe2 * vroe2 + vroe3 * vroe3;
  double el = gamma1i * s.pl + 0.5 * s.dl * (s.ul * s.ul + s.vl * s.vl + s.wl * s.wl);
  double er = gamma1i * s.pr + 0.5 * s.dr * (s.ur * s.ur + s.vr * s.vr + s.wr * s.wr);
  double hroe = (qdiv(el + s.pl, sqrtdl) + qdiv(er + s.pr, sqrtdr)) * isdlpdr;
  double cs = qsqrt(gamma1 * dmax((hroe - 0.5 * v2), kTiny));
  double char1 = vroe1 - cs;
  double char2 = vroe1 + cs;
  double csl0 = qsqrt(qdiv(gamma * s.pl, s.dl));
  double csr0 = qsqrt(qdiv(gamma * s.pr, s.dr));
  double csl = dmin(s.ul - csl0, char1);
  double csr = dmax(s.ur + csr0, char2);
  double bm = dmin(csl, 0.0);
  double bp = dmax(csr, 0.0);
  double bm0 = s.ul - bm;
  double bp0 = s.ur - bp;
  double q1 = qdiv(bp + bm, bp - bm);
  HllFace h;
  h.sl = 0.5 * (1.0 + q1);
  h.sr = 0.5 * (1.0 - q1);
  h.gesl = bm0;
  h.gesr = bp0;
  double dubl = s.dl * s.ul;
  double dubr = s.dr * s.ur;
  double dfl = s.dl * bm0, dfr = s.dr * bp0;
  double ufl = dubl * bm0 + s.pl, ufr = dubr * bp0 + s.pr;
  double vfl = s.dl * s.vl * bm0, vfr = s.dr * s.vr * bp0;
  double wfl = s.dl * s.wl * bm0, wfr = s.dr * s.wr * bp0;
  double efl = el * bm0 + s.pl * s.ul, efr = er * bp0 + s.pr * s.ur;
  h.df = h.sl * dfl + h.sr * dfr + 0.0;
  h.uf = h.sl * ufl + h.sr * ufr + 0.0;
  h.vf = h.sl * vfl + h.sr * vfr + 0.0;
  h.wf = h.sl * wfl + h.sr * wfr + 0.0;
  h.ef = h.sl * efl + h.sr * efr + 0.0;
  if (DUAL) {
    double gefl = bm0 * s.gel * s.dl;
    double gefr = bp0 * s.ger * s.dr;
    h.gef = h.sl * gefl + h.sr * gefr + 0.0;
  } else {
    h.gef = 0.0;
  }
  return h;
}

// ------------------------------- flux_hllc.F:105-300 for one face (no diffusion, HLLC)
// The HLLC weights sl, sr (the star region's side by the contact speed cw), the advective
// speeds gesl = ul - bm, gesr = ur - bp, and the fluxes before the dt/dx factor with the
// contact's momentum and energy terms (:282-286) included.
template <bool DUAL>
__device__ __forceinline__ HllFace hllc_face(const FaceState& s, const Phys& P) {
  const double gamma = P.gamma;
  const double gamma1 = gamma - 1.0;
  const double gamma1i = qrcp(gamma1);
  double sqrtdl = qsqrt(s.dl);
  double sqrtdr = qsqrt(s.dr);
  double isdlpdr = qrcp(sqrtdl + sqrtdr);
  double vroe1 = (sqrtdl * s.ul + sqrtdr * s.ur) * isdlpdr;
  double vroe2 = (sqrtdl * s.vl + sqrtdr * s.vr) * isdlpdr;
  double vroe3 = (sqrtdl * s.wl + sqrtdr * s.wr) * isdlpdr;
  double v2 = vroe1 * vroe1 + vroe2 * vroe2 + vroe3 * vroe3;
  double el = gamma1i * s.pl + 0.5 * s.dl * (s.ul * s.ul + s.vl * s.vl + s.wl * s.wl);
  double er = gamma1i * s.pr + 0.5 * s.dr * (s.ur * s.ur + s.vr * s.vr + s.wr * s.wr);
  double hroe = (qdiv(el + s.pl, sqrtdl) + qdiv(er + s.pr, sqrtdr)) * isdlpdr;
  double cs = qsqrt(gamma1 * dmax((hroe - 0.5 * v2), kTiny));
  double char1 = vroe1 - cs;
  double char2 = vroe1 + cs;
  double csl0 = qsqrt(qdiv(gamma * s.pl, s.dl));
  double csr0 = qsqrt(qdiv(gamma * s.pr, s.dr));
  double csl = dmin(s.ul - csl0, char1);
  double csr = dmax(s.ur + csr0, char2);
  double bm = dmin(csl, 0.0);
  double bp = dmax(csr, 0.0);
  // contact speed cw and pressure cp (flux_hllc.F:160-183)
  double tl = s.pl - (csl - s.ul) * s.dl * s.ul;
  double tr = s.pr - (csr - s.ur) * s.dr * s.ur;
  double dl = s.dl * (csl - s.ul);
  double dr = -(s.dr * (csr - s.ur));
  double q1 = qrcp(dl + dr);
  double cw = (tr - tl) * q1;
  double cp = (dl * tr + dr * tl) * q1;
  double sl, sr, sm;
  if (cw >= 0.0) {
    sl = qdiv(cw, cw - bm);
    sr = 0.0;
    sm = -qdiv(bm, cw - bm);
  } else {
    sl = 0.0;
    sr = -qdiv(cw, bp - cw);
    sm = qdiv(bp, bp - cw);
  }
  cp = dmax(cp, 0.0);
  const double bm0 = s.ul - bm, bp0 = s.ur - bp;
  double dubl = s.dl * s.ul;
  double dubr = s.dr * s.ur;
  double dfl = dubl - bm * s.dl, dfr = dubr - bp * s.dr;
  double ufl = dubl * bm0 + s.pl, ufr = dubr * bp0 + s.pr;
  double vfl = s.dl * s.vl * bm0, vfr = s.dr * s.vr * bp0;
  double wfl = s.dl * s.wl * bm0, wfr = s.dr * s.wr * bp0;
  double efl = el * bm0 + s.pl * s.ul, efr = er * bp0 + s.pr * s.ur;
  HllFace h;
  h.sl = sl;
  h.sr = sr;
  h.gesl = bm0;
  h.gesr = bp0;
  h.df = sl * dfl + sr * dfr + 0.0;
  h.uf = sl * ufl + sr * ufr + 0.0;
  h.vf = sl * vfl + sr * vfr + 0.0;
  h.wf = sl * wfl + sr * wfr + 0.0;
  h.ef = sl * efl + sr * efr + 0.0;
  if (DUAL) {
    double gefl = bm0 * s.gel * s.dl;
    double gefr = bp0 * s.ger * s.dr;
    h.gef = sl * gefl + sr * gefr + 0.0;
  } else {
    h.gef = 0.0;
  }
  h.uf = h.uf + sm * cp;
  h.ef = h.ef + sm * cp * cw;
  return h;
}

// -------------------------------------------------------------- euler.F:126-279 (one cell)
struct Cell {
  double d, e, u, v, w, ge;
};

template <bool DUAL, bool GRAV>
__device__ __forceinline__ Cell euler_update(const Cell& c, const Flux& F0, const Flux& F1,
                                             double ges, double gr, const Phys& P, bool& fatal) {
  Cell o;
  double dnu = c.d + (F0.df - F1.df);
  double dnuinv = qrcp(dnu);
  if (P.small_rho > 0.0) {
    dnu = dmax(dnu, P.small_rho);
    dnuinv = qrcp(dnu);
  }
  double uold = c.u;
  o.u = (c.u * c.d + (F0.uf - F1.uf)) * dnuinv;
  o.v = (c.v * c.d + (F0.vf - F1.vf)) * dnuinv;
  o.w = (c.w * c.d + (F0.wf - F1.wf)) * dnuinv;
  o.e = dmax(0.1 * c.e, (c.e * c.d + (F0.ef - F1.ef)) * dnuinv);
  if (DUAL) {
    o.ge = dmax((c.ge * c.d + (F0.gef - F1.gef) + ges) * dnuinv, 0.5 * c.ge);
    if (o.ge < 0.0) fatal = true;
  } else {
    o.ge = c.ge;
  }
  if (GRAV) {
    o.u = o.u + P.dt * gr * 0.5 * (c.d * dnuinv + 1.0);
    o.e = o.e + P.dt * gr * 0.5 * (o.u + uold * c.d * dnuinv);
    o.e = dmax(o.e, kTiny);
  }
  o.d = dnu;
  return o;
}

// ----------------------------------------------------- pgas2d_dual.F:70-117 (one cell)
// de_m / de_p: dslice*eslice of the clamped left / right neighbours, the left one
// already rewritten by this routine (the loop is sequential along the pencil).
__device__ __forceinline__ void pgas2d_dual(Cell& c, double de_m, double de_p, const Phys& P) {
  double ke = 0.5 * (c.u * c.u + c.v * c.v + c.w * c.w);
  double ge1 = c.e - ke;
  double demax = dmax(dmax(c.d * c.e, de_m), de_p);
  if (qdiv(ge1 * c.d, demax) > P.eta2) c.ge = ge1;
  double ge2 = (qdiv(ge1, c.e) > P.eta1) ? ge1 : c.ge;
  ge2 = dmax(ge2, qdiv(P.pmin, P.gm1 * c.d));
  c.e = c.e - ge1 + ge2;
}

}  // namespace ppm
