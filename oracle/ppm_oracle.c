/*
 * ppm_oracle.c -- CPU oracle for the PPM-DE hot path (TEST INFRASTRUCTURE ONLY).
 *
 * A plain-C FP64 restatement of Enzo's PPM Direct-Eulerian sweep chain.  Every
 * routine keeps the reference's loop ranges and the operand order of each
 * Fortran expression (left-to-right association, x**2 = x*x, x**3 = (x*x)*x),
 * and the file is built with -ffp-contract=off so no multiply-add is fused.
 * Index helpers are 1-based and column-major, exactly like the Fortran slices
 * (idim, jdim) that the sweep drivers build.
 *
 * Only tests/, the smoke check and the benchmark's CPU-baseline leg use this.
 */
#include "ppm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* fortran_types.def (CONFIG_PFLOAT_8): tiny = 1e-20, huge = 1e20 */
#define F_TINY 1.0e-20
#define F_HUGE 1.0e+20
/* fortran.def:8 and euler.F:104-105 (a Fortran parameter, folded in FP64) */
#define F_COLOR_FLOOR 1.0e-35
static const double F_MIN_COLOR = 1.0e-5 * F_TINY;
/* twoshock.F:97-106 (CONFIG_BFLOAT_8) */
#define TS_TOLERANCE 1.0e-14
#define TS_NUMITER 8

static ora_riemann_log_fn g_log_fn = 0;
static void *g_log_ctx = 0;

void ora_set_riemann_log(ora_riemann_log_fn fn, void *ctx) {
  g_log_fn = fn;
  g_log_ctx = ctx;
}

static inline double fmax2(double a, double b) { return a > b ? a : b; }
static inline double fmin2(double a, double b) { return a < b ? a : b; }
/* Fortran SIGN(1, x): gfortran honours the sign of a signed zero. */
static inline double fsign1(double x) { return copysign(1.0, x); }
/* Fortran MAX/MIN as gfortran lowers them without -ffinite-math-only: the first argument
   unless a later one compares greater (smaller) or the first is NaN, so a NaN argument
   after the first is ignored.  Used where a NaN is routine: calcdiss type 2's
   (p(i+1)-p(i-1))/(p(i+2)-p(i-2)) is 0/0 wherever the pressure is uniform. */
static inline double fmax_g(double a, double b) { return (b > a || isnan(a)) ? b : a; }
static inline double fmin_g(double a, double b) { return (b < a || isnan(a)) ? b : a; }

#define V(a, i) (a)[(i)-1]
#define S(a, i, j) (a)[((size_t)(j)-1) * (size_t)idim + ((size_t)(i)-1)]

/* ------------------------------------------------------------------------ */
/* per-slice workspace                                                       */
/* ------------------------------------------------------------------------ */
typedef struct {
  int idim, jdim;
  /* gathered slice (Grid_xEulerSweep.C:59-133) */
  double *d, *e, *u, *v, *w, *p, *gr, *ge;
  /* slice temporaries (Grid_xEulerSweep.C:137-166) */
  double *dls, *drs, *pbar, *pls, *prs, *ubar, *uls, *urs, *vls, *vrs, *gels, *gers, *wls, *wrs;
  double *df, *ef, *uf, *vf, *wf, *gef, *ges;
  /* 1-D temporaries (the ijkn-sized locals of the Fortran) */
  double *c1, *c2, *c3, *c4, *c5, *c6, *dxdt2, *dx2i;
  double *cs, *char1, *char2, *cm, *c0, *cp;
  double *t1, *t2, *t3, *t4;                       /* d: dq, ql, qr, q6 */
  double *dla, *dra, *dl0, *dr0;
  double *dp, *pl, *pr, *p6, *pla, *pra, *pl0, *pr0;
  double *du, *ul, *ur, *u6, *ula, *ura, *ul0, *ur0;
  double *dv, *vl, *vr, *v6, *vla, *vra, *vl0, *vr0;
  double *dw, *wl, *wr, *w6, *wla, *wra, *wl0, *wr0;
  double *dge, *gel, *ger, *ge6, *gela, *gera, *gel0, *ger0;
  double *plm, *prm, *plp, *prp, *ulm, *urm, *ulp, *urp;
  double *cla, *cra, *betalp, *betalm, *betal0, *betarp, *betarm, *betar0;
  /* twoshock locals */
  double *tcl, *tcr, *dpdul, *dpdur, *ps, *ubl, *ubr, *zl, *zr, *old_ps, *delta_ps;
  int *mask, *niter;
  /* flux_twoshock locals */
  double *sn, *u0, *p0, *d0, *fc0, *z0, *dbar, *cbar, *l0, *lbar, *ub, *vb, *wb, *db, *pb, *eb,
      *geb, *upb, *dub, *duub, *duvb, *duwb, *dueb, *dugeb, *pcent;
  /* flux_hll locals (sized idim+1 so that index i+2 of a single-cell call exists) */
  double *h_sl, *h_sr, *h_gesl, *h_gesr, *h_el, *h_er, *h_bm0, *h_bp0, *h_pcent;
  /* euler locals */
  double *dnu, *dnuinv, *uold;
  /* calcdiss / steepening locals */
  double *flat, *steep, *wflag, *ftemp, *d2d, *dxb;
  double *block;
  /* colours (ncolour > 0): slices colslice/colls/colrs/colf of (idim, jdim, ncolor), and
     the (ijkn, MAX_COLOR) locals of inteuler (dcol coll colr col6 colla colra coll0
     colr0) and flux_twoshock (colb), ncolor columns each */
  int ncol;
  double *col, *colls, *colrs, *colf;
  double *dcol, *coll, *colr, *col6, *colla, *colra, *coll0, *colr0, *colb;
  double *cblock;
} work_t;

static int work_alloc(work_t *W, int idim, int jdim, int ncol) {
  memset(W, 0, sizeof(*W));
  W->idim = idim;
  W->jdim = jdim;
  const size_t ns = (size_t)idim * (size_t)jdim;
  const size_t n1 = (size_t)idim + 4;
#define TAKE(x, n) \
  do {             \
    (x) = b;       \
    b += (n);      \
  } while (0)
  double *b = 0;
  double **one[] = {
      &W->c1, &W->c2, &W->c3, &W->c4, &W->c5, &W->c6, &W->dxdt2, &W->dx2i,
      &W->cs, &W->char1, &W->char2, &W->cm, &W->c0, &W->cp,
      &W->t1, &W->t2, &W->t3, &W->t4, &W->dla, &W->dra, &W->dl0, &W->dr0,
      &W->dp, &W->pl, &W->pr, &W->p6, &W->pla, &W->pra, &W->pl0, &W->pr0,
      &W->du, &W->ul, &W->ur, &W->u6, &W->ula, &W->ura, &W->ul0, &W->ur0,
      &W->dv, &W->vl, &W->vr, &W->v6, &W->vla, &W->vra, &W->vl0, &W->vr0,
      &W->dw, &W->wl, &W->wr, &W->w6, &W->wla, &W->wra, &W->wl0, &W->wr0,
      &W->dge, &W->gel, &W->ger, &W->ge6, &W->gela, &W->gera, &W->gel0, &W->ger0,
      &W->plm, &W->prm, &W->plp, &W->prp, &W->ulm, &W->urm, &W->ulp, &W->urp,
      &W->cla, &W->cra, &W->betalp, &W->betalm, &W->betal0, &W->betarp, &W->betarm, &W->betar0,
      &W->tcl, &W->tcr, &W->dpdul, &W->dpdur, &W->ps, &W->ubl, &W->ubr, &W->zl, &W->zr,
      &W->old_ps, &W->delta_ps,
      &W->sn, &W->u0, &W->p0, &W->d0, &W->fc0, &W->z0, &W->dbar, &W->cbar, &W->l0, &W->lbar,
      &W->ub, &W->vb, &W->wb, &W->db, &W->pb, &W->eb, &W->geb, &W->upb, &W->dub, &W->duub,
      &W->duvb, &W->duwb, &W->dueb, &W->dugeb, &W->pcent,
      &W->h_sl, &W->h_sr, &W->h_gesl, &W->h_gesr, &W->h_el, &W->h_er, &W->h_bm0, &W->h_bp0,
      &W->h_pcent,
      &W->dnu, &W->dnuinv, &W->uold,
      &W->flat, &W->steep, &W->wflag, &W->ftemp, &W->d2d, &W->dxb};
  const size_t n_one = sizeof(one) / sizeof(one[0]);
  /* 29 slice arrays + the 1-D temporaries */
  W->block = (double *)calloc(29 * ns + n_one * n1, sizeof(double));
  W->mask = (int *)calloc(2 * n1, sizeof(int));
  if (!W->block || !W->mask) return -1;
  b = W->block;
  TAKE(W->d, ns); TAKE(W->e, ns); TAKE(W->u, ns); TAKE(W->v, ns); TAKE(W->w, ns);
  TAKE(W->p, ns); TAKE(W->gr, ns); TAKE(W->ge, ns);
  TAKE(W->dls, ns); TAKE(W->drs, ns); TAKE(W->pbar, ns); TAKE(W->pls, ns); TAKE(W->prs, ns);
  TAKE(W->ubar, ns); TAKE(W->uls, ns); TAKE(W->urs, ns); TAKE(W->vls, ns); TAKE(W->vrs, ns);
  TAKE(W->gels, ns); TAKE(W->gers, ns); TAKE(W->wls, ns); TAKE(W->wrs, ns);
  TAKE(W->df, ns); TAKE(W->ef, ns); TAKE(W->uf, ns); TAKE(W->vf, ns); TAKE(W->wf, ns);
  TAKE(W->gef, ns); TAKE(W->ges, ns);
  for (size_t k = 0; k < n_one; ++k) TAKE(*one[k], n1);
#undef TAKE
  W->niter = W->mask + n1;
  W->ncol = ncol;
  if (ncol > 0) {
    const size_t nc = (size_t)ncol;
    W->cblock = (double *)calloc(4 * nc * ns + 9 * nc * n1, sizeof(double));
    if (!W->cblock) return -1;
    double *c = W->cblock;
    double **sl[] = {&W->col, &W->colls, &W->colrs, &W->colf};
    for (int k = 0; k < 4; k++) { *sl[k] = c; c += nc * ns; }
    double **on[] = {&W->dcol, &W->coll, &W->colr, &W->col6, &W->colla, &W->colra,
                     &W->coll0, &W->colr0, &W->colb};
    for (int k = 0; k < 9; k++) { *on[k] = c; c += nc * n1; }
  }
  return 0;
}

static void work_free(work_t *W) {
  free(W->block);
  free(W->mask);
  free(W->cblock);
}

/* colour n's slice and (ijkn) locals */
#define CS(a, i, j, n) (a)[(size_t)(n) * (size_t)idim * (size_t)W->jdim + ((size_t)(j)-1) * (size_t)idim + ((size_t)(i)-1)]
#define CV(a, i, n) (a)[(size_t)(n) * ((size_t)idim + 4) + ((size_t)(i)-1)]

/* ------------------------------------------------------------------------ */
/* intvar.F:5-179 (one pencil)                                               */
/* ------------------------------------------------------------------------ */
static void intvar(const double *q, int idim, int i1, int i2, int isteep,
                   const double *steepen, int iflatten, const double *flatten,
                   const double *c1, const double *c2, const double *c3, const double *c4,
                   const double *c5, const double *c6, const double *char1, const double *char2,
                   const double *c0, double *dq, double *ql, double *qr, double *q6,
                   double *qla, double *qra, double *ql0, double *qr0) {
  const double ft = 4.0 / 3.0;
  int i;
  /* intvar.F:70-73 */
  for (i = 1; i <= idim; i++) { V(dq, i) = 0.0; V(ql, i) = 0.0; V(qr, i) = 0.0; V(q6, i) = 0.0; }
  /* slopes, intvar.F:82-94 */
  for (i = i1 - 2; i <= i2 + 2; i++) {
    double qplus = V(q, i + 1) - V(q, i);
    double qmnus = V(q, i) - V(q, i - 1);
    if (qplus * qmnus > 0.0) {
      double qcent = V(c1, i) * qplus + V(c2, i) * qmnus;
      double qvanl = 2.0 * qplus * qmnus / (qmnus + qplus);
      double temp1 = fmin2(fmin2(fmin2(fabs(qcent), fabs(qvanl)), 2.0 * fabs(qmnus)),
                           2.0 * fabs(qplus));
      V(dq, i) = temp1 * fsign1(qcent);
    } else {
      V(dq, i) = 0.0;
    }
  }
  /* edge values, intvar.F:98-102 */
  for (i = i1 - 1; i <= i2 + 2; i++) {
    V(ql, i) = V(c3, i) * V(q, i - 1) + V(c4, i) * V(q, i) + V(c5, i) * V(dq, i - 1) +
               V(c6, i) * V(dq, i);
    V(qr, i - 1) = V(ql, i);
  }
  /* steepening, intvar.F:106-113 */
  if (isteep != 0) {
    for (i = i1 - 1; i <= i2 + 1; i++) {
      V(ql, i) = (1.0 - V(steepen, i)) * V(ql, i) +
                 V(steepen, i) * (V(q, i - 1) + 0.5 * V(dq, i - 1));
      V(qr, i) = (1.0 - V(steepen, i)) * V(qr, i) +
                 V(steepen, i) * (V(q, i + 1) - 0.5 * V(dq, i + 1));
    }
  }
  /* monotonise, intvar.F:117-131 */
  for (i = i1 - 1; i <= i2 + 1; i++) {
    double temp1 = (V(qr, i) - V(q, i)) * (V(q, i) - V(ql, i));
    double temp2 = V(qr, i) - V(ql, i);
    double temp3 = 6.0 * (V(q, i) - 0.5 * (V(qr, i) + V(ql, i)));
    if (temp1 <= 0.0) {
      V(ql, i) = V(q, i);
      V(qr, i) = V(q, i);
    }
    double temp22 = temp2 * temp2;
    double temp23 = temp2 * temp3;
    if (temp22 < temp23) V(ql, i) = 3.0 * V(q, i) - 2.0 * V(qr, i);
    if (temp22 < -temp23) V(qr, i) = 3.0 * V(q, i) - 2.0 * V(ql, i);
  }
  /* flattening, intvar.F:135-140 */
  if (iflatten != 0) {
    for (i = i1 - 1; i <= i2 + 1; i++) {
      V(ql, i) = V(q, i) * V(flatten, i) + V(ql, i) * (1.0 - V(flatten, i));
      V(qr, i) = V(q, i) * V(flatten, i) + V(qr, i) * (1.0 - V(flatten, i));
    }
  }
  /* CHECK_LR, intvar.F:145-153 */
  for (i = i1 - 1; i <= i2 + 2; i++) {
    V(ql, i) = fmax2(fmin2(V(q, i), V(q, i - 1)), V(ql, i));
    V(ql, i) = fmin2(fmax2(V(q, i), V(q, i - 1)), V(ql, i));
    V(qr, i) = fmax2(fmin2(V(q, i), V(q, i + 1)), V(qr, i));
    V(qr, i) = fmin2(fmax2(V(q, i), V(q, i + 1)), V(qr, i));
  }
  /* intvar.F:157-160 */
  for (i = i1 - 1; i <= i2 + 1; i++) {
    V(q6, i) = 6.0 * (V(q, i) - 0.5 * (V(ql, i) + V(qr, i)));
    V(dq, i) = V(qr, i) - V(ql, i);
  }
  /* intvar.F:162-174 */
  for (i = i1; i <= i2 + 1; i++) {
    V(qla, i) = V(qr, i - 1) - V(char1, i - 1) * (V(dq, i - 1) - (1.0 - ft * V(char1, i - 1)) * V(q6, i - 1));
    V(qra, i) = V(ql, i) + V(char2, i) * (V(dq, i) + (1.0 - ft * V(char2, i)) * V(q6, i));
  }
  for (i = i1; i <= i2 + 1; i++) {
    V(ql0, i) = V(qr, i - 1) - V(c0, i - 1) * (V(dq, i - 1) - (1.0 - ft * V(c0, i - 1)) * V(q6, i - 1));
    V(qr0, i) = V(ql, i) - V(c0, i) * (V(dq, i) + (1.0 + ft * V(c0, i)) * V(q6, i));
  }
}

/* ------------------------------------------------------------------------ */
/* calcdiss.F: the flattening coefficients of one pencil (iflatten 1 or 3;    */
/* no diffusion).  wflag (eq. A1) :213-224, type 1 (A1-A2) :407-438, type 3  */
/* (A7-A10) :486-559, both ending with the max of eq. A2.                     */
/* ------------------------------------------------------------------------ */
static void calcdiss_flatten(work_t *W, const ora_params *P, const double *dsl,
                             const double *esl, const double *usl, const double *psl, int i1,
                             int i2) {
  const double epsilon = 0.33, kappa1 = 2.0, kappa2 = 0.01, omega1 = 0.75, omega2 = 10.0,
               sigma1 = 0.5, sigma2 = 1.0;
  const double gamma = P->gamma;
  int i;
  for (i = i1 - 2; i <= i2 + 2; i++) {
    double qb = fabs(V(psl, i + 1) - V(psl, i - 1)) / fmin2(V(psl, i + 1), V(psl, i - 1));
    V(W->wflag, i) = (qb > epsilon && V(usl, i - 1) > V(usl, i + 1)) ? 1.0 : 0.0;
  }
  if (P->flatten == 1) {
    for (i = i1 - 1; i <= i2 + 1; i++) {
      double qa;
      if (fabs(V(psl, i + 2) - V(psl, i - 2)) / fmin2(V(psl, i + 2), V(psl, i - 2)) < epsilon)
        qa = 1.0;
      else
        qa = (V(psl, i + 1) - V(psl, i - 1)) / (V(psl, i + 2) - V(psl, i - 2));
      V(W->ftemp, i) = fmin2(1.0, (qa - omega1) * omega2 * V(W->wflag, i));
      V(W->ftemp, i) = fmax2(0.0, V(W->ftemp, i));
    }
  } else if (P->flatten == 2) {  /* calcdiss.F:445-478, eq. A4-A5 */
    for (i = i1 - 1; i <= i2 + 1; i++) {
      const double dp1 = V(psl, i + 1) - V(psl, i - 1);
      const int is2 = i + (int)copysign(2.0, dp1);
      const double omega =
          fmax_g(0.0, omega1 * (omega2 - dp1 / (V(psl, i + 2) - V(psl, i - 2))));
      const double di2p = 1.0 / V(dsl, i + 2), di2m = 1.0 / V(dsl, i - 2);
      const double Z = sqrt((fmax_g(V(psl, i + 2), V(psl, i - 2)) +
                             0.5 * (V(psl, i + 2) + V(psl, i - 2)) * (gamma - 1.0)) /
                            fmax_g(di2p, di2m));
      const double kappa_tilde = (Z + sqrt(gamma * V(psl, is2) * V(dsl, is2))) / Z;
      const double kappa = fmax_g(0.0, (kappa_tilde - kappa1) / (kappa_tilde + kappa2));
      V(W->ftemp, i) = fmin_g(V(W->wflag, i) * omega, kappa);
    }
  } else {  /* P->flatten == 3 */
    for (i = i1 - 1; i <= i2 + 1; i++) {
      const double dp1 = V(psl, i + 1) - V(psl, i - 1);
      const double dp2 = V(psl, i + 2) - V(psl, i - 2);
      const double de1 = V(esl, i + 1) - V(esl, i - 1);
      const double de2 = V(esl, i + 2) - V(esl, i - 2);
      double dpp = 0.0, dee = 0.0;
      if (dp2 != 0.0) dpp = dp1 / dp2;
      if (de2 != 0.0) dee = de1 / de2;
      const double omega_tilde = fmax2(dpp, dee);
      const int ism = i + (int)copysign(2.0, dp1); /* post-shock */
      const int isp = i - (int)copysign(2.0, dp1); /* upstream */
      double s = -copysign(1.0, dp1);
      if (dp1 == 0.0) s = 0.0;
      const double sigma_tilde =
          V(W->wflag, i) * fabs(dp2) / fmin2(V(psl, i + 2), V(psl, i - 2));
      const double sigma = fmax2(0.0, (sigma_tilde - sigma1) / (sigma_tilde + sigma2));
      const double omega = fmax2(0.0, omega2 * (omega_tilde - omega1));
      const double di2p = 1.0 / V(dsl, i + 2), di2m = 1.0 / V(dsl, i - 2);
      const double Z = sqrt((fmax2(V(psl, i + 2), V(psl, i - 2)) +
                             0.5 * (V(psl, i + 2) + V(psl, i - 2)) * (gamma - 1.0)) /
                            fmax2(di2p, di2m));
      const double ZE = s * Z / V(dsl, ism) + V(usl, ism) + F_TINY;
      const double cj2s = sqrt(gamma * V(psl, isp) / V(dsl, isp));
      const double kappa_tilde = fabs((ZE - V(usl, isp) + s * cj2s) / ZE);
      const double kappa = fmax2(0.0, (kappa_tilde - kappa1) / (kappa_tilde + kappa2));
      V(W->ftemp, i) =
          fmin2(fmin2(kappa, V(W->wflag, i) * omega), V(W->wflag, i) * sigma);
    }
  }
  V(W->ftemp, i1 - 2) = V(W->ftemp, i1 - 1);
  V(W->ftemp, i2 + 2) = V(W->ftemp, i2 + 1);
  for (i = i1 - 1; i <= i2 + 1; i++) {
    if (P->flatten == 2) /* eq. A6, calcdiss.F:480-483 */
      V(W->flat, i) = fmax_g(fmax_g(V(W->ftemp, i - 1), V(W->ftemp, i)), V(W->ftemp, i + 1));
    else if (V(psl, i + 1) - V(psl, i - 1) < 0.0)
      V(W->flat, i) = fmax2(V(W->ftemp, i), V(W->ftemp, i + 1));
    else
      V(W->flat, i) = fmax2(V(W->ftemp, i), V(W->ftemp, i - 1));
  }
}

/* inteuler.F:166-193: the density steepening coefficients of one pencil */
static void steepening(work_t *W, const ora_params *P, const double *dxi, const double *dsl,
                       const double *psl, int i1, int i2) {
  int i;
  for (i = i1 - 2; i <= i2 + 2; i++) {
    double qa = V(dxi, i - 1) + V(dxi, i) + V(dxi, i + 1);
    V(W->d2d, i) = (V(dsl, i + 1) - V(dsl, i)) / (V(dxi, i + 1) + V(dxi, i));
    V(W->d2d, i) = (V(W->d2d, i) - (V(dsl, i) - V(dsl, i - 1)) / (V(dxi, i) + V(dxi, i - 1))) / qa;
    V(W->dxb, i) = 0.5 * (V(dxi, i) + V(dxi, i + 1));
  }
  for (i = i1 - 1; i <= i2 + 1; i++) {
    double qc = fabs(V(dsl, i + 1) - V(dsl, i - 1)) -
                0.01 * fmin2(fabs(V(dsl, i + 1)), fabs(V(dsl, i - 1)));
    const double bm = V(W->dxb, i - 1), b0 = V(W->dxb, i);
    double s1 = (V(W->d2d, i - 1) - V(W->d2d, i + 1)) * (bm * bm * bm + b0 * b0 * b0) /
                ((b0 + bm) * (V(dsl, i + 1) - V(dsl, i - 1) + F_TINY));
    if (V(W->d2d, i + 1) * V(W->d2d, i - 1) > 0.0) s1 = 0.0;
    if (qc <= 0.0) s1 = 0.0;
    const double s2 = fmax2(0.0, fmin2(20.0 * (s1 - 0.05), 1.0));
    const double qa = fabs(V(dsl, i + 1) - V(dsl, i - 1)) / fmin2(V(dsl, i + 1), V(dsl, i - 1));
    const double qb = fabs(V(psl, i + 1) - V(psl, i - 1)) / fmin2(V(psl, i + 1), V(psl, i - 1));
    V(W->steep, i) = (P->gamma * 0.1 * qa >= qb) ? s2 : 0.0;
  }
}

/* ------------------------------------------------------------------------ */
/* inteuler.F:5-566 (conservative/positive reconstruction and colours off)   */
/* ------------------------------------------------------------------------ */
static void inteuler(work_t *W, const ora_params *P, const double *dxi, int i1, int i2,
                     int j1, int j2) {
  const int idim = W->idim;
  const double ft = 4.0 / 3.0;
  const double dt = P->dt, gamma = P->gamma, eta2 = P->eta2;
  int i, j;
  /* interpolation coefficients, inteuler.F:140-158 */
  for (i = i1 - 2; i <= i2 + 2; i++) {
    double qa = V(dxi, i) / (V(dxi, i - 1) + V(dxi, i) + V(dxi, i + 1));
    V(W->c1, i) = qa * (2.0 * V(dxi, i - 1) + V(dxi, i)) / (V(dxi, i + 1) + V(dxi, i));
    V(W->c2, i) = qa * (2.0 * V(dxi, i + 1) + V(dxi, i)) / (V(dxi, i - 1) + V(dxi, i));
    V(W->dxdt2, i) = 0.5 * dt / V(dxi, i);
  }
  for (i = i1 - 1; i <= i2 + 2; i++) {
    double qa = V(dxi, i - 2) + V(dxi, i - 1) + V(dxi, i) + V(dxi, i + 1);
    double qb = V(dxi, i - 1) / (V(dxi, i - 1) + V(dxi, i));
    double qc = (V(dxi, i - 2) + V(dxi, i - 1)) / (2.0 * V(dxi, i - 1) + V(dxi, i));
    double qd = (V(dxi, i + 1) + V(dxi, i)) / (2.0 * V(dxi, i) + V(dxi, i - 1));
    qb = qb + 2.0 * V(dxi, i) * qb / qa * (qc - qd);
    V(W->c3, i) = 1.0 - qb;
    V(W->c4, i) = qb;
    V(W->c5, i) = V(dxi, i) / qa * qd;
    V(W->c6, i) = -(V(dxi, i - 1) / qa * qc);
    V(W->dx2i, i) = 0.5 / V(dxi, i);
  }
  for (j = j1; j <= j2; j++) {
    const double *dsl = &S(W->d, 1, j), *psl = &S(W->p, 1, j), *usl = &S(W->u, 1, j);
    const double *vsl = &S(W->v, 1, j), *wsl = &S(W->w, 1, j), *gesl = &S(W->ge, 1, j);
    const double *grs = &S(W->gr, 1, j);
    /* characteristic distances, inteuler.F:197-208.  The reference sweeps
       i = 1..idim, but only i1-1..i2+2 are defined (dx2i) and used. */
    for (i = i1 - 1; i <= i2 + 2; i++) {
      V(W->cs, i) = sqrt(gamma * V(psl, i) / V(dsl, i));
      if (P->pressure_free == 1) V(W->cs, i) = F_TINY;
      V(W->char1, i) = fmax2(0.0, dt * (V(usl, i) + V(W->cs, i))) * V(W->dx2i, i);
      V(W->char2, i) = fmax2(0.0, -(dt * (V(usl, i) - V(W->cs, i)))) * V(W->dx2i, i);
    }
    for (i = i1 - 1; i <= i2 + 2; i++) {
      V(W->cm, i) = dt * (V(usl, i) - V(W->cs, i)) * V(W->dx2i, i);
      V(W->c0, i) = dt * (V(usl, i)) * V(W->dx2i, i);
      V(W->cp, i) = dt * (V(usl, i) + V(W->cs, i)) * V(W->dx2i, i);
    }
    /* the pencil's flattening (calcdiss, called by the sweep before inteuler) and
       steepening coefficients */
    if (P->flatten != 0) calcdiss_flatten(W, P, dsl, &S(W->e, 1, j), usl, psl, i1, i2);
    if (P->steepen != 0) steepening(W, P, dxi, dsl, psl, i1, i2);
    const int ist = P->steepen, ifl = P->flatten;
    /* inteuler.F:235-274 (steepening applies to the density only) */
    intvar(dsl, idim, i1, i2, ist, W->steep, ifl, W->flat, W->c1, W->c2, W->c3, W->c4, W->c5,
           W->c6, W->char1, W->char2, W->c0, W->t1, W->t2, W->t3, W->t4, W->dla, W->dra,
           W->dl0, W->dr0);
    intvar(psl, idim, i1, i2, 0, W->steep, ifl, W->flat, W->c1, W->c2, W->c3, W->c4, W->c5,
           W->c6, W->char1, W->char2, W->c0, W->dp, W->pl, W->pr, W->p6, W->pla, W->pra,
           W->pl0, W->pr0);
    intvar(usl, idim, i1, i2, 0, W->steep, ifl, W->flat, W->c1, W->c2, W->c3, W->c4, W->c5,
           W->c6, W->char1, W->char2, W->c0, W->du, W->ul, W->ur, W->u6, W->ula, W->ura,
           W->ul0, W->ur0);
    intvar(vsl, idim, i1, i2, 0, W->steep, ifl, W->flat, W->c1, W->c2, W->c3, W->c4, W->c5,
           W->c6, W->char1, W->char2, W->c0, W->dv, W->vl, W->vr, W->v6, W->vla, W->vra,
           W->vl0, W->vr0);
    intvar(wsl, idim, i1, i2, 0, W->steep, ifl, W->flat, W->c1, W->c2, W->c3, W->c4, W->c5,
           W->c6, W->char1, W->char2, W->c0, W->dw, W->wl, W->wr, W->w6, W->wla, W->wra,
           W->wl0, W->wr0);
    if (P->dual == 1)
      intvar(gesl, idim, i1, i2, 0, W->steep, ifl, W->flat, W->c1, W->c2, W->c3, W->c4, W->c5,
             W->c6, W->char1, W->char2, W->c0, W->dge, W->gel, W->ger, W->ge6, W->gela,
             W->gera, W->gel0, W->ger0);
    /* colours, inteuler.F:276-282 (no steepening, the slice's flattening) */
    for (int n = 0; n < W->ncol; n++)
      intvar(&CS(W->col, 1, j, n), idim, i1, i2, 0, W->steep, ifl, W->flat, W->c1, W->c2,
             W->c3, W->c4, W->c5, W->c6, W->char1, W->char2, W->c0, &CV(W->dcol, 1, n),
             &CV(W->coll, 1, n), &CV(W->colr, 1, n), &CV(W->col6, 1, n), &CV(W->colla, 1, n),
             &CV(W->colra, 1, n), &CV(W->coll0, 1, n), &CV(W->colr0, 1, n));
    /* characteristic domain-of-dependence averages, inteuler.F:304-316 */
    for (i = i1; i <= i2 + 1; i++) {
      V(W->plm, i) = V(W->pr, i - 1) - V(W->cm, i - 1) * (V(W->dp, i - 1) - (1.0 - ft * V(W->cm, i - 1)) * V(W->p6, i - 1));
      V(W->prm, i) = V(W->pl, i) - V(W->cm, i) * (V(W->dp, i) + (1.0 + ft * V(W->cm, i)) * V(W->p6, i));
      V(W->plp, i) = V(W->pr, i - 1) - V(W->cp, i - 1) * (V(W->dp, i - 1) - (1.0 - ft * V(W->cp, i - 1)) * V(W->p6, i - 1));
      V(W->prp, i) = V(W->pl, i) - V(W->cp, i) * (V(W->dp, i) + (1.0 + ft * V(W->cp, i)) * V(W->p6, i));
    }
    for (i = i1; i <= i2 + 1; i++) {
      V(W->ulm, i) = V(W->ur, i - 1) - V(W->cm, i - 1) * (V(W->du, i - 1) - (1.0 - ft * V(W->cm, i - 1)) * V(W->u6, i - 1));
      V(W->urm, i) = V(W->ul, i) - V(W->cm, i) * (V(W->du, i) + (1.0 + ft * V(W->cm, i)) * V(W->u6, i));
      V(W->ulp, i) = V(W->ur, i - 1) - V(W->cp, i - 1) * (V(W->du, i - 1) - (1.0 - ft * V(W->cp, i - 1)) * V(W->u6, i - 1));
      V(W->urp, i) = V(W->ul, i) - V(W->cp, i) * (V(W->du, i) + (1.0 + ft * V(W->cp, i)) * V(W->u6, i));
    }
    /* correction terms, inteuler.F:320-395 */
    for (i = i1; i <= i2 + 1; i++) {
      V(W->cla, i) = sqrt(fmax2(gamma * V(W->pla, i) * V(W->dla, i), 0.0));
      V(W->cra, i) = sqrt(fmax2(gamma * V(W->pra, i) * V(W->dra, i), 0.0));
    }
    for (i = i1; i <= i2 + 1; i++) {
      double f1 = 1.0 / V(W->cla, i);
      V(W->betalp, i) = (V(W->ula, i) - V(W->ulp, i)) + (V(W->pla, i) - V(W->plp, i)) * f1;
      V(W->betalm, i) = (V(W->ula, i) - V(W->ulm, i)) - (V(W->pla, i) - V(W->plm, i)) * f1;
      V(W->betal0, i) = (V(W->pla, i) - V(W->pl0, i)) * (f1 * f1) + 1.0 / V(W->dla, i) - 1.0 / V(W->dl0, i);
    }
    if (P->gravity == 1) {
      for (i = i1; i <= i2 + 1; i++) {
        V(W->betalp, i) = V(W->betalp, i) - 0.25 * dt * (V(grs, i - 1) + V(grs, i));
        V(W->betalm, i) = V(W->betalm, i) - 0.25 * dt * (V(grs, i - 1) + V(grs, i));
      }
    }
    for (i = i1; i <= i2 + 1; i++) {
      double f1 = 0.5 / V(W->cla, i);
      V(W->betalp, i) = -(V(W->betalp, i) * f1);
      V(W->betalm, i) = +V(W->betalm, i) * f1;
    }
    for (i = i1; i <= i2 + 1; i++) {
      if (V(W->cp, i - 1) <= 0.0) V(W->betalp, i) = 0.0;
      if (V(W->cm, i - 1) <= 0.0) V(W->betalm, i) = 0.0;
      if (V(W->c0, i - 1) <= 0.0) V(W->betal0, i) = 0.0;
    }
    for (i = i1; i <= i2 + 1; i++) {
      double f1 = 1.0 / V(W->cra, i);
      V(W->betarp, i) = (V(W->ura, i) - V(W->urp, i)) + (V(W->pra, i) - V(W->prp, i)) * f1;
      V(W->betarm, i) = (V(W->ura, i) - V(W->urm, i)) - (V(W->pra, i) - V(W->prm, i)) * f1;
      V(W->betar0, i) = (V(W->pra, i) - V(W->pr0, i)) * (f1 * f1) + 1.0 / V(W->dra, i) - 1.0 / V(W->dr0, i);
    }
    if (P->gravity == 1) {
      for (i = i1; i <= i2 + 1; i++) {
        V(W->betarp, i) = V(W->betarp, i) - 0.25 * dt * (V(grs, i - 1) + V(grs, i));
        V(W->betarm, i) = V(W->betarm, i) - 0.25 * dt * (V(grs, i - 1) + V(grs, i));
      }
    }
    for (i = i1; i <= i2 + 1; i++) {
      double f1 = 0.5 / V(W->cra, i);
      V(W->betarp, i) = -(V(W->betarp, i) * f1);
      V(W->betarm, i) = +V(W->betarm, i) * f1;
    }
    for (i = i1; i <= i2 + 1; i++) {
      if (V(W->cp, i) >= 0.0) V(W->betarp, i) = 0.0;
      if (V(W->cm, i) >= 0.0) V(W->betarm, i) = 0.0;
      if (V(W->c0, i) >= 0.0) V(W->betar0, i) = 0.0;
    }
    /* corrected states, inteuler.F:399-410 */
    for (i = i1; i <= i2 + 1; i++) {
      S(W->pls, i, j) = V(W->pla, i) + (V(W->betalp, i) + V(W->betalm, i)) * (V(W->cla, i) * V(W->cla, i));
      S(W->prs, i, j) = V(W->pra, i) + (V(W->betarp, i) + V(W->betarm, i)) * (V(W->cra, i) * V(W->cra, i));
      S(W->uls, i, j) = V(W->ula, i) + (V(W->betalp, i) - V(W->betalm, i)) * V(W->cla, i);
      S(W->urs, i, j) = V(W->ura, i) + (V(W->betarp, i) - V(W->betarm, i)) * V(W->cra, i);
      S(W->dls, i, j) = 1.0 / (1.0 / V(W->dla, i) - (V(W->betal0, i) + V(W->betalp, i) + V(W->betalm, i)));
      S(W->drs, i, j) = 1.0 / (1.0 / V(W->dra, i) - (V(W->betar0, i) + V(W->betarp, i) + V(W->betarm, i)));
    }
    /* advected quantities, inteuler.F:414-434 */
    for (i = i1; i <= i2 + 1; i++) {
      if (V(usl, i - 1) <= 0.0) {
        S(W->vls, i, j) = V(W->vla, i);
        S(W->wls, i, j) = V(W->wla, i);
        S(W->gels, i, j) = V(W->gela, i);
      } else {
        S(W->vls, i, j) = V(W->vl0, i);
        S(W->wls, i, j) = V(W->wl0, i);
        S(W->gels, i, j) = V(W->gel0, i);
      }
      if (V(usl, i) >= 0.0) {
        S(W->vrs, i, j) = V(W->vra, i);
        S(W->wrs, i, j) = V(W->wra, i);
        S(W->gers, i, j) = V(W->gera, i);
      } else {
        S(W->vrs, i, j) = V(W->vr0, i);
        S(W->wrs, i, j) = V(W->wr0, i);
        S(W->gers, i, j) = V(W->ger0, i);
      }
    }
    /* colour states scaled by the corrected density, inteuler.F:436-450 */
    for (int n = 0; n < W->ncol; n++) {
      for (i = i1; i <= i2 + 1; i++) {
        if (V(usl, i - 1) <= 0.0)
          CS(W->colls, i, j, n) = CV(W->colla, i, n) * S(W->dls, i, j) / V(W->dla, i);
        else
          CS(W->colls, i, j, n) = CV(W->coll0, i, n) * S(W->dls, i, j) / V(W->dl0, i);
        if (V(usl, i) >= 0.0)
          CS(W->colrs, i, j, n) = CV(W->colra, i, n) * S(W->drs, i, j) / V(W->dra, i);
        else
          CS(W->colrs, i, j, n) = CV(W->colr0, i, n) * S(W->drs, i, j) / V(W->dr0, i);
      }
    }
    /* dual-energy hypersonic override, inteuler.F:493-521 */
    if (P->dual == 1) {
      for (i = i1; i <= i2 + 1; i++) {
        double ml = fmax2(fmax2(fabs(V(W->cm, i - 1)), fabs(V(W->c0, i - 1))), fabs(V(W->cp, i - 1)));
        if (gamma * V(W->pla, i) / V(W->dla, i) < eta2 * (V(W->ula, i) * V(W->ula, i)) ||
            ml < 1.0e-3 || S(W->dls, i, j) / V(W->dla, i) > 5.0) {
          for (int n = 0; n < W->ncol; n++)
            CS(W->colls, i, j, n) = CS(W->colls, i, j, n) * V(W->dla, i) / S(W->dls, i, j);
          S(W->pls, i, j) = V(W->pla, i);
          S(W->uls, i, j) = V(W->ula, i);
          S(W->dls, i, j) = V(W->dla, i);
        }
        double mr = fmax2(fmax2(fabs(V(W->cm, i)), fabs(V(W->c0, i))), fabs(V(W->cp, i)));
        if (gamma * V(W->pra, i) / V(W->dra, i) < eta2 * (V(W->ura, i) * V(W->ura, i)) ||
            mr < 1.0e-3 || S(W->drs, i, j) / V(W->dra, i) > 5.0) {
          for (int n = 0; n < W->ncol; n++)
            CS(W->colrs, i, j, n) = CS(W->colrs, i, j, n) * V(W->dra, i) / S(W->drs, i, j);
          S(W->prs, i, j) = V(W->pra, i);
          S(W->urs, i, j) = V(W->ura, i);
          S(W->drs, i, j) = V(W->dra, i);
        }
      }
    }
    /* floors, inteuler.F:540-545 */
    for (i = i1; i <= i2 + 1; i++) {
      S(W->pls, i, j) = fmax2(S(W->pls, i, j), F_TINY);
      S(W->prs, i, j) = fmax2(S(W->prs, i, j), F_TINY);
      S(W->dls, i, j) = fmax2(S(W->dls, i, j), F_TINY);
      S(W->drs, i, j) = fmax2(S(W->drs, i, j), F_TINY);
    }
    for (int n = 0; n < W->ncol; n++) {  /* inteuler.F:546-551 */
      for (i = i1; i <= i2 + 1; i++) {
        CS(W->colls, i, j, n) = fmax2(CS(W->colls, i, j, n), F_COLOR_FLOOR);
        CS(W->colrs, i, j, n) = fmax2(CS(W->colrs, i, j, n), F_COLOR_FLOOR);
      }
    }
    if (P->pressure_free == 1) {
      for (i = i1; i <= i2 + 1; i++) {
        S(W->dls, i, j) = V(W->dla, i);
        S(W->drs, i, j) = V(W->dra, i);
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* twoshock.F:5-276 (gravity .ne. 99 branch)                                 */
/* ------------------------------------------------------------------------ */
static void twoshock(work_t *W, const ora_params *P, int i1, int i2, int j1, int j2,
                     ora_stats *st) {
  const int idim = W->idim;
  const double gamma = P->gamma, pmin = P->tiny_number;
  const double qa = (gamma + 1.0) / (2.0 * gamma);
  int i, j, n;
  for (j = j1; j <= j2; j++) {
    if (P->pressure_free == 1) {
      for (i = i1; i <= i2; i++) {
        S(W->pbar, i, j) = pmin;
        S(W->ubar, i, j) = 0.5 * (S(W->uls, i, j) + S(W->urs, i, j));
        S(W->pls, i, j) = pmin;
        S(W->prs, i, j) = pmin;
      }
      continue;
    }
    for (i = i1; i <= i2; i++) {
      V(W->tcl, i) = sqrt(gamma * S(W->pls, i, j) * S(W->dls, i, j));
      V(W->tcr, i) = sqrt(gamma * S(W->prs, i, j) * S(W->drs, i, j));
      V(W->ps, i) = (V(W->tcr, i) * S(W->pls, i, j) + V(W->tcl, i) * S(W->prs, i, j) +
                     V(W->tcr, i) * V(W->tcl, i) * (S(W->uls, i, j) - S(W->urs, i, j))) /
                    (V(W->tcr, i) + V(W->tcl, i));
      if (V(W->ps, i) < pmin) V(W->ps, i) = pmin;
    }
    for (i = i1; i <= i2; i++) {
      V(W->old_ps, i) = V(W->ps, i);
      V(W->delta_ps, i) = V(W->ps, i);
      W->mask[i - 1] = 1;
      W->niter[i - 1] = 0;
    }
    for (n = 2; n <= TS_NUMITER; n++) {
      for (i = i1; i <= i2; i++) {
        if (W->mask[i - 1] > 0) {
          V(W->zl, i) = V(W->tcl, i) * sqrt((1.0 + qa * (V(W->ps, i) / S(W->pls, i, j) - 1.0)));
          V(W->zr, i) = V(W->tcr, i) * sqrt((1.0 + qa * (V(W->ps, i) / S(W->prs, i, j) - 1.0)));
          V(W->ubl, i) = S(W->uls, i, j) - (V(W->ps, i) - S(W->pls, i, j)) / V(W->zl, i);
          V(W->ubr, i) = S(W->urs, i, j) + (V(W->ps, i) - S(W->prs, i, j)) / V(W->zr, i);
        }
      }
      for (i = i1; i <= i2; i++) {
        if (W->mask[i - 1] > 0) {
          double zl = V(W->zl, i), zr = V(W->zr, i);
          V(W->dpdul, i) = -(4.0 * (zl * zl * zl) / S(W->dls, i, j) /
                             (4.0 * (zl * zl) / S(W->dls, i, j) - (gamma + 1.0) * (V(W->ps, i) - S(W->pls, i, j))));
          V(W->dpdur, i) = 4.0 * (zr * zr * zr) / S(W->drs, i, j) /
                           (4.0 * (zr * zr) / S(W->drs, i, j) - (gamma + 1.0) * (V(W->ps, i) - S(W->prs, i, j)));
          V(W->ps, i) = V(W->ps, i) + (V(W->ubr, i) - V(W->ubl, i)) * V(W->dpdur, i) * V(W->dpdul, i) /
                                          (V(W->dpdur, i) - V(W->dpdul, i));
          if (V(W->ps, i) < pmin) V(W->ps, i) = pmin;
          V(W->delta_ps, i) = V(W->ps, i) - V(W->old_ps, i);
          V(W->old_ps, i) = V(W->ps, i);
          W->niter[i - 1] += 1;
          if (fabs(V(W->delta_ps, i) / V(W->ps, i)) < TS_TOLERANCE) W->mask[i - 1] = 0;
        }
      }
    }
    for (i = i1; i <= i2; i++) {
      if (V(W->ps, i) < pmin) V(W->ps, i) = fmin2(S(W->pls, i, j), S(W->prs, i, j));
      S(W->pbar, i, j) = V(W->ps, i);
      S(W->ubar, i, j) = V(W->ubl, i) + (V(W->ubr, i) - V(W->ubl, i)) * V(W->dpdur, i) /
                                            (V(W->dpdur, i) - V(W->dpdul, i));
      if (st) {
        st->interfaces += 1;
        st->newton_iters += W->niter[i - 1];
        st->newton_hist[W->niter[i - 1]] += 1;
      }
      if (g_log_fn) {
        double s6[6] = {S(W->dls, i, j), S(W->drs, i, j), S(W->pls, i, j),
                        S(W->prs, i, j), S(W->uls, i, j), S(W->urs, i, j)};
        g_log_fn(g_log_ctx, s6, S(W->pbar, i, j), W->niter[i - 1]);
      }
    }
  }
}

void ora_twoshock_point(const double s6[6], double gamma, double pmin, double guess,
                        double *pbar, double *ubar, int *iters) {
  const double dls = s6[0], drs = s6[1], pls = s6[2], prs = s6[3], uls = s6[4], urs = s6[5];
  const double qa = (gamma + 1.0) / (2.0 * gamma);
  double cl = sqrt(gamma * pls * dls);
  double cr = sqrt(gamma * prs * drs);
  double ps = (cr * pls + cl * prs + cr * cl * (uls - urs)) / (cr + cl);
  if (ps < pmin) ps = pmin;
  if (guess > 0.0) ps = guess;
  double old_ps = ps, zl = 0, zr = 0, ubl = 0, ubr = 0, dpdul = 0, dpdur = 0;
  int mask = 1, it = 0;
  for (int n = 2; n <= TS_NUMITER; n++) {
    if (!mask) break;
    zl = cl * sqrt((1.0 + qa * (ps / pls - 1.0)));
    zr = cr * sqrt((1.0 + qa * (ps / prs - 1.0)));
    ubl = uls - (ps - pls) / zl;
    ubr = urs + (ps - prs) / zr;
    dpdul = -(4.0 * (zl * zl * zl) / dls / (4.0 * (zl * zl) / dls - (gamma + 1.0) * (ps - pls)));
    dpdur = 4.0 * (zr * zr * zr) / drs / (4.0 * (zr * zr) / drs - (gamma + 1.0) * (ps - prs));
    ps = ps + (ubr - ubl) * dpdur * dpdul / (dpdur - dpdul);
    if (ps < pmin) ps = pmin;
    double delta = ps - old_ps;
    old_ps = ps;
    it++;
    if (fabs(delta / ps) < TS_TOLERANCE) mask = 0;
  }
  if (ps < pmin) ps = fmin2(pls, prs);
  *pbar = ps;
  *ubar = ubl + (ubr - ubl) * dpdur / (dpdur - dpdul);
  *iters = mask ? -it : it; /* negative: did not reach the tolerance */
}

/* ------------------------------------------------------------------------ */
/* flux_hll.F:6-415, called per cell as the fallback (i1 = i2 = i).          */
/* The single-cell call's ges(i+1) reads flux_hll locals at index i+2 that   */
/* the call itself never sets (flux_hll.F:302-307).  Here those are defined  */
/* as the HLL values of face i+2 when that face exists (i+2 <= i2 of the     */
/* enclosing sweep), and as zero otherwise (that ges is not consumed).       */
/* ------------------------------------------------------------------------ */
static void hll_face(work_t *W, const ora_params *P, int i, int j, int with_flux, double *sl_o,
                     double *sr_o, double *gesl_o, double *gesr_o, double *fl) {
  const int idim = W->idim;
  const double gamma = P->gamma;
  const double gamma1 = gamma - 1.0;
  const double gamma1i = 1.0 / gamma1;
  double dls = S(W->dls, i, j), drs = S(W->drs, i, j), pls = S(W->pls, i, j), prs = S(W->prs, i, j);
  double uls = S(W->uls, i, j), urs = S(W->urs, i, j), vls = S(W->vls, i, j), vrs = S(W->vrs, i, j);
  double wls = S(W->wls, i, j), wrs = S(W->wrs, i, j);
  double sqrtdl = sqrt(dls);
  double sqrtdr = sqrt(drs);
  double isdlpdr = 1.0 / (sqrtdl + sqrtdr);
  double vroe1 = (sqrtdl * uls + sqrtdr * urs) * isdlpdr;
  double vroe2 = (sqrtdl * vls + sqrtdr * vrs) * isdlpdr;
  double vroe3 = (sqrtdl * wls + sqrtdr * wrs) * isdlpdr;
  double v2 = vroe1 * vroe1 + vroe2 * vroe2 + vroe3 * vroe3;
  double el = gamma1i * pls + 0.5 * dls * (uls * uls + vls * vls + wls * wls);
  double er = gamma1i * prs + 0.5 * drs * (urs * urs + vrs * vrs + wrs * wrs);
  double hroe = ((el + pls) / sqrtdl + (er + prs) / sqrtdr) * isdlpdr;
  double cs = sqrt(gamma1 * fmax2((hroe - 0.5 * v2), F_TINY));
  double char1 = vroe1 - cs;
  double char2 = vroe1 + cs;
  double csl0 = sqrt(gamma * pls / dls);
  double csr0 = sqrt(gamma * prs / drs);
  double csl = fmin2(uls - csl0, char1);
  double csr = fmax2(urs + csr0, char2);
  double bm = fmin2(csl, 0.0);
  double bp = fmax2(csr, 0.0);
  double bm0 = uls - bm;
  double bp0 = urs - bp;
  double q1 = (bp + bm) / (bp - bm);
  double sl = 0.5 * (1.0 + q1);
  double sr = 0.5 * (1.0 - q1);
  *sl_o = sl;
  *sr_o = sr;
  *gesl_o = bm0;
  *gesr_o = bp0;
  if (!with_flux) return;
  double dubl = dls * uls;
  double dubr = drs * urs;
  double dfl = dls * bm0, dfr = drs * bp0;
  double ufl = dubl * bm0 + pls, ufr = dubr * bp0 + prs;
  double vfl = dls * vls * bm0, vfr = drs * vrs * bp0;
  double wfl = dls * wls * bm0, wfr = drs * wrs * bp0;
  double efl = el * bm0 + pls * uls, efr = er * bp0 + prs * urs;
  fl[0] = sl * dfl + sr * dfr + 0.0;
  fl[1] = sl * ufl + sr * ufr + 0.0;
  fl[2] = sl * vfl + sr * vfr + 0.0;
  fl[3] = sl * wfl + sr * wfr + 0.0;
  fl[4] = sl * efl + sr * efr + 0.0;
  if (P->dual == 1) {
    double gefl = bm0 * S(W->gels, i, j) * dls;
    double gefr = bp0 * S(W->gers, i, j) * drs;
    fl[5] = sl * gefl + sr * gefr + 0.0;
  }
}

/* returns 0, or -1 on the fatal negative-density condition of flux_hll.F:336-383 */
static int flux_hll_cell(work_t *W, const ora_params *P, const double *dx, int i, int j,
                         int i2_sweep) {
  const int idim = W->idim;
  const double dt = P->dt, gamma = P->gamma;
  double sl[3], sr[3], gl[3], gr[3], fl[2][6];
  int f;
  for (f = 0; f < 2; f++) hll_face(W, P, i + f, j, 1, &sl[f], &sr[f], &gl[f], &gr[f], fl[f]);
  const int have3 = (i + 2 <= i2_sweep + 1);
  if (have3) {
    hll_face(W, P, i + 2, j, 0, &sl[2], &sr[2], &gl[2], &gr[2], 0);
  } else {
    sl[2] = sr[2] = gl[2] = gr[2] = 0.0;
  }
  for (f = 0; f < 2; f++) {
    const int ii = i + f;
    if (P->dual == 1) {
      double pcent = fmax2((gamma - 1.0) * S(W->ge, ii, j) * S(W->d, ii, j), F_TINY);
      double qc = dt / V(dx, ii);
      S(W->ges, ii, j) = qc * pcent * (sl[f] * gl[f] + sr[f] * gr[f] - sl[f + 1] * gl[f + 1] - sr[f + 1] * gr[f + 1]);
    }
  }
  for (f = 0; f < 2; f++) {
    const int ii = i + f;
    double qc = dt / V(dx, ii);
    S(W->df, ii, j) = qc * fl[f][0];
    S(W->uf, ii, j) = qc * fl[f][1];
    S(W->vf, ii, j) = qc * fl[f][2];
    S(W->wf, ii, j) = qc * fl[f][3];
    S(W->ef, ii, j) = qc * fl[f][4];
    if (P->dual == 1) S(W->gef, ii, j) = dt / V(dx, ii) * fl[f][5];
  }
  /* colours: bm0 = gesl, bp0 = gesr (flux_hll.F:236-262, :328-332) */
  for (int n = 0; n < W->ncol; n++) {
    for (f = 0; f < 2; f++) {
      const int ii = i + f;
      const double colfl = gl[f] * CS(W->colls, ii, j, n);
      const double colfr = gr[f] * CS(W->colrs, ii, j, n);
      CS(W->colf, ii, j, n) = sl[f] * colfl + sr[f] * colfr;
      CS(W->colf, ii, j, n) = dt * CS(W->colf, ii, j, n);
    }
  }
  if (S(W->d, i, j) + S(W->df, i, j) - S(W->df, i + 1, j) <= 0.0) return -1;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* HLLC face (flux_hllc.F:105-300 for one interface, no diffusion): the      */
/* weights sl, sr, the advective speeds gesl = ul - bm, gesr = ur - bp and   */
/* the five (six) fluxes before the dt/dx factor, the contact's momentum and  */
/* energy terms included (:282-286).                                         */
/* ------------------------------------------------------------------------ */
static void hllc_face(work_t *W, const ora_params *P, int i, int j, double *sl_o, double *sr_o,
                      double *gesl_o, double *gesr_o, double *fl) {
  const int idim = W->idim;
  const double gamma = P->gamma;
  const double gamma1 = gamma - 1.0;
  const double gamma1i = 1.0 / gamma1;
  double dls = S(W->dls, i, j), drs = S(W->drs, i, j), pls = S(W->pls, i, j), prs = S(W->prs, i, j);
  double uls = S(W->uls, i, j), urs = S(W->urs, i, j), vls = S(W->vls, i, j), vrs = S(W->vrs, i, j);
  double wls = S(W->wls, i, j), wrs = S(W->wrs, i, j);
  double sqrtdl = sqrt(dls);
  double sqrtdr = sqrt(drs);
  double isdlpdr = 1.0 / (sqrtdl + sqrtdr);
  double vroe1 = (sqrtdl * uls + sqrtdr * urs) * isdlpdr;
  double vroe2 = (sqrtdl * vls + sqrtdr * vrs) * isdlpdr;
  double vroe3 = (sqrtdl * wls + sqrtdr * wrs) * isdlpdr;
  double v2 = vroe1 * vroe1 + vroe2 * vroe2 + vroe3 * vroe3;
  double el = gamma1i * pls + 0.5 * dls * (uls * uls + vls * vls + wls * wls);
  double er = gamma1i * prs + 0.5 * drs * (urs * urs + vrs * vrs + wrs * wrs);
  double hroe = ((el + pls) / sqrtdl + (er + prs) / sqrtdr) * isdlpdr;
  double cs = sqrt(gamma1 * fmax2((hroe - 0.5 * v2), F_TINY));
  double char1 = vroe1 - cs;
  double char2 = vroe1 + cs;
  double csl0 = sqrt(gamma * pls / dls);
  double csr0 = sqrt(gamma * prs / drs);
  double csl = fmin2(uls - csl0, char1);
  double csr = fmax2(urs + csr0, char2);
  double bm = fmin2(csl, 0.0);
  double bp = fmax2(csr, 0.0);
  /* contact speed cw and pressure cp, flux_hllc.F:160-183 */
  double tl = pls - (csl - uls) * dls * uls;
  double tr = prs - (csr - urs) * drs * urs;
  double dl = dls * (csl - uls);
  double dr = -(drs * (csr - urs));
  double q1 = 1.0 / (dl + dr);
  double cw = (tr - tl) * q1;
  double cp = (dl * tr + dr * tl) * q1;
  double sl, sr, sm;
  if (cw >= 0.0) {
    sl = cw / (cw - bm);
    sr = 0.0;
    sm = -(bm / (cw - bm));
  } else {
    sl = 0.0;
    sr = -(cw / (bp - cw));
    sm = bp / (bp - cw);
  }
  cp = fmax2(cp, 0.0);
  double dubl = dls * uls;
  double dubr = drs * urs;
  double dfl = dubl - bm * dls, dfr = dubr - bp * drs;
  double ufl = dubl * (uls - bm) + pls, ufr = dubr * (urs - bp) + prs;
  double vfl = dls * vls * (uls - bm), vfr = drs * vrs * (urs - bp);
  double wfl = dls * wls * (uls - bm), wfr = drs * wrs * (urs - bp);
  double efl = el * (uls - bm) + pls * uls, efr = er * (urs - bp) + prs * urs;
  *sl_o = sl;
  *sr_o = sr;
  *gesl_o = uls - bm;
  *gesr_o = urs - bp;
  fl[0] = sl * dfl + sr * dfr + 0.0;
  fl[1] = sl * ufl + sr * ufr + 0.0;
  fl[2] = sl * vfl + sr * vfr + 0.0;
  fl[3] = sl * wfl + sr * wfr + 0.0;
  fl[4] = sl * efl + sr * efr + 0.0;
  if (P->dual == 1) {
    double gefl = (uls - bm) * S(W->gels, i, j) * dls;
    double gefr = (urs - bp) * S(W->gers, i, j) * drs;
    fl[5] = sl * gefl + sr * gefr + 0.0;
  }
  fl[1] = fl[1] + sm * cp;
  fl[4] = fl[4] + sm * cp * cw;
}

/* ------------------------------------------------------------------------ */
/* RiemannSolver = HLL (flux_hll.F:6-415) or HLLC (flux_hllc.F:6-421) over   */
/* the pencils: fluxes of faces i1..i2+1, the gas-energy source, colours,    */
/* dt/dx; then the negative-density check, fatal for HLL, the per-cell HLL  */
/* fallback for HLLC (flux_hllc.F:331-389).  ges(i2+1) reads locals at i2+2 */
/* that the reference never sets; it is not consumed and is zero here.      */
/* ------------------------------------------------------------------------ */
static int flux_hll_family(work_t *W, const ora_params *P, const double *dx, int i1, int i2,
                           int j1, int j2, int hllc, ora_stats *st) {
  const int idim = W->idim;
  const double gamma = P->gamma, dt = P->dt;
  int i, j, rc = 0;
  for (j = j1; j <= j2; j++) {
    /* per-face weights in the flux_hll locals (index i2+2 zero) */
    for (i = i1; i <= i2 + 2; i++) {
      V(W->h_sl, i) = V(W->h_sr, i) = V(W->h_gesl, i) = V(W->h_gesr, i) = 0.0;
    }
    for (i = i1; i <= i2 + 1; i++) {
      double fl[6] = {0, 0, 0, 0, 0, 0};
      if (hllc)
        hllc_face(W, P, i, j, &V(W->h_sl, i), &V(W->h_sr, i), &V(W->h_gesl, i), &V(W->h_gesr, i), fl);
      else
        hll_face(W, P, i, j, 1, &V(W->h_sl, i), &V(W->h_sr, i), &V(W->h_gesl, i), &V(W->h_gesr, i), fl);
      S(W->df, i, j) = fl[0];
      S(W->uf, i, j) = fl[1];
      S(W->vf, i, j) = fl[2];
      S(W->wf, i, j) = fl[3];
      S(W->ef, i, j) = fl[4];
      if (P->dual == 1) S(W->gef, i, j) = fl[5];
    }
    for (int n = 0; n < W->ncol; n++)
      for (i = i1; i <= i2 + 1; i++) {
        const double colfl = V(W->h_gesl, i) * CS(W->colls, i, j, n);
        const double colfr = V(W->h_gesr, i) * CS(W->colrs, i, j, n);
        CS(W->colf, i, j, n) = V(W->h_sl, i) * colfl + V(W->h_sr, i) * colfr;
      }
    if (P->dual == 1) {
      for (i = i1; i <= i2 + 1; i++)
        V(W->h_pcent, i) = fmax2((gamma - 1.0) * S(W->ge, i, j) * S(W->d, i, j), F_TINY);
      for (i = i1; i <= i2 + 1; i++) {
        double qc = dt / V(dx, i);
        S(W->ges, i, j) = qc * V(W->h_pcent, i) *
                          (V(W->h_sl, i) * V(W->h_gesl, i) + V(W->h_sr, i) * V(W->h_gesr, i) -
                           V(W->h_sl, i + 1) * V(W->h_gesl, i + 1) -
                           V(W->h_sr, i + 1) * V(W->h_gesr, i + 1));
      }
    }
    for (i = i1; i <= i2 + 1; i++) {
      double qc = dt / V(dx, i);
      S(W->df, i, j) = qc * S(W->df, i, j);
      S(W->uf, i, j) = qc * S(W->uf, i, j);
      S(W->vf, i, j) = qc * S(W->vf, i, j);
      S(W->wf, i, j) = qc * S(W->wf, i, j);
      S(W->ef, i, j) = qc * S(W->ef, i, j);
    }
    if (P->dual == 1)
      for (i = i1; i <= i2 + 1; i++) S(W->gef, i, j) = dt / V(dx, i) * S(W->gef, i, j);
    for (int n = 0; n < W->ncol; n++)
      for (i = i1; i <= i2 + 1; i++) CS(W->colf, i, j, n) = dt * CS(W->colf, i, j, n);
    /* flux_hll.F:336-383 / flux_hllc.F:331-389 */
    for (i = i1; i <= i2; i++) {
      if (S(W->d, i, j) + S(W->df, i, j) - S(W->df, i + 1, j) <= 0.0) {
        if (!hllc || P->fallback == 0) {
          rc = -1;
          if (st) st->fatal = 1;
        } else {
          if (st) st->fallbacks += 1;
          if (flux_hll_cell(W, P, dx, i, j, i2) != 0) {
            rc = -1;
            if (st) st->fatal = 1;
          }
        }
      }
    }
  }
  return rc;
}

/* ------------------------------------------------------------------------ */
/* flux_twoshock.F:6-490 (RAREFACTION2, no diffusion)                        */
/* ------------------------------------------------------------------------ */
static int flux_twoshock(work_t *W, const ora_params *P, const double *dx, int i1, int i2,
                         int j1, int j2, ora_stats *st) {
  const int idim = W->idim;
  const double gamma = P->gamma, dt = P->dt;
  const double qa = (gamma + 1.0) / (2.0 * gamma);
  int i, j, rc = 0;
  for (j = j1; j <= j2; j++) {
    for (i = i1; i <= i2 + 1; i++) {
      V(W->sn, i) = fsign1(-S(W->ubar, i, j));
      if (V(W->sn, i) < 0.0) {
        V(W->u0, i) = S(W->uls, i, j);
        V(W->p0, i) = S(W->pls, i, j);
        V(W->d0, i) = S(W->dls, i, j);
      } else {
        V(W->u0, i) = S(W->urs, i, j);
        V(W->p0, i) = S(W->prs, i, j);
        V(W->d0, i) = S(W->drs, i, j);
      }
      V(W->fc0, i) = sqrt(fmax2(gamma * V(W->p0, i) / V(W->d0, i), F_TINY));
      V(W->z0, i) = V(W->fc0, i) * V(W->d0, i) *
                    sqrt(fmax2(1.0 + qa * (S(W->pbar, i, j) / V(W->p0, i) - 1.0), F_TINY));
    }
    for (i = i1; i <= i2 + 1; i++) {
      V(W->dbar, i) = 1.0 / (1.0 / V(W->d0, i) - (S(W->pbar, i, j) - V(W->p0, i)) /
                                                  fmax2(V(W->z0, i) * V(W->z0, i), F_TINY));
      V(W->cbar, i) = sqrt(fmax2(gamma * S(W->pbar, i, j) / V(W->dbar, i), F_TINY));
    }
    for (i = i1; i <= i2 + 1; i++) {
      if (S(W->pbar, i, j) < V(W->p0, i)) {
        V(W->l0, i) = V(W->u0, i) * V(W->sn, i) + V(W->fc0, i);
        V(W->lbar, i) = V(W->sn, i) * S(W->ubar, i, j) + V(W->cbar, i);
      } else {
        V(W->l0, i) = V(W->u0, i) * V(W->sn, i) + V(W->z0, i) / V(W->d0, i);
        V(W->lbar, i) = V(W->l0, i);
      }
      double frac = V(W->l0, i) - V(W->lbar, i);
      if (frac < F_TINY) frac = F_TINY;
      frac = (0.0 - V(W->lbar, i)) / frac;
      frac = fmin2(fmax2(frac, 0.0), 1.0);
      V(W->pb, i) = V(W->p0, i) * frac + S(W->pbar, i, j) * (1.0 - frac);
      V(W->db, i) = V(W->d0, i) * frac + V(W->dbar, i) * (1.0 - frac);
      V(W->ub, i) = V(W->u0, i) * frac + S(W->ubar, i, j) * (1.0 - frac);
    }
    for (i = i1; i <= i2 + 1; i++) {
      if (V(W->lbar, i) >= 0.0) {
        V(W->pb, i) = S(W->pbar, i, j);
        V(W->db, i) = V(W->dbar, i);
        V(W->ub, i) = S(W->ubar, i, j);
      }
      if (V(W->l0, i) < 0.0) {
        V(W->pb, i) = V(W->p0, i);
        V(W->db, i) = V(W->d0, i);
        V(W->ub, i) = V(W->u0, i);
      }
    }
    for (i = i1; i <= i2 + 1; i++) {
      if (V(W->ub, i) > 0.0) {
        V(W->vb, i) = S(W->vls, i, j);
        V(W->wb, i) = S(W->wls, i, j);
        V(W->geb, i) = S(W->gels, i, j);
      } else {
        V(W->vb, i) = S(W->vrs, i, j);
        V(W->wb, i) = S(W->wrs, i, j);
        V(W->geb, i) = S(W->gers, i, j);
      }
    }
    /* colours at the Godunov state, flux_twoshock.F:251-259 */
    for (int n = 0; n < W->ncol; n++) {
      for (i = i1; i <= i2 + 1; i++) {
        if (V(W->ub, i) > 0.0)
          CV(W->colb, i, n) = CS(W->colls, i, j, n) * V(W->db, i) / S(W->dls, i, j);
        else
          CV(W->colb, i, n) = CS(W->colrs, i, j, n) * V(W->db, i) / S(W->drs, i, j);
      }
    }
    for (i = i1; i <= i2 + 1; i++) {
      V(W->eb, i) = V(W->pb, i) / ((gamma - 1.0) * V(W->db, i)) +
                    0.5 * (V(W->ub, i) * V(W->ub, i) + V(W->vb, i) * V(W->vb, i) + V(W->wb, i) * V(W->wb, i));
    }
    for (i = i1; i <= i2 + 1; i++) {
      V(W->upb, i) = V(W->pb, i) * V(W->ub, i);
      V(W->dub, i) = V(W->ub, i) * V(W->db, i);
      V(W->duub, i) = V(W->dub, i) * V(W->ub, i);
      V(W->duvb, i) = V(W->dub, i) * V(W->vb, i);
      V(W->duwb, i) = V(W->dub, i) * V(W->wb, i);
      V(W->dueb, i) = V(W->dub, i) * V(W->eb, i);
    }
    if (P->dual == 1)
      for (i = i1; i <= i2 + 1; i++) V(W->dugeb, i) = V(W->dub, i) * V(W->geb, i);
    for (i = i1; i <= i2 + 1; i++) {
      double qc = dt / V(dx, i);
      S(W->df, i, j) = qc * V(W->dub, i);
      S(W->ef, i, j) = qc * (V(W->dueb, i) + V(W->upb, i));
      S(W->uf, i, j) = qc * (V(W->duub, i) + V(W->pb, i));
      S(W->vf, i, j) = qc * V(W->duvb, i);
      S(W->wf, i, j) = qc * V(W->duwb, i);
    }
    /* colour fluxes times dt only, flux_twoshock.F:375-380 */
    for (int n = 0; n < W->ncol; n++)
      for (i = i1; i <= i2 + 1; i++)
        CS(W->colf, i, j, n) = dt * V(W->ub, i) * CV(W->colb, i, n);
    if (P->dual == 1) {
      for (i = i1; i <= i2 + 1; i++)
        V(W->pcent, i) = fmax2((gamma - 1.0) * S(W->ge, i, j) * S(W->d, i, j), F_TINY);
      /* ub(i2+2) is never set by the reference either; ges(i2+1) is not consumed */
      V(W->ub, i2 + 2) = 0.0;
      for (i = i1; i <= i2 + 1; i++) {
        double qc = dt / V(dx, i);
        S(W->gef, i, j) = qc * V(W->dugeb, i);
        S(W->ges, i, j) = qc * V(W->pcent, i) * (V(W->ub, i) - V(W->ub, i + 1));
      }
    }
    /* negative-state check and per-cell HLL fallback, flux_twoshock.F:401-456 */
    for (i = i1; i <= i2; i++) {
      if (S(W->d, i, j) + (S(W->df, i, j) - S(W->df, i + 1, j)) <= 0.0 || S(W->e, i, j) < 0.0) {
        if (P->fallback == 0) {
          rc = -1;
          if (st) st->fatal = 1;
        } else {
          if (st) st->fallbacks += 1;
          if (flux_hll_cell(W, P, dx, i, j, i2) != 0) {
            rc = -1;
            if (st) st->fatal = 1;
          }
        }
      }
    }
  }
  return rc;
}

/* ------------------------------------------------------------------------ */
/* euler.F:7-285 (GRAVITY_METHOD1, no second-order gravity correction,       */
/* no diffusion)                                                             */
/* ------------------------------------------------------------------------ */
static int euler(work_t *W, const ora_params *P, const double *dx, int i1, int i2, int j1, int j2,
                 ora_stats *st) {
  const int idim = W->idim;
  const double dt = P->dt, dfloor = P->small_rho;
  int i, j, rc = 0;
  for (j = j1; j <= j2; j++) {
    for (i = i1; i <= i2; i++) {
      V(W->dnu, i) = S(W->d, i, j) + (S(W->df, i, j) - S(W->df, i + 1, j));
      V(W->dnuinv, i) = 1.0 / V(W->dnu, i);
      if (dfloor > 0.0) {
        V(W->dnu, i) = fmax2(V(W->dnu, i), dfloor);
        V(W->dnuinv, i) = 1.0 / V(W->dnu, i);
      }
      V(W->uold, i) = S(W->u, i, j);
      S(W->u, i, j) = (S(W->u, i, j) * S(W->d, i, j) + (S(W->uf, i, j) - S(W->uf, i + 1, j))) * V(W->dnuinv, i);
      S(W->v, i, j) = (S(W->v, i, j) * S(W->d, i, j) + (S(W->vf, i, j) - S(W->vf, i + 1, j))) * V(W->dnuinv, i);
      S(W->w, i, j) = (S(W->w, i, j) * S(W->d, i, j) + (S(W->wf, i, j) - S(W->wf, i + 1, j))) * V(W->dnuinv, i);
      S(W->e, i, j) = fmax2(0.1 * S(W->e, i, j),
                            (S(W->e, i, j) * S(W->d, i, j) + (S(W->ef, i, j) - S(W->ef, i + 1, j))) * V(W->dnuinv, i));
    }
    if (P->dual == 1) {
      for (i = i1; i <= i2; i++) {
        S(W->ge, i, j) = fmax2((S(W->ge, i, j) * S(W->d, i, j) + (S(W->gef, i, j) - S(W->gef, i + 1, j)) +
                                S(W->ges, i, j)) * V(W->dnuinv, i),
                               0.5 * S(W->ge, i, j));
        if (S(W->ge, i, j) < 0.0) {
          rc = -1;
          if (st) st->fatal = 1;
        }
      }
    }
    if (P->gravity == 1) {
      for (i = i1; i <= i2; i++) {
        S(W->u, i, j) = S(W->u, i, j) + dt * S(W->gr, i, j) * 0.5 * (S(W->d, i, j) * V(W->dnuinv, i) + 1.0);
        S(W->e, i, j) = S(W->e, i, j) + dt * S(W->gr, i, j) * 0.5 *
                                            (S(W->u, i, j) + V(W->uold, i) * S(W->d, i, j) * V(W->dnuinv, i));
        S(W->e, i, j) = fmax2(S(W->e, i, j), F_TINY);
      }
    }
    /* colours, euler.F:171-186: colf divided by dx in place (the subgrid flux capture
       reads it afterwards), then the advective update with its floor */
    for (int n = 0; n < W->ncol; n++)
      for (i = i1; i <= i2 + 1; i++) CS(W->colf, i, j, n) = CS(W->colf, i, j, n) / V(dx, i);
    for (int n = 0; n < W->ncol; n++)
      for (i = i1; i <= i2; i++) {
        CS(W->col, i, j, n) = CS(W->col, i, j, n) + (CS(W->colf, i, j, n) - CS(W->colf, i + 1, j, n));
        CS(W->col, i, j, n) = fmax2(CS(W->col, i, j, n), F_MIN_COLOR);
      }
    for (i = i1; i <= i2; i++) S(W->d, i, j) = V(W->dnu, i);
  }
  return rc;
}

/* ------------------------------------------------------------------------ */
/* pgas2d_dual.F:4-122 (pressure output discarded by the caller)             */
/* ------------------------------------------------------------------------ */
static void pgas2d_dual(work_t *W, const ora_params *P, int i1, int i2, int j1, int j2) {
  const int idim = W->idim;
  const double gamma = P->gamma, eta1 = P->eta1, eta2 = P->eta2, pmin = P->tiny_number;
  int i, j;
  for (j = j1; j <= j2; j++) {
    for (i = i1; i <= i2; i++) {
      double ke = 0.5 * (S(W->u, i, j) * S(W->u, i, j) + S(W->v, i, j) * S(W->v, i, j) +
                         S(W->w, i, j) * S(W->w, i, j));
      double ge1 = S(W->e, i, j) - ke;
      int im1 = i - 1 > i1 ? i - 1 : i1;
      int ip1 = i + 1 < i2 ? i + 1 : i2;
      double demax = fmax2(fmax2(S(W->d, i, j) * S(W->e, i, j), S(W->d, im1, j) * S(W->e, im1, j)),
                           S(W->d, ip1, j) * S(W->e, ip1, j));
      if (ge1 * S(W->d, i, j) / demax > eta2) S(W->ge, i, j) = ge1;
      double ge2;
      if (ge1 / S(W->e, i, j) > eta1)
        ge2 = ge1;
      else
        ge2 = S(W->ge, i, j);
      ge2 = fmax2(ge2, pmin / ((gamma - 1.0) * S(W->d, i, j)));
      S(W->e, i, j) = S(W->e, i, j) - ge1 + ge2;
      S(W->p, i, j) = (gamma - 1.0) * S(W->d, i, j) * ge2;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Grid_ComputePressure.C:96-164 (time == Time, EOSType 0, no MHD/CR)        */
/* ------------------------------------------------------------------------ */
void ora_compute_pressure(const ora_params *P, double *const F[ORA_NFIELD], double *pressure) {
  size_t size = 1;
  for (int dim = 0; dim < P->rank; dim++) size *= (size_t)P->dims[dim];
  const double Gamma = P->gamma;
  for (size_t i = 0; i < size; i++) {
    double density = F[ORA_D][i];
    double gas_energy;
    if (P->eos_type == 3) {
      /* Grid_ComputePressure.C:112-124 with hydro_rk/EOS.h type 3: the pressure from the
         density and the total energy reset to the EOS energy plus the kinetic one */
      double velocity1 = F[ORA_V1][i], velocity2 = 0.0, velocity3 = 0.0;
      if (P->max_velocity_index > 1) velocity2 = F[ORA_V2][i];
      if (P->max_velocity_index > 2) velocity3 = F[ORA_V3][i];
      const double cs = P->eos_sound_speed;
      const double p = density * cs * cs;
      const double e = p / ((Gamma - 1.0) * density);
      pressure[i] = p;
      F[ORA_TE][i] = e + 0.5 * (velocity1 * velocity1 + velocity2 * velocity2 +
                                velocity3 * velocity3);
      continue;
    }
    if (P->dual == 0) {
      double velocity1 = F[ORA_V1][i], velocity2 = 0.0, velocity3 = 0.0;
      if (P->max_velocity_index > 1) velocity2 = F[ORA_V2][i];
      if (P->max_velocity_index > 2) velocity3 = F[ORA_V3][i];
      gas_energy = F[ORA_TE][i] - 0.5 * (velocity1 * velocity1 + velocity2 * velocity2 +
                                         velocity3 * velocity3);
    } else {
      gas_energy = F[ORA_GE][i];
    }
    pressure[i] = (Gamma - 1.0) * density * gas_energy;
    if (pressure[i] < P->tiny_number) pressure[i] = P->tiny_number;
    double min_pressure = P->min_support * (Gamma - 1.0) * density * density;
    if (pressure[i] < min_pressure) pressure[i] = min_pressure;
  }
}

/* ------------------------------------------------------------------------ */
/* sweep drivers: gather / solve / capture / scatter                         */
/* (Grid_xEulerSweep.C:33-463 and the y/z permutations)                      */
/* ------------------------------------------------------------------------ */

/* geometry of the direction-dim slices: the slice is (idim = GD[dim],
   jdim = GD[nd]) and slice index s runs over GD[sd]. */
static void sweep_axes(int dim, int *nd, int *sd) {
  if (dim == 0) { *nd = 1; *sd = 2; }
  else if (dim == 1) { *nd = 2; *sd = 0; }
  else { *nd = 0; *sd = 1; }
}

static inline size_t gidx(const int *GD, int dim, int a, int b, int s) {
  /* a: position along dim, b: along the slice's second axis, s: slice index */
  int ijk[3];
  int nd, sd;
  sweep_axes(dim, &nd, &sd);
  ijk[dim] = a;
  ijk[nd] = b;
  ijk[sd] = s;
  return ((size_t)ijk[2] * (size_t)GD[1] + (size_t)ijk[1]) * (size_t)GD[0] + (size_t)ijk[0];
}

static int sweep_slice(work_t *W, int dim, int s, const ora_params *P, double *const F[],
                       const double *pressure, double *const accel[3], double *const cw[3],
                       int nsub, ora_fluxes *sub, const long long ggs[3], ora_stats *st) {
  const int *GD = P->dims;
  int nd, sd;
  sweep_axes(dim, &nd, &sd);
  const int idim = GD[dim], jdim = GD[nd];
  const int rank = P->rank;
  /* velocity roles: x (u,v,w)=(1,2,3); y (w,u,v); z (v,w,u) */
  int vu, vv, vw; /* field slot feeding uslice/vslice/wslice */
  int hu, hv, hw; /* whether the slot exists for this rank */
  if (dim == 0) { vu = ORA_V1; vv = ORA_V2; vw = ORA_V3; hu = 1; hv = rank > 1; hw = rank > 2; }
  else if (dim == 1) { vu = ORA_V2; vv = ORA_V3; vw = ORA_V1; hu = rank > 1; hv = rank > 2; hw = 1; }
  else { vu = ORA_V3; vv = ORA_V1; vw = ORA_V2; hu = rank > 2; hv = 1; hw = rank > 1; }
  int a, b;
  for (b = 0; b < jdim; b++) {
    for (a = 0; a < idim; a++) {
      size_t g = gidx(GD, dim, a, b, s);
      size_t l = (size_t)b * idim + a;
      W->d[l] = F[ORA_D][g];
      W->e[l] = F[ORA_TE][g];
      W->p[l] = pressure[g];
      W->u[l] = hu ? F[vu][g] : 0.0;
      W->v[l] = hv ? F[vv][g] : 0.0;
      W->w[l] = hw ? F[vw][g] : 0.0;
      if (P->gravity) W->gr[l] = accel[dim][g];
      if (P->dual) W->ge[l] = F[ORA_GE][g];
      for (int n = 0; n < W->ncol; n++)  /* Grid_xEulerSweep.C:124-132 */
        W->col[(size_t)n * (size_t)idim * (size_t)jdim + l] = F[ORA_NFIELD + n][g];
    }
  }
  const int is = P->start[dim] + 1, ie = P->end[dim] + 1, js = 1, je = jdim;
  const double *dx = cw[dim];
  int rc = 0;
  inteuler(W, P, dx, is, ie, js, je);
  /* the solver switch of Grid_xEulerSweep.C:223-283 */
  if (P->riemann == ORA_RIEMANN_HLL || P->riemann == ORA_RIEMANN_HLLC) {
    if (flux_hll_family(W, P, dx, is, ie, js, je, P->riemann == ORA_RIEMANN_HLLC, st) != 0)
      rc = -1;
  } else {
    twoshock(W, P, is, ie + 1, js, je, st);
    if (flux_twoshock(W, P, dx, is, ie, js, je, st) != 0) rc = -1;
  }
  if (euler(W, P, dx, is, ie, js, je, st) != 0) rc = -1;
  if (P->dual) pgas2d_dual(W, P, is - 3, ie + 3, js, je);

  /* subgrid flux capture, Grid_xEulerSweep.C:313-377 */
  const int nxz = P->end[0] - P->start[0] + 1;
  const int nyz = P->end[1] - P->start[1] + 1;
  const int nzz = P->end[2] - P->start[2] + 1;
  const int nact[3] = {nxz, nyz, nzz};
  for (int n = 0; n < nsub; n++) {
    ora_fluxes *fx = &sub[n];
    /* (idim_axis, jdim_axis) of the flux face plane as in the reference */
    int ia, ja;
    if (dim == 0) { ia = 1; ja = 2; }
    else if (dim == 1) { ia = 0; ja = 2; }
    else { ia = 0; ja = 1; }
    long long fistart = fx->right_start[dim][ia] - ggs[ia];
    long long fiend = fx->right_end[dim][ia] - ggs[ia];
    long long fjstart = fx->right_start[dim][ja] - ggs[ja];
    long long fjend = fx->right_end[dim][ja] - ggs[ja];
    long long nfi = fiend - fistart + 1;
    long long lface = fx->left_start[dim][dim] - ggs[dim];
    long long rface = fx->right_start[dim][dim] - ggs[dim] + 1;
    /* the slice index s is the coordinate along sd; pencils run along nd */
    for (b = 0; b < jdim; b++) {
      int c[3];
      c[sd] = s;
      c[nd] = b;
      if (c[ia] < fistart || c[ia] > fiend || c[ja] < fjstart || c[ja] > fjend) continue;
      long long offset = (c[ia] - fistart) + (c[ja] - fjstart) * nfi;
      size_t li = (size_t)b * idim + (size_t)lface;
      size_t ri = (size_t)b * idim + (size_t)rface;
      fx->left[ORA_D][dim][offset] = W->df[li];
      fx->right[ORA_D][dim][offset] = W->df[ri];
      fx->left[ORA_TE][dim][offset] = W->ef[li];
      fx->right[ORA_TE][dim][offset] = W->ef[ri];
      /* velocity component c <- slice role; transverse only if active > 1 */
      const double *roles[3] = {W->uf, W->vf, W->wf};
      const int slot_of_role[3] = {vu, vv, vw};
      for (int r = 0; r < 3; r++) {
        int comp = slot_of_role[r] - ORA_V1;
        if (r != 0 && nact[comp] <= 1) continue;
        fx->left[slot_of_role[r]][dim][offset] = roles[r][li];
        fx->right[slot_of_role[r]][dim][offset] = roles[r][ri];
      }
      if (P->dual) {
        fx->left[ORA_GE][dim][offset] = W->gef[li];
        fx->right[ORA_GE][dim][offset] = W->gef[ri];
      }
      for (int n = 0; n < W->ncol; n++) {  /* Grid_xEulerSweep.C:361-371 */
        const size_t cn = (size_t)n * (size_t)idim * (size_t)jdim;
        if (fx->colour_left[n][dim]) fx->colour_left[n][dim][offset] = W->colf[cn + li];
        if (fx->colour_right[n][dim]) fx->colour_right[n][dim][offset] = W->colf[cn + ri];
      }
    }
  }

  /* scatter, Grid_xEulerSweep.C:381-417 */
  for (b = 0; b < jdim; b++) {
    for (a = 0; a < idim; a++) {
      size_t g = gidx(GD, dim, a, b, s);
      size_t l = (size_t)b * idim + a;
      F[ORA_D][g] = W->d[l];
      F[ORA_TE][g] = W->e[l];
      if (hu) F[vu][g] = W->u[l];
      if (hv) F[vv][g] = W->v[l];
      if (hw) F[vw][g] = W->w[l];
      if (P->dual) F[ORA_GE][g] = W->ge[l];
      for (int n = 0; n < W->ncol; n++)
        F[ORA_NFIELD + n][g] = W->col[(size_t)n * (size_t)idim * (size_t)jdim + l];
    }
  }
  return rc;
}

int ora_sweep(int dim, const ora_params *P, double *const F[], const double *pressure,
              double *const accel[3], double *const cw[3], int nsub, ora_fluxes *sub,
              const long long ggs[3], ora_stats *st, int nthreads) {
  int nd, sd;
  sweep_axes(dim, &nd, &sd);
  const int nslices = P->dims[sd];
  int rc = 0;
  (void)nthreads;
#ifdef _OPENMP
  if (nthreads > 1 && nsub == 0 && !g_log_fn) {
    int err = 0;
    long long fb = 0, itf = 0, itn = 0, hist[8] = {0};
    int fatal = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : fb, itf, itn) reduction(| : err, fatal)
    {
      work_t W;
      ora_stats lst;
      memset(&lst, 0, sizeof(lst));
      if (work_alloc(&W, P->dims[dim], P->dims[nd], P->ncolour) != 0) {
        err |= 1;
      } else {
#pragma omp for schedule(dynamic, 1)
        for (int s = 0; s < nslices; s++)
          if (sweep_slice(&W, dim, s, P, F, pressure, accel, cw, 0, 0, ggs, &lst) != 0) err |= 1;
        work_free(&W);
      }
      fb += lst.fallbacks;
      itf += lst.interfaces;
      itn += lst.newton_iters;
      fatal |= lst.fatal;
#pragma omp critical
      for (int h = 0; h < 8; h++) hist[h] += lst.newton_hist[h];
    }
    if (st) {
      st->fallbacks += fb;
      st->interfaces += itf;
      st->newton_iters += itn;
      st->fatal |= fatal;
      for (int h = 0; h < 8; h++) st->newton_hist[h] += hist[h];
    }
    return err ? -1 : 0;
  }
#endif
  work_t W;
  if (work_alloc(&W, P->dims[dim], P->dims[nd], P->ncolour) != 0) return -2;
  for (int s = 0; s < nslices; s++)
    if (sweep_slice(&W, dim, s, P, F, pressure, accel, cw, nsub, sub, ggs, st) != 0) rc = -1;
  work_free(&W);
  return rc;
}

int ora_solve_ppm_de(const ora_params *P, int cycle, double *const F[],
                     double *const accel[3], double *const cw[3], int nsub, ora_fluxes *sub,
                     const long long ggs[3], ora_stats *st, int nthreads) {
  ora_params Q = *P;
  for (int d = P->rank; d < 3; d++) {
    Q.dims[d] = 1;
    Q.start[d] = 0;
    Q.end[d] = 0;
  }
  size_t size = 1;
  for (int d = 0; d < 3; d++) size *= (size_t)Q.dims[d];
  double *pressure = (double *)calloc(size, sizeof(double));
  if (!pressure) return -2;
  ora_compute_pressure(&Q, F, pressure);
  const int nxz = Q.end[0] - Q.start[0] + 1;
  const int nyz = Q.end[1] - Q.start[1] + 1;
  const int nzz = Q.end[2] - Q.start[2] + 1;
  const int ixyz = cycle % Q.rank;
  int rc = 0;
  for (int n = ixyz; n < ixyz + Q.rank; n++) {
    if ((n % Q.rank == 0) && nxz > 1)
      if (ora_sweep(0, &Q, F, pressure, accel, cw, nsub, sub, ggs, st, nthreads) != 0) rc = -1;
    if ((n % Q.rank == 1) && nyz > 1)
      if (ora_sweep(1, &Q, F, pressure, accel, cw, nsub, sub, ggs, st, nthreads) != 0) rc = -1;
    if ((n % Q.rank == 2) && nzz > 1)
      if (ora_sweep(2, &Q, F, pressure, accel, cw, nsub, sub, ggs, st, nthreads) != 0) rc = -1;
  }
  /* energies consistent with the EOS again, Grid_SolvePPM_DE.C:155-157 */
  if (Q.eos_type > 0) ora_compute_pressure(&Q, F, pressure);
  free(pressure);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* calc_dt.F:6-181 (ihydro = 0)                                              */
/* ------------------------------------------------------------------------ */
double ora_calc_dt(const ora_params *P, double *const F[ORA_NFIELD], const double *p,
                   double *const cw[3], double aye, const double vg[3]) {
  const int *GD = P->dims;
  const int idim = GD[0], jdim = P->rank > 1 ? GD[1] : 1;
  const double gamma = P->gamma;
  double dt = F_HUGE;
  const double *d = F[ORA_D], *u = F[ORA_V1];
  const double *v = P->rank > 1 ? F[ORA_V2] : 0, *w = P->rank > 2 ? F[ORA_V3] : 0;
  const int kmax = P->rank > 2 ? P->end[2] : 0, kmin = P->rank > 2 ? P->start[2] : 0;
  const int jmax = P->rank > 1 ? P->end[1] : 0, jmin = P->rank > 1 ? P->start[1] : 0;
  for (int k = kmin; k <= kmax; k++)
    for (int j = jmin; j <= jmax; j++)
      for (int i = P->start[0]; i <= P->end[0]; i++) {
        size_t g = ((size_t)k * jdim + j) * idim + i;
        double cs = fmax2(sqrt(gamma * p[g] / d[g]), F_TINY);
        if (P->pressure_free == 1) cs = F_TINY;
        double dt1;
        if (P->rank == 1) {
          dt1 = cw[0][i] * aye / (cs + fabs(u[g] - vg[0]));
        } else if (P->rank == 2) {
          dt1 = aye / ((cs + fabs(u[g] - vg[0])) / cw[0][i] + (cs + fabs(v[g] - vg[1])) / cw[1][j]);
        } else {
          dt1 = aye / ((cs + fabs(u[g] - vg[0])) / cw[0][i] + (cs + fabs(v[g] - vg[1])) / cw[1][j] +
                       (cs + fabs(w[g] - vg[2])) / cw[2][k]);
        }
        dt = fmin2(dt, dt1);
      }
  return dt;
}

/* ------------------------------------------------------------------------ */
/* comoving expansion terms                                                  */
/* ------------------------------------------------------------------------ */

/* Grid_ComputePressure.C:51-58 and :168-223 (time strictly between OldTime and Time). */
static void pressure_interpolated(const ora_params *P, double *const F[ORA_NFIELD],
                                  double *const O[ORA_NFIELD], double time, double Time,
                                  double OldTime, double *pressure) {
  size_t size = 1;
  for (int dim = 0; dim < P->rank; dim++) size *= (size_t)P->dims[dim];
  const double Gamma = P->gamma;
  double coef, coefold;
  if (Time - OldTime > 0)
    coef = (time - OldTime) / (Time - OldTime);
  else
    coef = 1;
  coefold = 1 - coef;
  for (size_t i = 0; i < size; i++) {
    double velocity2 = 0.0, velocity3 = 0.0, gas_energy;
    double total_energy = coef * F[ORA_TE][i] + coefold * O[ORA_TE][i];
    double density = coef * F[ORA_D][i] + coefold * O[ORA_D][i];
    double velocity1 = coef * F[ORA_V1][i] + coefold * O[ORA_V1][i];
    if (P->max_velocity_index > 1) velocity2 = coef * F[ORA_V2][i] + coefold * O[ORA_V2][i];
    if (P->max_velocity_index > 2) velocity3 = coef * F[ORA_V3][i] + coefold * O[ORA_V3][i];
    if (P->dual == 0) {
      double kineticE = 0.5 * (velocity1 * velocity1 + velocity2 * velocity2 +
                               velocity3 * velocity3);
      gas_energy = total_energy - kineticE;
    } else {
      gas_energy = coef * F[ORA_GE][i] + coefold * O[ORA_GE][i];
    }
    pressure[i] = (Gamma - 1.0) * density * gas_energy;
    if (pressure[i] < P->tiny_number) pressure[i] = P->tiny_number;
    double min_pressure = P->min_support * (Gamma - 1.0) * density * density;
    if (pressure[i] < min_pressure) pressure[i] = min_pressure;
  }
}

void ora_expansion_terms(const ora_params *P, double *const F[ORA_NFIELD],
                         double *const O[ORA_NFIELD], double Time, double OldTime,
                         double coefficient) {
  size_t size = 1;
  for (int dim = 0; dim < P->rank; dim++) size *= (size_t)P->dims[dim];
  double *p = (double *)malloc(size * sizeof(double));
  /* Grid_ComovingExpansionTerms.C:84-89: the pressure at the mid time when the old
     fields exist, else at Time; ComputePressure's MinimumSupportEnergyCoefficient keeps
     its default 0 here (Grid.h:576-578) */
  ora_params Q = *P;
  Q.min_support = 0.0;
  if (O != NULL) {
    double PressureTime = 0.5 * (Time + OldTime);
    if (PressureTime == Time)
      ora_compute_pressure(&Q, F, p);
    else
      pressure_interpolated(&Q, F, O, PressureTime, Time, OldTime, p);
  } else {
    ora_compute_pressure(&Q, F, p);
  }
  const double coef = coefficient, gamma = P->gamma;
  double *d = F[ORA_D], *e = F[ORA_TE], *ge = F[ORA_GE];
  double *u = F[ORA_V1], *v = F[ORA_V2], *w = F[ORA_V3];
  /* expand_terms.F: gas energy, ENERGY_METHOD3 */
  if (P->dual == 1)
    for (size_t i = 0; i < size; i++) ge[i] = ge[i] * (1.0 - coef) / (1.0 + coef);
  /* total energy, ENERGY_METHOD3 (imethod != 2, no cosmic rays) */
  for (size_t i = 0; i < size; i++) {
    e[i] = e[i] * (1.0 - coef) / (1.0 + coef);
    double a = e[i] - coef * (3.0 - 2.0 / (gamma - 1.0)) * p[i] / d[i];
    double b = 0.5 * e[i];
    e[i] = a > b ? a : b; /* max(a, b) */
  }
  /* velocities, VELOCITY_METHOD3 */
  for (size_t i = 0; i < size; i++) {
    u[i] = u[i] * (1.0 - 0.5 * coef) / (1.0 + 0.5 * coef);
    if (P->rank > 1) v[i] = v[i] * (1.0 - 0.5 * coef) / (1.0 + 0.5 * coef);
    if (P->rank > 2) w[i] = w[i] * (1.0 - 0.5 * coef) / (1.0 + 0.5 * coef);
  }
  free(p);
}

/* ------------------------------------------------------------------------ */
/* Grid_CorrectForRefinedFluxes.C:38-760, proper subgrids, Cartesian         */
/* ------------------------------------------------------------------------ */
/* One call of grid::CorrectForRefinedFluxes (Grid_CorrectForRefinedFluxes.C:38-760) for
   one (initial, refined) pair.  subling: SUBlingGrid == TRUE, the refined fluxes of a
   sibling's subgrid projected to this level, I the grid's own boundary fluxes; gdims and
   periodic: the level's extent in zones and the periodic faces (:147-221). */
static int correct_one(const ora_params *P, double *const F[], const int *order,
                       int nf, const ora_fluxes *I, ora_fluxes *R, const long long gl[3],
                       int subling, const long long gdims[3], const int periodic[3]) {
  const int rank = P->rank;
  const int *GD = P->dims;
  for (int dim = 0; dim < rank; dim++) {
    if (GD[dim] <= 1) continue;
    int correct_left = 1, correct_right = 1;
    long long rls[3], rle[3];  /* the refined box as the routine sees it along dim */
    int RefinedDim[3] = {0, 0, 0}, RefinedOffset[3] = {0, 0, 0}, InitialOffset[3] = {0, 0, 0};
    for (int i = 0; i < 3; i++) {
      rls[i] = R->left_start[dim][i];
      rle[i] = R->left_end[dim][i];
    }
    if (subling) {
      const long long GlobalDim = gdims[dim];
      for (int i = 0; i < 3; i++)
        RefinedDim[i] = (int)(R->left_end[dim][i] - R->left_start[dim][i] + 1);
      long long rrs = R->right_start[dim][dim];
      /* a face on a periodic domain boundary wraps; otherwise step outward (:163-179) */
      if (rls[dim] == 0 && periodic[dim]) {
        rls[dim] = rle[dim] = GlobalDim - 1;
      } else {
        rls[dim]--;
        rle[dim]--;
      }
      if (rrs == GlobalDim - 1 && periodic[dim])
        rrs = 0;
      else
        rrs++;
      correct_right = I->right_start[dim][dim] == rls[dim];
      correct_left = I->left_start[dim][dim] == rrs;
      for (int i = 0; i < 3; i++) {
        const long long d = I->left_start[dim][i] - rls[i];
        RefinedOffset[i] = (int)(d > 0 ? d : 0);
      }
      rls[dim] = 0;
      RefinedOffset[dim] = 0;
    }
    if (!correct_left && !correct_right) continue;
    int Start[3] = {0, 0, 0}, End[3] = {0, 0, 0}, Dim[3];
    for (int i = 0; i < rank; i++) {
      const long long s0 = I->left_start[dim][i] > rls[i] ? I->left_start[dim][i] : rls[i];
      const long long e0 = I->left_end[dim][i] < rle[i] ? I->left_end[dim][i] : rle[i];
      Start[i] = (int)(s0 - gl[i]);
      End[i] = (int)(e0 - gl[i]);
      if (Start[i] < 0 || End[i] > GD[i]) return -1;
    }
    /* the layer just outside the left face (:225-230) */
    Start[dim] = Start[dim] - 1 > 0 ? Start[dim] - 1 : 0;
    End[dim] = Start[dim];
    for (int i = 0; i < 3; i++) Dim[i] = End[i] - Start[i] + 1;
    /* :234-237 */
    long long Offset = I->right_start[dim][dim] - I->left_start[dim][dim] + 2;
    if (Offset > GD[dim] - 1) Offset = GD[dim] - 1;
    if (subling) {  /* the grid's own edge layers (:284-305) */
      Offset -= 2;
      Start[dim]++;
      End[dim]++;
      for (int i = 0; i < rank; i++) {
        if (i != dim) {
          Dim[i] = P->end[i] - P->start[i] + 1;
          const long long d = rls[i] - I->left_start[dim][i];
          InitialOffset[i] = (int)(d > 0 ? d : 0);
        } else {
          Dim[i] = 1;
          InitialOffset[i] = 0;
        }
      }
    }
    /* a layer that is this grid's ghost zone is not corrected (:311-320) */
    if (Start[dim] == P->start[dim] - 1) correct_left = 0;
    if (Start[dim] + Offset == P->end[dim] + 1) correct_right = 0;
    for (int i = 0; i < dim; i++) Offset *= GD[i];
#define CELL(k, j, i) (((size_t)(k) * GD[1] + (j)) * GD[0] + (i))
#define FLUX(k, j, i)                                                                  \
  (((size_t)((k) - Start[2] + InitialOffset[2]) * Dim[1] + ((j) - Start[1] + InitialOffset[1])) * \
       Dim[0] + ((i) - Start[0] + InitialOffset[0]))
#define RFLUX(k, j, i)                                                                 \
  (((size_t)((k) - Start[2] + RefinedOffset[2]) * RefinedDim[1] +                      \
    ((j) - Start[1] + RefinedOffset[1])) * RefinedDim[0] + ((i) - Start[0] + RefinedOffset[0]))
    /* conserved quantities on both layers (:370-394): all but density */
    for (int q = 0; q < nf; q++) {
      const int f = order[q];
      if (f == ORA_D) continue;
      for (int k = Start[2]; k <= End[2]; k++)
        for (int j = Start[1]; j <= End[1]; j++)
          for (int i = Start[0]; i <= End[0]; i++) {
            const size_t c = CELL(k, j, i);
            F[f][c] *= F[ORA_D][c];
            F[f][c + Offset] *= F[ORA_D][c + Offset];
          }
    }
    /* species as fractions of the density (:397-421) */
    for (int n = 0; n < P->ncolour && P->colour_species; n++) {
      if (!P->colour_species[n]) continue;
      double *q = F[ORA_NFIELD + n];
      for (int k = Start[2]; k <= End[2]; k++)
        for (int j = Start[1]; j <= End[1]; j++)
          for (int i = Start[0]; i <= End[0]; i++) {
            const size_t c = CELL(k, j, i);
            q[c] /= F[ORA_D][c];
            q[c + Offset] /= F[ORA_D][c + Offset];
          }
    }
    /* the corrections with the undo for density and energies (:455-656) */
    for (int q = 0; q < nf; q++) {
      const int f = order[q];
      for (int k = Start[2]; k <= End[2]; k++)
        for (int j = Start[1]; j <= End[1]; j++)
          for (int i = Start[0]; i <= End[0]; i++) {
            const size_t c = CELL(k, j, i), x = FLUX(k, j, i);
            const size_t xr = subling ? RFLUX(k, j, i) : x;
            if (correct_left) {
              const double amount = subling ? -(I->left[f][dim][x] - R->right[f][dim][xr])
                                            : I->left[f][dim][x] - R->left[f][dim][x];
              F[f][c] += amount;
            }
            if (correct_right) {
              const double amount = subling ? I->right[f][dim][x] - R->left[f][dim][xr]
                                            : -(I->right[f][dim][x] - R->right[f][dim][x]);
              F[f][c + Offset] += amount;
            }
            if (f == ORA_D || f == ORA_TE || f == ORA_GE) {
              if (correct_left && F[f][c] <= 0) {
                for (int u = 0; u < nf; u++) {
                  const int g = order[u];
                  if (subling) {
                    if (u <= q) F[g][c] -= -(I->left[g][dim][x] - R->right[g][dim][xr]);
                    R->right[g][dim][xr] = I->left[g][dim][x];
                  } else {
                    if (u <= q) F[g][c] -= (I->left[g][dim][x] - R->left[g][dim][x]);
                    R->left[g][dim][x] = I->left[g][dim][x];
                  }
                }
              }
              if (correct_right && F[f][c + Offset] <= 0) {
                for (int u = 0; u < nf; u++) {
                  const int g = order[u];
                  if (subling) {
                    /* the reference subtracts the triggering field's amount from every
                       undone field here (:643-645) */
                    if (u <= q) F[g][c + Offset] -= (I->right[f][dim][x] - R->left[f][dim][xr]);
                    R->left[g][dim][xr] = I->right[g][dim][x];
                  } else {
                    if (u <= q) F[g][c + Offset] -= -(I->right[g][dim][x] - R->right[g][dim][x]);
                    R->right[g][dim][x] = I->right[g][dim][x];
                  }
                }
              }
            }
          }
    }
    /* back to specific quantities with the new density (:683-700) */
    for (int q = 0; q < nf; q++) {
      const int f = order[q];
      if (f == ORA_D) continue;
      for (int k = Start[2]; k <= End[2]; k++)
        for (int j = Start[1]; j <= End[1]; j++)
          for (int i = Start[0]; i <= End[0]; i++) {
            const size_t c = CELL(k, j, i);
            F[f][c] /= F[ORA_D][c];
            F[f][c + Offset] /= F[ORA_D][c + Offset];
          }
    }
    /* total and gas energy made consistent again (:704-742) */
    if (P->dual) {
      for (int k = Start[2]; k <= End[2]; k++)
        for (int j = Start[1]; j <= End[1]; j++)
          for (int i = Start[0]; i <= End[0]; i++) {
            const size_t c1 = CELL(k, j, i), c2 = c1 + Offset;
            F[ORA_GE][c1] = fmax2(F[ORA_GE][c1], P->tiny_number);
            F[ORA_GE][c2] = fmax2(F[ORA_GE][c2], P->tiny_number);
            F[ORA_TE][c1] = F[ORA_GE][c1] + 0.5 * F[ORA_V1][c1] * F[ORA_V1][c1];
            F[ORA_TE][c2] = F[ORA_GE][c2] + 0.5 * F[ORA_V1][c2] * F[ORA_V1][c2];
            if (rank > 1) {
              F[ORA_TE][c1] += 0.5 * F[ORA_V2][c1] * F[ORA_V2][c1];
              F[ORA_TE][c2] += 0.5 * F[ORA_V2][c2] * F[ORA_V2][c2];
            }
            if (rank > 2) {
              F[ORA_TE][c1] += 0.5 * F[ORA_V3][c1] * F[ORA_V3][c1];
              F[ORA_TE][c2] += 0.5 * F[ORA_V3][c2] * F[ORA_V3][c2];
            }
          }
    }
    /* species back to densities with the corrected density (:849-866) */
    for (int n = 0; n < P->ncolour && P->colour_species; n++) {
      if (!P->colour_species[n]) continue;
      double *q = F[ORA_NFIELD + n];
      for (int k = Start[2]; k <= End[2]; k++)
        for (int j = Start[1]; j <= End[1]; j++)
          for (int i = Start[0]; i <= End[0]; i++) {
            const size_t c = CELL(k, j, i);
            q[c] *= F[ORA_D][c];
            q[c + Offset] *= F[ORA_D][c + Offset];
          }
    }
#undef CELL
#undef FLUX
#undef RFLUX
  }
  return 0;
}

/* the fields in the order the routine corrects them: density and the energies first
   (:341-360), then the remaining fields in BaryonField order (:396-452) */
static int correction_order(const ora_params *P, double *const F[], int *order) {
  int nf = 0;
  const int base_order[ORA_NFIELD] = {ORA_D, ORA_TE, ORA_GE, ORA_V1, ORA_V2, ORA_V3};
  for (int q = 0; q < ORA_NFIELD; q++) {
    const int f = base_order[q];
    if (!F[f]) continue;
    if (f == ORA_GE && !P->dual) continue;
    if (f >= ORA_V1 && f <= ORA_V3 && f - ORA_V1 >= P->rank) continue;
    order[nf++] = f;
  }
  return nf;
}

int ora_correct_fluxes(const ora_params *P, double *const F[], int nsub,
                       const ora_fluxes *IN, ora_fluxes *RF, const long long gl[3]) {
  int order[ORA_NFIELD];
  const int nf = correction_order(P, F, order);
  for (int n = 0; n < nsub; n++)
    if (correct_one(P, F, order, nf, &IN[n], &RF[n], gl, 0, 0, 0) != 0) return -1;
  return 0;
}

int ora_correct_fluxes_sublings(const ora_params *P, double *const F[], int nsib,
                                const ora_fluxes *own, ora_fluxes *RF, const long long gl[3],
                                const long long gdims[3], const int periodic[3]) {
  int order[ORA_NFIELD];
  const int nf = correction_order(P, F, order);
  for (int n = 0; n < nsib; n++)
    if (correct_one(P, F, order, nf, own, &RF[n], gl, 1, gdims, periodic) != 0) return -1;
  return 0;
}
