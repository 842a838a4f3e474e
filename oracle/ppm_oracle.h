/*
 * ppm_oracle.h -- CPU oracle for the PPM-DE hydro hot path (TEST INFRASTRUCTURE).
 *
 * This is a plain-C, FP64 restatement of Enzo's directionally split PPM
 * "Direct Eulerian" solver (HydroMethod = 0), kept in the reference's
 * Fortran evaluation order and built without floating-point contraction.
 * It exists only to check the CUDA implementation: tests, the smoke check
 * and the CPU-baseline leg of the benchmark call it; the product library
 * never links or calls it.
 *
 * Reference routines restated (paths relative to the enzo-dev tree):
 *   grid::SolvePPM_DE          src/enzo/Grid_SolvePPM_DE.C:36-164
 *   grid::{x,y,z}EulerSweep    src/enzo/Grid_{x,y,z}EulerSweep.C
 *   inteuler / intvar          src/enzo/inteuler.F:5-566, intvar.F:5-179
 *   (colour fields: inteuler.F:276-282, :436-450, :500-515, :546-551,
 *    flux_twoshock.F:251-259, :375-380, flux_hll.F:236-262, euler.F:171-186,
 *    Grid_xEulerSweep.C:124-132, :361-371, :409-416)
 *   twoshock                   src/enzo/twoshock.F:5-276
 *   flux_twoshock / flux_hll   src/enzo/flux_twoshock.F:6-490, flux_hll.F:6-415
 *   flux_hllc                  src/enzo/flux_hllc.F:6-421 (RiemannSolver = HLLC)
 *   euler                      src/enzo/euler.F:7-285
 *   pgas2d_dual                src/enzo/pgas2d_dual.F:4-122
 *   grid::ComputePressure      src/enzo/Grid_ComputePressure.C:36-164
 *   calc_dt (PPM branch)       src/enzo/calc_dt.F:6-181
 *   calcdiss (flattening 1-3) src/enzo/calcdiss.F:213-224, 407-483, 486-559
 *   CorrectForRefinedFluxes    src/enzo/Grid_CorrectForRefinedFluxes.C:38-760
 *
 * Parity anchors: the reference's analytic shock-tube answer tests
 * (run/Hydro/Hydro-1D/{SodShockTube,Toro-*}) at the reference's own
 * tolerances; no bit-level golden output of the Fortran exists in the tree
 * and no Fortran compiler is available, so bit-level parity of this
 * restatement against the Fortran itself is unpinned.
 */
#ifndef PPM_ORACLE_H
#define PPM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* field slots, in BaryonField roles */
enum { ORA_D = 0, ORA_TE = 1, ORA_V1 = 2, ORA_V2 = 3, ORA_V3 = 4, ORA_GE = 5, ORA_NFIELD = 6 };
/* MAX_COLOR (fortran.def:2): colour fields follow the six hydro fields in the field
   array, fields[ORA_NFIELD + n] for n < ncolour (the colnum[] list of
   Grid_SolveHydroEquations.C:90-285, in that order) */
#define ORA_MAX_COLOUR 45

typedef struct {
  int rank;            /* GridRank (1..3) */
  int dims[3];         /* GridDimension, ghosts included */
  int start[3];        /* GridStartIndex, 0-based */
  int end[3];          /* GridEndIndex, 0-based inclusive */
  double gamma;        /* Gamma */
  double dt;           /* dtFixed */
  double eta1, eta2;   /* DualEnergyFormalismEta1/2 */
  double small_rho;    /* SmallRho: density floor applied in euler */
  double tiny_number;  /* tiny_number: MinimumPressure of the sweeps */
  double min_support;  /* MinimumSupportEnergyCoefficient (ComputePressure) */
  int dual;            /* DualEnergyFormalism */
  int gravity;         /* GravityOn */
  int pressure_free;   /* PressureFree */
  int fallback;        /* RiemannSolverFallback */
  int max_velocity_index; /* MaxVelocityIndex used by ComputePressure */
  int steepen;         /* PPMSteepeningParameter (0 or 1: density steepening) */
  int flatten;         /* PPMFlatteningParameter (0, 1, 2 or 3) */
  int ncolour;         /* NumberOfColours: advected colour fields after the hydro fields */
  int riemann;         /* RiemannSolver (typedefs.h:279-280): 5 TwoShock (0 taken as 5),
                          1 HLL, 4 HLLC */
  const int *colour_species; /* flux correction: ncolour flags, nonzero for a colour that
                                keeps its fraction of the corrected density; NULL: none */
  int eos_type;        /* EOSType: 0 ideal gas, 3 isothermal (hydro_rk/EOS.h) */
  double eos_sound_speed; /* EOSSoundSpeed */
} ora_params;

enum { ORA_RIEMANN_HLL = 1, ORA_RIEMANN_HLLC = 4, ORA_RIEMANN_TWOSHOCK = 5 };

/* struct fluxes (src/enzo/Fluxes.h:29-37), restricted to the six hydro slots */
typedef struct {
  long long left_start[3][3], left_end[3][3];
  long long right_start[3][3], right_end[3][3];
  double *left[ORA_NFIELD][3];
  double *right[ORA_NFIELD][3];
  /* LeftFluxes/RightFluxes[colnum[n]][dim] of the colour fields (NULL: not captured) */
  double *colour_left[ORA_MAX_COLOUR][3];
  double *colour_right[ORA_MAX_COLOUR][3];
} ora_fluxes;

typedef struct {
  long long interfaces;      /* Riemann problems solved */
  long long newton_iters;    /* total Newton updates */
  long long newton_hist[8];  /* [n] = interfaces that took n Newton updates (1..7) */
  long long fallbacks;       /* cells whose fluxes were recomputed with HLL */
  int fatal;                 /* 1 if a state the reference aborts on was met */
} ora_stats;

/* Optional hook: called for every Riemann problem with the six interface
   states and the converged pbar (training-data logging). */
typedef void (*ora_riemann_log_fn)(void *ctx, const double st[6], double pbar, int iters);

/* grid::ComputePressure at time == Time (Grid_ComputePressure.C:96-164). */
void ora_compute_pressure(const ora_params *P, double *const fields[ORA_NFIELD], double *pressure);

/* One directional sweep over all slices of the grid (dim 0,1,2), i.e. the
   `for k ... xEulerSweep(k)` loop of Grid_SolvePPM_DE.C:91-97 and its y/z
   siblings.  accel may be NULL when gravity is off.  fields: the six hydro fields,
   then P->ncolour colour fields. */
int ora_sweep(int dim, const ora_params *P, double *const fields[],
              const double *pressure, double *const accel[3],
              double *const cellwidth[3], int nsub, ora_fluxes *sub,
              const long long ggs[3], ora_stats *st, int nthreads);

/* grid::SolvePPM_DE (Grid_SolvePPM_DE.C:36-164), EOSType = 0. */
int ora_solve_ppm_de(const ora_params *P, int cycle, double *const fields[],
                     double *const accel[3], double *const cellwidth[3],
                     int nsub, ora_fluxes *sub, const long long ggs[3],
                     ora_stats *st, int nthreads);

/* calc_dt (rank 1..3, ihydro = 0) on a pressure field; returns dt without
   the Courant factor (calc_dt.F:6-181). */
double ora_calc_dt(const ora_params *P, double *const fields[ORA_NFIELD],
                   const double *pressure, double *const cellwidth[3],
                   double aye, const double vgrid[3]);

/* A single two-shock Riemann problem (twoshock.F:115-254 for one interface).
   st = {dl, dr, pl, pr, ul, ur}. If guess > 0 it replaces the acoustic
   starting pressure (learned-guess semantics; guess <= 0 = reference). */
void ora_twoshock_point(const double st[6], double gamma, double pmin, double guess,
                        double *pbar, double *ubar, int *iters);

void ora_set_riemann_log(ora_riemann_log_fn fn, void *ctx);

/* grid::ComovingExpansionTerms for PPM (Grid_ComovingExpansionTerms.C:36-99 with
   expand_terms.F, ENERGY_METHOD3 and VELOCITY_METHOD3): pressure at
   0.5*(time + old_time) interpolated between old and current fields
   (Grid_ComputePressure.C:51-58, :168-223) when old != NULL, else at time; then the
   expansion terms over every cell.  coefficient = dtFixed * adot / a. */
void ora_expansion_terms(const ora_params *P, double *const fields[ORA_NFIELD],
                         double *const old[ORA_NFIELD], double time, double old_time,
                         double coefficient);

/* grid::CorrectForRefinedFluxes (Grid_CorrectForRefinedFluxes.C:38-760) for the
   proper subgrids of one grid (SUBlingGrid == FALSE), Cartesian coordinates, the six
   hydro fields (no species or colours), RadiativeCooling == 0, CorrectParentBoundaryFlux
   == FALSE.  initial[n] / refined[n]: the subgrid's coarse and refined boundary fluxes
   (same index boxes); refined entries of undone corrections are set to the initial ones,
   as the reference does.  gl: global index of the grid's first zone (ghosts included).
   Returns 0, or -1 if a flux box does not fit the grid. */
int ora_correct_fluxes(const ora_params *P, double *const fields[], int nsub,
                       const ora_fluxes *initial, ora_fluxes *refined, const long long gl[3]);

/* The SUBling calls of grid::CorrectForRefinedFluxes (SUBlingGrid == TRUE,
   UpdateFromFinerGrids.C:176-206): for each sibling subgrid n, refined[n] holds its
   refined boundary fluxes projected to this level and `own` this grid's own boundary
   fluxes (SubgridFluxesEstimate[grid][NumberOfSubgrids - 1]); the grid's edge layers that
   touch the sibling's projected faces are corrected (Grid_CorrectForRefinedFluxes.C:147-
   305, :464-656).  gdims: the level's extent in zones per axis; periodic: periodic
   faces per axis.  refined[n]'s index boxes are not modified; its flux values are where a
   correction is undone.  Returns 0, or -1 if a flux box does not fit the grid. */
int ora_correct_fluxes_sublings(const ora_params *P, double *const fields[], int nsib,
                                const ora_fluxes *own, ora_fluxes *refined,
                                const long long gl[3], const long long gdims[3],
                                const int periodic[3]);

#ifdef __cplusplus
}
#endif
#endif
