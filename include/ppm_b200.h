/*
 * ppm_b200.h -- C ABI of the B200 PPM-DE hydro library.
 *
 * Drop-in replacement for the directionally split PPM "Direct Eulerian"
 * solver of Enzo (HydroMethod = 0).  The entry points mirror the reference's
 * own seam: grid::SolvePPM_DE (src/enzo/Grid_SolvePPM_DE.C:36) and the
 * per-direction sweep loops it runs (Grid_SolvePPM_DE.C:86-146, each a loop of
 * grid::{x,y,z}EulerSweep, src/enzo/Grid_xEulerSweep.C:33), and the
 * UseCUDA branch that the reference reserves for a GPU solver
 * (cuPPMInitParameter / cuPPMInitData / cuPPMSweep / cuPPMSaveSubgridFluxes /
 * cuPPMGetBaryon / cuPPMDestroy, src/enzo/cuPPM.h, called from
 * Grid_SolvePPM_DE.C:63-153).
 *
 * All arithmetic is FP64.  Fields keep Enzo's BaryonField layout: one array
 * per field, x fastest, index (k*GD1 + j)*GD0 + i, ghost zones included.
 * Subgrid fluxes keep the layout of struct fluxes (src/enzo/Fluxes.h:29-37).
 *
 * Plain pointers and sizes only: no C++ or CUDA types cross this boundary.
 * Every call returns PPM_B200_OK (0) or a negative PPM_B200_ERR_* code and
 * never exits or traps the GPU.
 */
#ifndef PPM_B200_H
#define PPM_B200_H

/* Enzo includes its headers with `#define int long_int` (LARGE_INTS, which the
   default CONFIG_INTEGERS = 64 selects: macros_and_parameters.h:217) and
   `#define float double` (CONFIG_BFLOAT_8: macros_and_parameters.h:257) in force.
   Under those macros every `int` below would become a 64-bit integer and every
   `float` a double, so the caller's view of the structs, the return values and the
   weight arrays would no longer be the library's.  Both macros are suspended for
   the length of this header and restored at its end; the declarations always mean
   the C types written here.  ppm_b200_abi_check lets a caller confirm at start-up
   that its compiled view of the structs matches the library's. */
#pragma push_macro("int")
#pragma push_macro("float")
#undef int
#undef float

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PPM_B200_VERSION 100

/* return codes */
#define PPM_B200_OK 0
#define PPM_B200_ERR_UNSUPPORTED (-1)  /* configuration this library does not cover: caller keeps the Fortran path */
#define PPM_B200_ERR_INVALID (-2)      /* bad arguments (NULL field, ghost zones != 3, ...) */
#define PPM_B200_ERR_CUDA (-3)         /* a CUDA runtime call failed */
#define PPM_B200_ERR_NEGATIVE (-4)     /* a state the reference aborts on (flux_twoshock.F:440-443, flux_hll.F:336-383, euler.F:203-215) */
#define PPM_B200_ERR_NONFINITE (-5)    /* non-finite output detected */
#define PPM_B200_ERR_TOO_LARGE (-6)    /* size beyond a fixed limit of the entry point */
#define PPM_B200_ERR_TIMEOUT (-7)      /* a bounded device wait on an asynchronous copy gave up: outputs invalid */

/* memory kinds of the field pointers */
#define PPM_B200_MEM_HOST 0   /* fields in host memory: copied in and out inside the call (like cuPPMSetBaryon/GetBaryon) */
#define PPM_B200_MEM_DEVICE 1 /* fields already resident in device memory */

/* MAX_COLOR (fortran.def:2): the most colour fields a sweep advects */
#define PPM_B200_MAX_COLOURS 45

/* Riemann solver / reconstruction enums, values as in Enzo's typedefs.h */
#define PPM_B200_RIEMANN_TWOSHOCK 5   /* twoshock + flux_twoshock (the PPM default) */
#define PPM_B200_RIEMANN_HLL 1        /* flux_hll.F */
#define PPM_B200_RIEMANN_HLLC 4       /* flux_hllc.F */
#define PPM_B200_RECONSTRUCTION_PPM 1

/* Hydro globals consumed by the sweeps (global_data.h, defaults in
   SetDefaultGlobalValues.C).  POD, filled by the caller from the same globals
   the Fortran path reads. */
typedef struct ppm_b200_params {
  double gamma;             /* Gamma */
  double dt;                /* dtFixed of the grid */
  double eta1, eta2;        /* DualEnergyFormalismEta1 / Eta2 */
  double small_rho;         /* SmallRho (density floor of euler.F:141-144) */
  double tiny_number;       /* tiny_number = MinimumPressure of the sweeps */
  double min_support;       /* MinimumSupportEnergyCoefficient (ComputePressure) */
  int dual_energy;          /* DualEnergyFormalism */
  int gravity;              /* GravityOn (AccelerationField used) */
  int pressure_free;        /* PressureFree: 0 or 1 (inteuler.F:199, :556-561, twoshock.F:124-130) */
  int riemann_solver;       /* RiemannSolver: PPM_B200_RIEMANN_TWOSHOCK, _HLL or _HLLC
                               (learned_guess applies to the two-shock solver only) */
  int riemann_fallback;     /* RiemannSolverFallback */
  int reconstruction;       /* ReconstructionMethod: PPM_B200_RECONSTRUCTION_PPM */
  int steepening;           /* PPMSteepeningParameter: 0 or 1 (density steepening, inteuler.F:166-193) */
  int flattening;           /* PPMFlatteningParameter: 0, 1, 2 or 3 (calcdiss.F eq. A1-A2 / A4-A6 / A7-A10) */
  int diffusion;            /* PPMDiffusionParameter: must be 0 */
  int conservative_rec;     /* ConservativeReconstruction: must be 0 */
  int positive_rec;         /* PositiveReconstruction: must be 0 */
  int eos_type;             /* EOSType: 0, or 3 (isothermal, hydro_rk/EOS.h): p = rho cs^2 and the
                               total energy reset where the pressure is computed (the solve's
                               start and end, Grid_SolvePPM_DE.C:60, :155-157) */
  int number_of_colours;    /* NumberOfColours: 0 .. PPM_B200_MAX_COLOURS advected colour fields
                               (Grid_SolveHydroEquations.C:90-285); their fields are
                               ppm_b200_grid.colours[] */
  int learned_guess;        /* start twoshock's Newton iteration from the learned p* guess
                               (weights from ppm_b200_set_guess): 0 off; 1 the net evaluated
                               inside the Riemann kernel (mma.sync); 2 a guess pass on the
                               tcgen05 tensor cores before the Riemann kernel */
  const double *dt_device;  /* optional: device pointer holding dtFixed (overrides dt) */
  const int *colour_species; /* optional HOST array of number_of_colours flags for
                               ppm_b200_correct_fluxes[_sublings]: nonzero for a colour
                               that keeps its fraction of the corrected density there
                               (FluxCorrection = 1: fields ElectronDensity .. ExtraType1
                               and the SN Ia / II metal densities,
                               Grid_CorrectForRefinedFluxes.C:397-421, :849-866); other
                               colours are left alone.  NULL: none */
  double eos_sound_speed;   /* EOSSoundSpeed (EOSType 3) */
  int reserved[2];
} ppm_b200_params;

/* One grid.  Field pointers are host or device memory as the call says.
   velocity[d] may be NULL for d >= rank; gas_energy may be NULL unless
   dual_energy; acceleration[] is read only when gravity. */
typedef struct ppm_b200_grid {
  int rank;                 /* GridRank */
  int dims[3];              /* GridDimension (ghosts included) */
  int start[3];             /* GridStartIndex (0-based) */
  int end[3];               /* GridEndIndex (0-based, inclusive) */
  double *density;          /* BaryonField[DensNum] */
  double *total_energy;     /* BaryonField[TENum] */
  double *velocity[3];      /* BaryonField[Vel1Num..Vel3Num] */
  double *gas_energy;       /* BaryonField[GENum] */
  const double *acceleration[3]; /* AccelerationField[dim] */
  const double *cell_width[3];   /* CellWidthTemp[dim]: HOST arrays of dims[dim] values */
  double *const *colours;        /* HOST array of params->number_of_colours field pointers,
                                    BaryonField[colnum[n]] in colnum[] order; the fields
                                    are updated in place (NULL when there are none) */
} ppm_b200_grid;

/* struct fluxes (Fluxes.h:29-37) restricted to the six hydro slots.
   Slot order: density, total energy, velocity1, velocity2, velocity3, gas
   energy.  Arrays are HOST memory, allocated and zeroed by the caller
   (Grid_SolveHydroEquations.C:320-369); NULL slots are skipped. */
typedef struct ppm_b200_fluxes {
  long long left_start[3][3], left_end[3][3];
  long long right_start[3][3], right_end[3][3];
  double *left[6][3];
  double *right[6][3];
  /* colours: HOST arrays of number_of_colours * 3 pointers, entry n*3 + dim =
     LeftFluxes/RightFluxes[colnum[n]][dim] (NULL arrays or entries are skipped).  Like
     the reference these hold colf / dx: dt * ub * colour, divided by the cell width
     (Grid_xEulerSweep.C:361-371 after euler.F:173-176). */
  double *const *colour_left;
  double *const *colour_right;
} ppm_b200_fluxes;

typedef struct ppm_b200_stats {
  long long interfaces;     /* Riemann problems solved */
  long long newton_iters;   /* Newton updates performed */
  long long newton_hist[8]; /* interfaces by Newton updates taken (1..7) */
  long long fallbacks;      /* cells recomputed with the HLL fallback */
  long long fatal_cells;    /* cells in a state the reference aborts on */
  long long guess_rejected; /* learned guesses that did not converge (plain guess reused) */
  long long warp_newton_iters; /* sum over the Riemann kernel's warps of the most Newton
                               updates any of its lanes took: what the divergent loop costs */
  long long warps;          /* Riemann warps with at least one interface */
} ppm_b200_stats;

typedef struct ppm_b200_context ppm_b200_context;

/* Context: one per MPI rank / device (InitGPU selects rank % ngpu,
   CUDAUtil.cu:19-31).  Owns the stream, persistent device scratch (grown on
   demand, never reallocated per call) and device-side status counters.
   stream may be NULL (the context creates its own non-blocking stream). */
int ppm_b200_create(int device, void *cuda_stream, ppm_b200_context **ctx);
int ppm_b200_destroy(ppm_b200_context *ctx);

/* grid::SolvePPM_DE (Grid_SolvePPM_DE.C:36-164) for EOSType 0: pressure once,
   then the x/y/z sweeps in the order rotated by cycle_number % rank, each over
   every pencil including transverse ghost pencils, with subgrid flux capture.
   memory = PPM_B200_MEM_HOST: synchronous, like the Fortran path.
   memory = PPM_B200_MEM_DEVICE: asynchronous on the context stream when
   nsub == 0 and stats == NULL; call ppm_b200_synchronize for the status. */
int ppm_b200_solve_ppm_de(ppm_b200_context *ctx, const ppm_b200_params *params,
                          int cycle_number, ppm_b200_grid *grid, int memory, int nsub,
                          ppm_b200_fluxes *subgrid_fluxes, const long long grid_global_start[3],
                          ppm_b200_stats *stats);

/* One direction: the `for k ... xEulerSweep(k)` loop (Grid_SolvePPM_DE.C:89-97)
   or its y (:108-116) / z (:127-136) sibling, with a caller-supplied pressure
   field (same memory kind as the fields). */
int ppm_b200_euler_sweep(ppm_b200_context *ctx, int dim, const ppm_b200_params *params,
                         ppm_b200_grid *grid, const double *pressure, int memory, int nsub,
                         ppm_b200_fluxes *subgrid_fluxes, const long long grid_global_start[3],
                         ppm_b200_stats *stats);

/* grid::ComputePressure at time == Time (Grid_ComputePressure.C:96-164). */
int ppm_b200_compute_pressure(ppm_b200_context *ctx, const ppm_b200_params *params,
                              ppm_b200_grid *grid, double *pressure, int memory);

/* Courant time step of grid::ComputeTimeStep for PPM (Grid_ComputeTimeStep.C
   :146-209 with calc_dt.F ihydro = 0): pressure on the fly, min over active
   cells of aye / sum_d (c_s + |v_d - vgrid_d|)/dx_d, times courant.
   Writes the result to *dt_device (device pointer, may be NULL) without a host
   sync, and to *dt_host (may be NULL; synchronises). */
int ppm_b200_compute_timestep(ppm_b200_context *ctx, const ppm_b200_params *params,
                              ppm_b200_grid *grid, int memory, double courant, double aye,
                              const double vgrid[3], double *dt_device, double *dt_host);

/* Ghost-zone fill of one grid on device memory (periodic = 0 / outflow = 1 /
   2 = leave alone, for faces a halo exchange fills, per dimension); the
   external-boundary part of SetBoundaryConditions for a single grid
   (ExternalBoundary_SetExternalBoundaryIO.C:201-209, :378-386). */
int ppm_b200_set_boundary(ppm_b200_context *ctx, ppm_b200_grid *grid, int dual_energy,
                          int number_of_colours, const int bc_type[3]);

/* The time step of the next cycle, folded into every later solve on this context:
   the last sweep's update kernel evaluates calc_dt (ihydro = 0, calc_dt.F:136-153 with
   the pressure of grid::ComputePressure, Grid_ComputePressure.C:96-164) on each active
   cell as soon as its final state is known, and the solve writes courant * min dt1 over
   its grid(s) to *dt_device (device memory) -- the value ppm_b200_compute_timestep (or
   _level) would return after the solve, without its pass over the fields.
   dt_device = NULL turns it off.  aye and vgrid as in ppm_b200_compute_timestep. */
int ppm_b200_set_cfl(ppm_b200_context *ctx, double *dt_device, double courant, double aye,
                     const double vgrid[3]);

/* --- AMR level entry points: every grid of a level in one batch (DEVICE memory) ---
   The reference advances a level one grid at a time: the grid loop of
   EvolveLevel.C:569-585 calls grid::SolveHydroEquations -> SolvePPM_DE per grid,
   and SetLevelTimeStep.C:66 takes the min of grid::ComputeTimeStep over the grids.
   These run each stage of that loop as ONE kernel launch over all grids (largest
   first); results are bit-identical to calling the single-grid entry points on
   each grid in turn.  All grids share rank and physics parameters. */

/* SolvePPM_DE of every grid of a level (no subgrid flux capture).  Asynchronous
   unless stats != NULL.  With graphs enabled (ppm_b200_set_graphs) and
   params->dt_device set, the level's launches are captured once into a CUDA graph
   per sweep rotation and replayed while the grid list and parameters stay the
   same. */
int ppm_b200_solve_level(ppm_b200_context *ctx, const ppm_b200_params *params,
                         int cycle_number, ppm_b200_grid *grids, int ngrids,
                         ppm_b200_stats *stats);

/* enable != 0: replay level solves from CUDA graphs (see ppm_b200_solve_level). */
int ppm_b200_set_graphs(ppm_b200_context *ctx, int enable);

/* Which kernels run a directional sweep of the plain path (two-shock solver with the
   acoustic start, no colours, no flattening or steepening; other paths always split).
   PPM_B200_SWEEP_SPLIT: two marching reconstruction kernels write the interface states
   of every face, a face-parallel Riemann kernel reads them and writes the fluxes.
   PPM_B200_SWEEP_FUSED: one kernel reconstructs and solves every face (a warp per
   pencil segment of 31 faces, neighbours by warp shuffles), so the interface states never
   reach device memory.  Both give the same bits; the update and fallback kernels are
   shared.  No reference counterpart (the reference runs one slice at a time,
   Grid_xEulerSweep.C:196-305). */
#define PPM_B200_SWEEP_SPLIT 0
#define PPM_B200_SWEEP_FUSED 1
int ppm_b200_set_sweep_mode(ppm_b200_context *ctx, int mode);

/* How ppm_b200_solve_level schedules a level (no reference counterpart: the reference
   runs its grid loop, EvolveLevel.C:569-585, one grid at a time).
   schedule: PPM_B200_LEVEL_BATCHED -- every grid in one launch per kernel stage;
             PPM_B200_LEVEL_CLASSES -- one such batch per size class, one after another,
             each with its class's Riemann settings;
             PPM_B200_LEVEL_PER_GRID -- one launch per kernel stage per grid, largest
             first: the reference's loop, kept for comparison (graph-replayable).
   Size classes by active cells: class 0 below class_cells[0], class 1 below
   class_cells[1], class 2 the rest.  The two-shock Riemann stage (plain start, no
   colours) of a batch runs riemann_threads faces per block (64, 128 or 256) and, with
   persistent != 0, as a persistent launch of the resident blocks that walks the batch's
   block list; index 3 is the setting of the BATCHED schedule, 0-2 those of the classes.
   max_scratch_bytes > 0 bounds the level's device scratch (ring sets, pressure and face
   planes): grids are then solved in waves that each fit it (a single grid larger than
   the bound still runs, alone).  Results are bit-identical whatever the schedule. */
#define PPM_B200_LEVEL_BATCHED 0
#define PPM_B200_LEVEL_CLASSES 1
#define PPM_B200_LEVEL_PER_GRID 2
typedef struct ppm_b200_level_config {
  int schedule;
  int riemann_threads[4];
  int persistent[4];
  long long class_cells[2];
  long long max_scratch_bytes;
} ppm_b200_level_config;
int ppm_b200_set_level_config(ppm_b200_context *ctx, const ppm_b200_level_config *cfg);
int ppm_b200_get_level_config(ppm_b200_context *ctx, ppm_b200_level_config *cfg);

/* The per-size-class autotuner (no reference counterpart).  Times, on copies of the
   grids' fields made in the context (DEVICE memory; the grids themselves are not
   changed), one solve of every size class for each Riemann setting -- candidate
   k = 2 * t + persistent with t = 0, 1, 2 for 64, 128, 256 faces per block -- then the
   whole level as one batch for each candidate and as one batch per class with each
   class's best, and keeps the fastest schedule as the context's level configuration
   (max_scratch_bytes is kept).  Synchronises; about 40 level solves. */
typedef struct ppm_b200_level_tuning {
  int class_grids[3];          /* grids per size class */
  long long class_active[3];   /* active cells per size class */
  double class_ms[3][6];       /* ms of one solve of the class, per candidate (0: no grids) */
  double batched_ms[6];        /* ms of one solve of the whole level as one batch */
  double classes_ms;           /* ms with one batch per class, each with its best candidate */
  ppm_b200_level_config chosen;
} ppm_b200_level_tuning;
int ppm_b200_autotune_level(ppm_b200_context *ctx, const ppm_b200_params *params,
                            int cycle_number, ppm_b200_grid *grids, int ngrids,
                            ppm_b200_level_tuning *report);

/* min over the grids of the hydro Courant time step (SetLevelTimeStep.C:66 over
   grid::ComputeTimeStep), one reduction for the whole level. */
int ppm_b200_compute_timestep_level(ppm_b200_context *ctx, const ppm_b200_params *params,
                                    ppm_b200_grid *grids, int ngrids, double courant,
                                    double aye, const double vgrid[3], double *dt_device,
                                    double *dt_host);

/* ppm_b200_set_boundary on every grid of a list, one launch. */
int ppm_b200_set_boundary_level(ppm_b200_context *ctx, ppm_b200_grid *grids, int ngrids,
                                int dual_energy, int number_of_colours, const int bc_type[3]);

/* grid::CopyZonesFromGrid (Grid_CopyZonesFromGrid.C:37-300, without the shearing box)
   over a level, the sibling and periodic part of SetBoundaryConditions
   (SetBoundaryConditions.C:113-201): every grid receives, into its whole region (ghost
   zones included), the zones of every grid's active region that overlap it -- its
   siblings', and the periodic images of all grids (itself included) shifted by
   domain[d] along the axes with periodic[d] != 0.  Zones outside the domain on
   non-periodic axes and zones covered only by the parent grid are left as they are
   (ppm_b200_set_boundary_level fills the former).  left[3*k + d]: the index, at this
   level's resolution, of grid k's first zone (ghosts included) along axis d; the grids
   share their rank.  Active regions of a level are disjoint, so every zone receives at
   most one copy; all copies run as one launch on device fields. */
int ppm_b200_copy_zones_level(ppm_b200_context *ctx, ppm_b200_grid *grids, int ngrids,
                              const long long *left, const long long domain[3],
                              const int periodic[3], int dual_energy, int number_of_colours);

/* grid::CorrectForRefinedFluxes (Grid_CorrectForRefinedFluxes.C:38-760) for the proper
   subgrids of one grid: Cartesian coordinates, the six hydro fields (no species or
   colours), RadiativeCooling == 0 and CorrectParentBoundaryFlux off (the defaults).  The
   zones just outside each subgrid face get the difference of the coarse (initial, as
   captured by the solve) and refined fluxes, in conserved form, with the reference's
   undo when density or an energy would become non-positive -- which also resets those
   refined fluxes to the initial ones, as the reference does -- and the dual-energy
   consistency of the corrected zones.  initial[n] / refined[n]: the n-th subgrid's flux
   structures (host arrays, the same index boxes); grid_global_start: the global index of
   the grid's first zone (ghosts included).  memory: where the grid's fields live. */
/* Test hook for the bounded device waits (not for production use): with extra_bytes > 0
   (a multiple of 16, at most 4096) every TMA chunk of the x sweep's update kernel
   expects that many bytes more than its copies deliver, so its barrier never completes;
   each wait gives up after about a second, the kernel drains its copies and returns,
   and the call reports PPM_B200_ERR_TIMEOUT with the context still usable.  0 restores
   normal operation.  Nothing faults or hangs. */
int ppm_b200_debug_tma_stall(ppm_b200_context *ctx, int extra_bytes);

int ppm_b200_correct_fluxes(ppm_b200_context *ctx, const ppm_b200_params *params,
                            ppm_b200_grid *grid, int memory, int nsub,
                            const ppm_b200_fluxes *initial, ppm_b200_fluxes *refined,
                            const long long grid_global_start[3]);

/* The SUBling calls of grid::CorrectForRefinedFluxes (SUBlingGrid == TRUE,
   UpdateFromFinerGrids.C:176-206, Grid_CorrectForRefinedFluxes.C:147-305, :455-656), in
   order, for the nsib sibling subgrids of a grid: refined[n] holds sibling subgrid n's
   refined boundary fluxes projected to this level (GetProjectedBoundaryFluxes), own
   this grid's own boundary fluxes (SubgridFluxesEstimate[grid][NumberOfSubgrids - 1]).
   The grid's edge layer that touches a sibling's projected face is corrected by the
   difference; a periodic level boundary wraps.  level_dims: the level's extent in zones
   (nint((DomainRightEdge - DomainLeftEdge)/CellWidth)) per axis; periodic: periodic
   faces per axis.  The refined index boxes are read only; refined flux values are
   updated where a correction is undone.  Cartesian, hydro fields, as
   ppm_b200_correct_fluxes. */
int ppm_b200_correct_fluxes_sublings(ppm_b200_context *ctx, const ppm_b200_params *params,
                                     ppm_b200_grid *grid, int memory, int nsib,
                                     const ppm_b200_fluxes *own, ppm_b200_fluxes *refined,
                                     const long long grid_global_start[3],
                                     const long long level_dims[3], const int periodic[3]);

/* Waits for all work queued on the context and returns the first error code
   recorded by device work since the last call; accumulates device counters
   into *stats (may be NULL). */
int ppm_b200_synchronize(ppm_b200_context *ctx, ppm_b200_stats *stats);

/* Device memory the context holds (scratch, staging of host-memory calls, descriptor
   images), in bytes (no reference counterpart). */
int ppm_b200_device_bytes(ppm_b200_context *ctx, long long *bytes);

/* Number of kernels this library has launched on the context since creation. */
long long ppm_b200_launch_count(ppm_b200_context *ctx);

/* Kernel timing with CUDA events recorded on the context stream around every sweep
   launch (the per-direction timers of the reference's EnzoTiming sections,
   Grid_SolveHydroEquations.C:68 / :632, at kernel granularity).  enable = 0 stops.
   ppm_b200_profile_read synchronises, returns the summed sweep-kernel time in ms
   and the number of timed sweep launches since the last read, and resets them. */
int ppm_b200_profile(ppm_b200_context *ctx, int enable);
int ppm_b200_profile_read(ppm_b200_context *ctx, double *sweep_ms, long long *sweep_launches);
/* Per-kernel split of the last ppm_b200_profile_read: summed ms of the five kernels of
   a sweep (reconstruct d/p/u, reconstruct v/w/ge, Riemann, update, HLL fallback pass). */
int ppm_b200_profile_stages(ppm_b200_context *ctx, double stage_ms[5]);

/* grid::ComovingExpansionTerms for PPM (Grid_ComovingExpansionTerms.C:36-99 with
   expand_terms.F, ENERGY_METHOD3 / VELOCITY_METHOD3), called after the hydro step of
   a grid when ComovingCoordinates (EvolveLevel.C:753-754): the pressure at
   0.5*(time + old_time), interpolated between `old` (the fields at OldTime,
   OldBaryonField) and the current fields, or at `time` when old is NULL; then the
   expansion terms of the gas energy, total energy and velocities in every cell.
   coefficient = dtFixed * (da/dt) / a at the mid time (CosmologyComputeExpansionFactor,
   the caller's).  Same memory kind for grid and old. */
int ppm_b200_expansion_terms(ppm_b200_context *ctx, const ppm_b200_params *params,
                             ppm_b200_grid *grid, const ppm_b200_grid *old, double time,
                             double old_time, double coefficient, int memory);
/* The same for every grid of a level (DEVICE memory; olds may be NULL). */
int ppm_b200_expansion_terms_level(ppm_b200_context *ctx, const ppm_b200_params *params,
                                   ppm_b200_grid *grids, const ppm_b200_grid *olds,
                                   int ngrids, double time, double old_time,
                                   double coefficient);

/* --- learned starting pressure of twoshock's Newton iteration (twoshock.F:156-170) ---
   A 6 -> 64 -> 64 -> 1 MLP predicts ln(p* / p_acoustic) from the two interface states;
   with params->learned_guess = 1 the Riemann kernel evaluates it with warp-level MMAs,
   with 2 a separate pass evaluates it with tcgen05.mma (accumulators in tensor memory)
   into the face's flux-plane slot (BF16 operands, FP32 accumulation either way); the
   Riemann kernel starts Newton from that pressure, iterates to the
   reference tolerance, and re-solves from the acoustic start (the plain solver) any
   face that does not converge (counted in stats->guess_rejected).  The fields then
   agree with the plain solver to round-off, not bit for bit.
   Weights: 4673 floats, W1[6][64] b1[64] W2[64][64] b2[64] w3[64] b3 (row = input).
   All pointers below are DEVICE memory unless stated; calls queue on the context
   stream and return without waiting, except where noted. */

/* Host weights for the learned start (NULL: forget them).  Synchronises. */
int ppm_b200_set_guess(ppm_b200_context *ctx, const float *weights_host);

/* Log about one in `stride` Riemann problems of later plain solves on this context:
   8 doubles per record (dl dr pl pr ul ur p* iterations, the count negative when
   Newton did not converge), at most `capacity` records.  NULL / 0 stops logging. */
int ppm_b200_riemann_log(ppm_b200_context *ctx, double *records, long long capacity,
                         int stride);
/* Records written so far (synchronises). */
int ppm_b200_riemann_log_count(ppm_b200_context *ctx, long long *count);

/* Training samples from log records: 8 floats each (the 6 inputs, the target
   ln(p* / p_acoustic), 1 if usable else 0 -- unconverged or non-finite). */
int ppm_b200_guess_features(ppm_b200_context *ctx, const double *records, long long n,
                            double gamma, double pmin, float *samples);

/* Forward + backward over samples[index[0..n-1]] (index may be NULL: the first n):
   adds d(loss)/d(weights) to grad (4673 floats, zero it first) and the summed squared
   error to *loss (one double), loss = mean squared error of the n samples. */
int ppm_b200_guess_grad(ppm_b200_context *ctx, const float *weights, const float *samples,
                        const long long *index, long long n, float *grad, double *loss);

/* One Adam step (step counts from 1) on the FP32 master weights; zeroes grad. */
int ppm_b200_guess_adam(ppm_b200_context *ctx, float *weights, float *grad, float *m,
                        float *v, int step, float lr, float beta1, float beta2, float eps);

/* The net on given inputs (6 floats each), with the weights of ppm_b200_set_guess, on
   the tcgen05 tensor cores (the kernel of learned_guess = 2): y[i] = the net's output
   (the predicted ln(p* / p_acoustic) / |x|^2).  Queues and returns.  Waits on the MMAs
   are bounded: a CTA whose MMA does not complete within about a second stops, leaves its
   remaining outputs unwritten and counts a timeout, which the context's next status
   read (ppm_b200_synchronize, a synchronous solve) reports as PPM_B200_ERR_TIMEOUT. */
int ppm_b200_guess_eval(ppm_b200_context *ctx, const float *features, long long n, float *y);

/* One directional sweep that allocates nothing (no counterpart in the reference).
   For callers that cannot call cudaMalloc when they advance a grid -- code running
   under a memory arena that owns all device memory, or inside a callback where an
   allocation could synchronise or deadlock.  `in` and `out` are caller-owned DEVICE
   arrays (cell widths stay host arrays), `pressure` a device array; no output may
   overlap an input or the pressure (an in-place call returns PPM_B200_ERR_INVALID).
   The sweep's scratch comes from a fixed array compiled into the library.
   Limit: 19 * 8 * (active cells along dim + 1) * pencils bytes <= 48 MiB (grids up
   to 64^3 active cells) and pencils of at most 1031 cells; larger sizes return
   PPM_B200_ERR_TOO_LARGE.  The first call in a CUDA context (the device current)
   looks up the array's address and keeps it for that context.  The call copies from
   host memory and waits for its stream, so it must never run while cuda_stream is
   being captured into a graph: it then returns PPM_B200_ERR_INVALID without touching
   the stream.  The array is shared by all calls on a device: calls that overlap on the
   GPU race.  Synchronous on cuda_stream (NULL = default stream); no subgrid flux
   capture. */
int ppm_b200_euler_sweep_static(int dim, const ppm_b200_params *params,
                                const ppm_b200_grid *in, const double *pressure,
                                ppm_b200_grid *out, void *cuda_stream, ppm_b200_stats *stats);

const char *ppm_b200_error_string(int code);
int ppm_b200_version(void);

/* --- ABI self-check (no counterpart in the reference) ---
   PPM_B200_ABI_LAYOUT(X) lists the sizes and member offsets of the structs above as
   the including translation unit sees them.  A caller builds the list once,
     static const long long layout[] = { PPM_B200_ABI_LAYOUT(PPM_B200_ABI_ITEM) };
     if (ppm_b200_abi_check(layout, (int)(sizeof layout / sizeof layout[0])) != 0) ...
   and the library compares it with its own: PPM_B200_OK when they agree,
   PPM_B200_ERR_INVALID otherwise (different build flags, packing or a stale header). */
#define PPM_B200_ABI_ITEM(e) (long long)(e),
#define PPM_B200_ABI_LAYOUT(X)                                                        \
  X(sizeof(ppm_b200_params)) X(offsetof(ppm_b200_params, min_support))              \
  X(offsetof(ppm_b200_params, dual_energy)) X(offsetof(ppm_b200_params, learned_guess)) \
  X(offsetof(ppm_b200_params, dt_device)) X(offsetof(ppm_b200_params, colour_species)) \
  X(offsetof(ppm_b200_params, eos_sound_speed)) X(offsetof(ppm_b200_params, reserved)) \
  X(sizeof(ppm_b200_grid)) X(offsetof(ppm_b200_grid, dims))                          \
  X(offsetof(ppm_b200_grid, end)) X(offsetof(ppm_b200_grid, density))                \
  X(offsetof(ppm_b200_grid, velocity)) X(offsetof(ppm_b200_grid, acceleration))      \
  X(offsetof(ppm_b200_grid, cell_width)) X(offsetof(ppm_b200_grid, colours))         \
  X(sizeof(ppm_b200_fluxes)) X(offsetof(ppm_b200_fluxes, right_end))                 \
  X(offsetof(ppm_b200_fluxes, left)) X(offsetof(ppm_b200_fluxes, right))             \
  X(offsetof(ppm_b200_fluxes, colour_left)) X(offsetof(ppm_b200_fluxes, colour_right)) \
  X(sizeof(ppm_b200_stats)) X(offsetof(ppm_b200_stats, newton_hist))                 \
  X(offsetof(ppm_b200_stats, guess_rejected)) X(offsetof(ppm_b200_stats, warps))             \
  X(sizeof(ppm_b200_level_config)) X(offsetof(ppm_b200_level_config, max_scratch_bytes))     \
  X(sizeof(ppm_b200_level_tuning)) X(offsetof(ppm_b200_level_tuning, chosen))
int ppm_b200_abi_check(const long long *layout, int n);

#ifdef __cplusplus
}
#endif

#pragma pop_macro("float")
#pragma pop_macro("int")
#endif /* PPM_B200_H */
