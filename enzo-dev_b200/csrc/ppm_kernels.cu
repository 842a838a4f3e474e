// ppm_kernels.cu -- the grid-wide kernels around the sweeps (sm_100a):
//
//   pressure_kernel           grid::ComputePressure (time == Time)
//   timestep_kernel           calc_dt (ihydro = 0) min-reduction + Courant factor
//   boundary_kernel           outflow / periodic ghost-zone fill
// Each covers a whole batch of grids (one grid, or an AMR level) in one launch.
//
// The directional sweeps themselves are in ppm_split.cu.
#include <cuda_runtime.h>

#include "ppm_device.cuh"
#include "ppm_sweep.cuh"

namespace ppm {

// ------------------------------------------------------------------ batched grid records
// One record per grid of a batch (a single grid, or every grid of an AMR level).
// Blocks of 256 threads are assigned to grids through prefix tables, so one launch
// covers the whole batch; batch_locate (ppm_sweep.cuh) maps a block to its grid.
struct ElemGrid {
  const double* d;
  const double* te;
  const double* v[3];   // null for v[d] with d >= rank
  const double* ge;     // non-null selects the dual-energy pressure
  double* p;            // pressure output (pressure kernel)
  double* f[6];         // fields filled by the ghost-zone kernel (null entries skipped)
  const double* cw[3];  // device cell widths (time-step kernel)
  const double* old[6]; // fields at OldTime: d, te, v1, v2, v3, ge (expansion kernel)
  int rank;
  int dims[3], start[3], end[3];
  int bc[3];            // 0 periodic, 1 outflow, 2 left alone
  int64_t size;         // cells incl. ghosts
  int64_t active;       // active cells
};

struct ElemBatch {
  const ElemGrid* grids;
  int ngrids;
  const int64_t* size_prefix;    // ceil(size / 256) blocks per grid
  const int64_t* active_prefix;  // ceil(active / 256) blocks per grid
  const int64_t* row_prefix;     // ceil(rows / 32) blocks per grid (ghost fill: 8 warps x 4 rows)
  double gamma, tiny_number, min_support;
  double aye, vg[3];
  unsigned long long* min_bits;  // running minimum of dt1 (positive doubles order as integers)
  // expansion kernel: dt * adot / a, and the pressure's interpolation weights
  double expansion, coef_new, coef_old;
  int interpolate;
  int presfree;                  // PressureFree: calc_dt's sound speed tiny (calc_dt.F:78-137)
  // EOSType 3 (isothermal, EOS.h): p = rho cs^2 and the total energy reset to
  // p/((gamma-1) rho) + v^2/2 wherever the pressure is computed (Grid_ComputePressure.C:112-124)
  int eos_type;
  double eos_cs;
};

// grid::ComputePressure at time == Time (Grid_ComputePressure.C:96-164)
__device__ __forceinline__ double cell_pressure(const ElemGrid& G, int64_t i, double gamma,
                                                double tiny_number, double min_support) {
  const double gm1 = gamma - 1.0;
  const double density = __ldg(G.d + i);
  double gas_energy;
  if (G.ge) {
    gas_energy = __ldg(G.ge + i);
  } else {
    const double velocity1 = __ldg(G.v[0] + i);
    const double velocity2 = G.v[1] ? __ldg(G.v[1] + i) : 0.0;
    const double velocity3 = G.v[2] ? __ldg(G.v[2] + i) : 0.0;
    gas_energy = __ldg(G.te + i) -
                 0.5 * (velocity1 * velocity1 + velocity2 * velocity2 + velocity3 * velocity3);
  }
  double p = gm1 * density * gas_energy;
  if (p < tiny_number) p = tiny_number;
  const double min_pressure = min_support * gm1 * density * density;
  if (p < min_pressure) p = min_pressure;
  return p;
}

// EOSType 3: the pressure of cell i, and (RESET) its total energy reset (G.f[1] is the
// field).  The time step does not reset: after a solve the energies are already
// consistent, and the reset is idempotent.
template <bool RESET>
__device__ __forceinline__ double eos_pressure(const ElemGrid& G, int64_t i, const ElemBatch& B) {
  const double density = G.d[i];
  const double velocity1 = G.v[0][i];
  const double velocity2 = G.v[1] ? G.v[1][i] : 0.0;
  const double velocity3 = G.v[2] ? G.v[2][i] : 0.0;
  const double cs = B.eos_cs;
  const double p = density * cs * cs;
  const double e = p / ((B.gamma - 1.0) * density);
  if (RESET)
    G.f[1][i] = e + 0.5 * (velocity1 * velocity1 + velocity2 * velocity2 + velocity3 * velocity3);
  return p;
}

__global__ void __launch_bounds__(256) pressure_kernel(const __grid_constant__ ElemBatch B) {
  int64_t lb;
  const ElemGrid& G = B.grids[batch_locate(B.size_prefix, B.ngrids, blockIdx.x, lb)];
  const int64_t i = lb * 256 + threadIdx.x;
  if (i < G.size)
    G.p[i] = B.eos_type == 3 ? eos_pressure<true>(G, i, B)
                             : cell_pressure(G, i, B.gamma, B.tiny_number, B.min_support);
}

// calc_dt (ihydro = 0) over the active cells of every grid; min over the batch
__global__ void __launch_bounds__(256) timestep_kernel(const __grid_constant__ ElemBatch B) {
  int64_t lb;
  const ElemGrid& G = B.grids[batch_locate(B.active_prefix, B.ngrids, blockIdx.x, lb)];
  const int64_t c = lb * 256 + threadIdx.x;
  double best = 1.0e20;  // calc_dt.F:71 (huge)
  if (c < G.active) {
    const int nx = G.end[0] - G.start[0] + 1;
    const int ny = G.rank > 1 ? G.end[1] - G.start[1] + 1 : 1;
    const int i = G.start[0] + (int)(c % nx);
    const int j = (G.rank > 1 ? G.start[1] : 0) + (int)((c / nx) % ny);
    const int k = (G.rank > 2 ? G.start[2] : 0) + (int)(c / ((int64_t)nx * ny));
    const int64_t g = ((int64_t)k * G.dims[1] + j) * G.dims[0] + i;
    const double density = __ldg(G.d + g);
    const double u = __ldg(G.v[0] + g);
    const double v = G.v[1] ? __ldg(G.v[1] + g) : 0.0;
    const double w = G.v[2] ? __ldg(G.v[2] + g) : 0.0;
    const double p = B.eos_type == 3 ? eos_pressure<false>(G, g, B)
                                     : cell_pressure(G, g, B.gamma, B.tiny_number, B.min_support);
    // calc_dt.F:136-153
    const double cs = B.presfree ? kTiny : dmax(sqrt(B.gamma * p / density), kTiny);
    double dt1;
    if (G.rank == 1) {
      dt1 = G.cw[0][i] * B.aye / (cs + fabs(u - B.vg[0]));
    } else if (G.rank == 2) {
      dt1 = B.aye / ((cs + fabs(u - B.vg[0])) / G.cw[0][i] + (cs + fabs(v - B.vg[1])) / G.cw[1][j]);
    } else {
      dt1 = B.aye / ((cs + fabs(u - B.vg[0])) / G.cw[0][i] + (cs + fabs(v - B.vg[1])) / G.cw[1][j] +
                     (cs + fabs(w - B.vg[2])) / G.cw[2][k]);
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
    if (lane == 0) atomicMin(B.min_bits, (unsigned long long)__double_as_longlong(best));
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
__device__ __forceinline__ int bc_map(int i, int s, int e, int bc) {
  if (i >= s && i <= e) return i;
  if (bc == 2) return i;  // left alone: filled by a halo exchange
  if (bc == 0) {
    const int nn = e - s + 1;
    int r = (i - s) % nn;
    if (r < 0) r += nn;
    return s + r;
  }
  return i < s ? s : e;
}

// f: the grid's field pointers held in registers (a store through one of them could
// otherwise alias the record in global memory and force the pointers to be reloaded)
__device__ __forceinline__ void copy_cell(double* const (&f)[6], int64_t dst, int64_t src) {
#pragma unroll
  for (int n = 0; n < 6; ++n)
    if (f[n]) f[n][dst] = f[n][src];
}

// One warp per row (j, k) of the padded grid: every ghost cell copies the cell it maps
// to.  A row whose (j, k) maps to itself holds ghosts only at its x ends; any other row
// is copied whole from its source row, with consecutive lanes on consecutive cells.
// Sources are cells that map to themselves in all three dimensions (active cells, or
// ghosts of a face left to a halo exchange), which this kernel never writes, so the
// in-place fill has no read-after-write hazard.  A grid's blocks (ceil(rows / 32), 8
// warps each) stride over its rows, about four per warp, so that the block-to-grid search
// and the record's fields are amortised over several rows.
__global__ void __launch_bounds__(256) boundary_kernel(const __grid_constant__ ElemBatch B) {
  int64_t lb;
  const int gi = batch_locate(B.row_prefix, B.ngrids, blockIdx.x, lb);
  const ElemGrid& G = B.grids[gi];
  const int64_t warps = (B.row_prefix[gi + 1] - B.row_prefix[gi]) * 8;
  const int n0 = G.dims[0], n1 = G.dims[1], n2 = G.dims[2];
  const int s0 = G.start[0], e0 = G.end[0], bc0 = G.bc[0];
  const int s1 = G.start[1], e1 = G.end[1], bc1 = G.bc[1];
  const int s2 = G.start[2], e2 = G.end[2], bc2 = G.bc[2];
  double* const f[6] = {G.f[0], G.f[1], G.f[2], G.f[3], G.f[4], G.f[5]};
  const int64_t rows = (int64_t)n1 * n2;
  const int lane = threadIdx.x & 31;
  for (int64_t row = lb * 8 + (threadIdx.x >> 5); row < rows; row += warps) {
    const int k = (int)(row / n1), j = (int)(row - (int64_t)k * n1);
    const int sj = n1 > 1 ? bc_map(j, s1, e1, bc1) : j;
    const int sk = n2 > 1 ? bc_map(k, s2, e2, bc2) : k;
    const int64_t dst = row * n0;
    const int64_t src = ((int64_t)sk * n1 + sj) * n0;
    if (sj == j && sk == k) {
      if (n0 > 1) {  // the x ghosts: i in [0, s0) and (e0, n0)
        const int lo = s0, nx = s0 + (n0 - 1 - e0);
        for (int m = lane; m < nx; m += 32) {
          const int i = m < lo ? m : e0 + 1 + (m - lo);
          const int si = bc_map(i, s0, e0, bc0);
          if (si != i) copy_cell(f, dst + i, src + si);
        }
      }
    } else {
      for (int i = lane; i < n0; i += 32)
        copy_cell(f, dst + i, src + (n0 > 1 ? bc_map(i, s0, e0, bc0) : i));
    }
  }
}

// ------------------------------------------------------------------ sibling zones
// Grid_CopyZonesFromGrid.C:100-300 (the copy3drel of every field) for a list of boxes: box
// b copies ext[0] x ext[1] x ext[2] zones of grid src, starting at s0, into grid dst at
// d0.  Blocks of 256 zones; box b owns blocks [prefix[b], prefix[b+1]).  The boxes read
// active zones and write zones outside every active region, so they never race.
struct CopyBox {
  int dst, src;
  int d0[3], s0[3], ext[3];
  int pad;
};

__global__ void __launch_bounds__(256) copy_zones_kernel(const ElemGrid* __restrict__ grids,
                                                         const CopyBox* __restrict__ boxes,
                                                         const int64_t* __restrict__ prefix,
                                                         int nboxes) {
  int64_t lb;
  const CopyBox& X = boxes[batch_locate(prefix, nboxes, blockIdx.x, lb)];
  const int64_t c = lb * 256 + threadIdx.x;
  const int64_t e0 = X.ext[0], e01 = (int64_t)X.ext[0] * X.ext[1];
  if (c >= e01 * X.ext[2]) return;
  const int k = (int)(c / e01);
  const int j = (int)((c - (int64_t)k * e01) / e0);
  const int i = (int)(c - (int64_t)k * e01 - (int64_t)j * e0);
  const ElemGrid& D = grids[X.dst];
  const ElemGrid& S = grids[X.src];
  const int64_t di =
      ((int64_t)(k + X.d0[2]) * D.dims[1] + (j + X.d0[1])) * D.dims[0] + (i + X.d0[0]);
  const int64_t si =
      ((int64_t)(k + X.s0[2]) * S.dims[1] + (j + X.s0[1])) * S.dims[0] + (i + X.s0[0]);
  double* dp[6];
  const double* sp[6];
#pragma unroll
  for (int n = 0; n < 6; ++n) {  // pointers first: the stores below may not reload them
    dp[n] = D.f[n];
    sp[n] = S.f[n];
  }
#pragma unroll
  for (int n = 0; n < 6; ++n)
    if (dp[n] && sp[n]) dp[n][di] = sp[n][si];
}

void launch_copy_zones(const ElemGrid* grids, const CopyBox* boxes, const int64_t* prefix,
                       int nboxes, int64_t blocks, cudaStream_t st) {
  copy_zones_kernel<<<(unsigned)blocks, 256, 0, st>>>(grids, boxes, prefix, nboxes);
}

// ------------------------------------------------------------------ flux correction
// grid::CorrectForRefinedFluxes (Grid_CorrectForRefinedFluxes.C:38-760) for the proper
// subgrids of one grid, Cartesian, the six hydro fields.  One phase per (subgrid, axis):
// the layers of zones just outside the subgrid's left and right faces (Offset apart);
// phases run in the reference's order, one block, a barrier between phases (two
// subgrids may correct the same zone).  Within a phase every zone is independent: the
// reference's loops over fields (outer) and zones (inner) give each zone the same
// sequence as one thread running through the fields.
struct FluxPhase {
  int start[3], dim[3];      // the left layer in this grid's zones, and its extents
  long long offset;          // from a left-layer zone to its right-layer zone
  int correct_left, correct_right;
  // flux indexes of a layer zone (i, j, k): initial ((k+io2)*id1 + (j+io1))*id0 + i+io0,
  // refined likewise with rd / ro (Grid_CorrectForRefinedFluxes.C:458-468)
  int id[3], io[3], rd[3], ro[3];
  int subling;               // SUBlingGrid: refined fluxes of a sibling's subgrid
  // per field slot (d, te, v1, v2, v3, ge): initial / refined left and right fluxes,
  // indexed like the layer (null: field absent)
  const double* il[6];
  double* rl[6];
  const double* ir[6];
  double* rr[6];
};

struct FluxFix {
  double* f[6];              // fields d, te, v1, v2, v3, ge (null: absent)
  int dims[3], rank, dual;
  double tiny_number;
  int nphases;
  // colours that keep their fraction of the density (species): device array of nspecies
  // field pointers, divided by the density before the corrections and multiplied by the
  // corrected density after them (Grid_CorrectForRefinedFluxes.C:397-421, :849-866)
  double* const* species;
  int nspecies;
};

__global__ void __launch_bounds__(256) correct_fluxes_kernel(const FluxFix X,
                                                             const FluxPhase* __restrict__ ph) {
  // correction order: density and the energies first, then the velocities
  // (Grid_CorrectForRefinedFluxes.C:288-350): slots d, te, ge, v1, v2, v3
  const int order[6] = {0, 1, 5, 2, 3, 4};
  double* const* F = X.f;
  for (int n = 0; n < X.nphases; ++n) {
    const FluxPhase& P = ph[n];
    const long long nz = (long long)P.dim[0] * P.dim[1] * P.dim[2];
    for (long long z = threadIdx.x; z < nz; z += blockDim.x) {
      const int i = (int)(z % P.dim[0]);
      const int j = (int)((z / P.dim[0]) % P.dim[1]);
      const int k = (int)(z / ((long long)P.dim[0] * P.dim[1]));
      const long long c = ((long long)(k + P.start[2]) * X.dims[1] + (j + P.start[1])) * X.dims[0] +
                          (i + P.start[0]);
      const long long c2 = c + P.offset;
      const long long x = ((long long)(k + P.io[2]) * P.id[1] + (j + P.io[1])) * P.id[0] +
                          (i + P.io[0]);
      const long long xr = ((long long)(k + P.ro[2]) * P.rd[1] + (j + P.ro[1])) * P.rd[0] +
                           (i + P.ro[0]);
      const bool sub = P.subling != 0;
      // conserved quantities on both layers (:370-394): every field but density; species
      // as fractions of the density (:397-421)
      for (int s = 1; s < 6; ++s)
        if (F[s]) {
          F[s][c] *= F[0][c];
          F[s][c2] *= F[0][c2];
        }
      for (int s = 0; s < X.nspecies; ++s) {
        double* q = X.species[s];
        q[c] /= F[0][c];
        q[c2] /= F[0][c2];
      }
      for (int q = 0; q < 6; ++q) {
        const int f = order[q];
        if (!F[f]) continue;
        // a SUBling's correction uses its opposite face (:495-542)
        if (P.correct_left) {
          const double amount = sub ? -(P.il[f][x] - P.rr[f][xr]) : P.il[f][x] - P.rl[f][x];
          F[f][c] += amount;
        }
        if (P.correct_right) {
          const double amount = sub ? P.ir[f][x] - P.rl[f][xr] : -(P.ir[f][x] - P.rr[f][x]);
          F[f][c2] += amount;
        }
        if (f == 0 || f == 1 || f == 5) {  // density and the energies stay positive
          if (P.correct_left && F[f][c] <= 0) {
            for (int u = 0; u < 6; ++u) {
              const int g = order[u];
              if (!F[g]) continue;
              if (sub) {
                if (u <= q) F[g][c] -= -(P.il[g][x] - P.rr[g][xr]);
                P.rr[g][xr] = P.il[g][x];
              } else {
                if (u <= q) F[g][c] -= (P.il[g][x] - P.rl[g][x]);
                P.rl[g][x] = P.il[g][x];
              }
            }
          }
          if (P.correct_right && F[f][c2] <= 0) {
            for (int u = 0; u < 6; ++u) {
              const int g = order[u];
              if (!F[g]) continue;
              if (sub) {
                // the reference subtracts the triggering field's amount here (:643-645)
                if (u <= q) F[g][c2] -= (P.ir[f][x] - P.rl[f][xr]);
                P.rl[g][xr] = P.ir[g][x];
              } else {
                if (u <= q) F[g][c2] -= -(P.ir[g][x] - P.rr[g][x]);
                P.rr[g][x] = P.ir[g][x];
              }
            }
          }
        }
      }
      // back to specific quantities (:683-700)
      for (int s = 1; s < 6; ++s)
        if (F[s]) {
          F[s][c] /= F[0][c];
          F[s][c2] /= F[0][c2];
        }
      // gas and total energy consistent again (:704-742)
      if (X.dual) {
        F[5][c] = dmax(F[5][c], X.tiny_number);
        F[5][c2] = dmax(F[5][c2], X.tiny_number);
        F[1][c] = F[5][c] + 0.5 * F[2][c] * F[2][c];
        F[1][c2] = F[5][c2] + 0.5 * F[2][c2] * F[2][c2];
        if (X.rank > 1) {
          F[1][c] += 0.5 * F[3][c] * F[3][c];
          F[1][c2] += 0.5 * F[3][c2] * F[3][c2];
        }
        if (X.rank > 2) {
          F[1][c] += 0.5 * F[4][c] * F[4][c];
          F[1][c2] += 0.5 * F[4][c2] * F[4][c2];
        }
      }
      // species back to densities with the corrected density (:849-866)
      for (int s = 0; s < X.nspecies; ++s) {
        double* q = X.species[s];
        q[c] *= F[0][c];
        q[c2] *= F[0][c2];
      }
    }
    __syncthreads();  // the next phase may touch the same zones
  }
}

void launch_correct_fluxes(const FluxFix& X, const FluxPhase* phases, cudaStream_t st) {
  correct_fluxes_kernel<<<1, 256, 0, st>>>(X, phases);
}

// ------------------------------------------------------------------ comoving expansion
// grid::ComovingExpansionTerms for PPM (Grid_ComovingExpansionTerms.C:36-99 with
// expand_terms.F, ENERGY_METHOD3 / VELOCITY_METHOD3) over every cell of every grid:
// the pressure at the mid time, interpolated between the old and current fields
// (Grid_ComputePressure.C:168-223) or at the current time, with
// MinimumSupportEnergyCoefficient 0 (ComputePressure's default); then the gas energy,
// total energy and velocity terms of the cell.
__device__ __forceinline__ double cell_pressure_interp(const ElemGrid& G, int64_t i,
                                                       const ElemBatch& B) {
  const double coef = B.coef_new, coefold = B.coef_old;
  double velocity2 = 0.0, velocity3 = 0.0, gas_energy;
  const double total_energy = coef * __ldg(G.te + i) + coefold * __ldg(G.old[1] + i);
  const double density = coef * __ldg(G.d + i) + coefold * __ldg(G.old[0] + i);
  const double velocity1 = coef * __ldg(G.v[0] + i) + coefold * __ldg(G.old[2] + i);
  if (G.v[1]) velocity2 = coef * __ldg(G.v[1] + i) + coefold * __ldg(G.old[3] + i);
  if (G.v[2]) velocity3 = coef * __ldg(G.v[2] + i) + coefold * __ldg(G.old[4] + i);
  if (!G.ge) {
    const double kineticE =
        0.5 * (velocity1 * velocity1 + velocity2 * velocity2 + velocity3 * velocity3);
    gas_energy = total_energy - kineticE;
  } else {
    gas_energy = coef * __ldg(G.ge + i) + coefold * __ldg(G.old[5] + i);
  }
  const double gm1 = B.gamma - 1.0;
  double p = gm1 * density * gas_energy;
  if (p < B.tiny_number) p = B.tiny_number;
  const double min_pressure = 0.0 * gm1 * density * density;  // coefficient 0
  if (p < min_pressure) p = min_pressure;
  return p;
}

__global__ void __launch_bounds__(256) expansion_kernel(const __grid_constant__ ElemBatch B) {
  int64_t lb;
  const ElemGrid& G = B.grids[batch_locate(B.size_prefix, B.ngrids, blockIdx.x, lb)];
  const int64_t i = lb * 256 + threadIdx.x;
  if (i >= G.size) return;
  const double p = B.interpolate ? cell_pressure_interp(G, i, B)
                                 : cell_pressure(G, i, B.gamma, B.tiny_number, 0.0);
  const double coef = B.expansion;
  double* d = G.f[0];
  double* e = G.f[1];
  if (G.f[5]) {  // gas energy (idual = 1)
    double* ge = G.f[5];
    ge[i] = ge[i] * (1.0 - coef) / (1.0 + coef);
  }
  double en = e[i] * (1.0 - coef) / (1.0 + coef);
  const double a = en - coef * (3.0 - 2.0 / (B.gamma - 1.0)) * p / d[i];
  const double b = 0.5 * en;
  e[i] = a > b ? a : b;
  for (int c = 0; c < G.rank; ++c) {
    double* vel = G.f[2 + c];
    vel[i] = vel[i] * (1.0 - 0.5 * coef) / (1.0 + 0.5 * coef);
  }
}

// ------------------------------------------------------------------ launchers
void launch_pressure_batch(const ElemBatch& B, int64_t blocks, cudaStream_t st) {
  pressure_kernel<<<(unsigned)blocks, 256, 0, st>>>(B);
}

void launch_timestep_batch(const ElemBatch& B, int64_t blocks, double courant, double* dt_out,
                           cudaStream_t st) {
  cudaMemsetAsync(B.min_bits, 0xFF, sizeof(unsigned long long), st);
  timestep_kernel<<<(unsigned)blocks, 256, 0, st>>>(B);
  timestep_finalize_kernel<<<1, 32, 0, st>>>(B.min_bits, courant, dt_out);
}

// The time step folded into a solve's last sweep: reset before it, finalise after it.
void launch_cfl_reset(unsigned long long* min_bits, cudaStream_t st) {
  cudaMemsetAsync(min_bits, 0xFF, sizeof(unsigned long long), st);
}

void launch_cfl_finalize(const unsigned long long* min_bits, double courant, double* dt_out,
                         cudaStream_t st) {
  timestep_finalize_kernel<<<1, 32, 0, st>>>(min_bits, courant, dt_out);
}

void launch_expansion_batch(const ElemBatch& B, int64_t blocks, cudaStream_t st) {
  expansion_kernel<<<(unsigned)blocks, 256, 0, st>>>(B);
}

void launch_boundary_batch(const ElemBatch& B, int64_t blocks, cudaStream_t st) {
  boundary_kernel<<<(unsigned)blocks, 256, 0, st>>>(B);
}

}  // namespace ppm
