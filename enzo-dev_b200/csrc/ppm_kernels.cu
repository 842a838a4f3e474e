// ppm_kernels.cu -- the grid-wide kernels around the sweeps (sm_100a):
//
//   pressure_kernel           grid::ComputePressure (time == Time)
//   timestep_kernel           calc_dt (ihydro = 0) min-reduction + Courant factor
//   boundary_kernel           outflow / periodic ghost-zone fill of one grid
//
// The directional sweeps themselves are in ppm_split.cu.
#include <cuda_runtime.h>

#include "ppm_device.cuh"
#include "ppm_sweep.cuh"

namespace ppm {

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
