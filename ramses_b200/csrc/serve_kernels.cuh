// serve_kernels.cuh -- FP64 bookkeeping kernels of the serving engine: the
// initial CFL time step of a dense problem and the per-problem clock advance
// after each batched step. Compiled without multiply-add contraction so the
// clocks are bitwise those of the single-problem path (reduce_partials_kernel
// modes 0 and 1).
#pragma once
#include <cstdint>

#include "rb_aux.cuh"
#include "stream_kernel.cuh"

namespace rb {

// Largest CFL wave speed (cmpdt, godunov_utils.f90:5-120) over a dense
// problem; combined across blocks by an integer max on the bit patterns of
// non-negative doubles, which is exact and order-independent.
static __global__ void __launch_bounds__(256) dense_cfl_kernel(const double* __restrict__ u, int64_t n,
                                                        rb_hydro_params hp, unsigned long long* __restrict__ smax_bits) {
  double smax = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double q[5];
    for (int v = 0; v < 5; v++) q[v] = u[v * n + i];
    smax = fmx(smax, cfl_speed(q, hp));
  }
  for (int o = 16; o > 0; o >>= 1) smax = fmx(smax, __shfl_xor_sync(0xffffffffu, smax, o));
  if ((threadIdx.x & 31) == 0) atomicMax(smax_bits, (unsigned long long)__double_as_longlong(smax));
}

// clock = (dt, t0, 0, 0, 0, steps=0, done, -) from the largest wave speed,
// as courant_fine + newdt_fine give the first dt (dtnew = min(boxlen/smallc,
// courant_factor*dx/smallc, min cell dt)).
static __global__ void dense_clock_init_kernel(double* __restrict__ clock, const unsigned long long* __restrict__ smax_bits,
                                        double t0, double t_end, double max_steps, double dt_max, double dt0,
                                        double dx, double courant_factor) {
  const double smax = __longlong_as_double((long long)*smax_bits);
  const double dt_cell = smax > 0.0 ? cfl_dt_from_speed(smax, dx, courant_factor) : 1.0e300;
  clock[0] = fmn(dt_max, fmn(dt0, dt_cell));
  clock[1] = t0;
  clock[2] = clock[3] = clock[4] = 0.0;
  clock[5] = 0.0;
  clock[6] = (!(t0 < t_end) || !(0.0 < max_steps)) ? 1.0 : 0.0;
  clock[7] = 0.0;
}

// After one batched step: one CTA per problem reduces the problem's CFL
// partials, advances t by the dt just used, sets the next dt, counts the step
// and raises the done flag when the stop rule is met. Finished problems are
// left untouched.
static __global__ void __launch_bounds__(RB_RED_NT) batch_clock_kernel(const BatchDesc* __restrict__ desc,
                                                                const int32_t* __restrict__ item_off) {
  const BatchDesc& d = desc[blockIdx.x];
  double* clock = d.clock;
  if (clock[6] != 0.0) return;
  __shared__ double red[4][RB_RED_NT];
  reduce4_block(d.a.partial, item_off[blockIdx.x + 1] - item_off[blockIdx.x], red);
  if (threadIdx.x == 0) {
    const double dt_lev = fmn(d.dt0, red[0][0]);
    clock[1] = clock[1] + clock[0];
    clock[0] = fmn(d.dt_max, dt_lev);
    clock[2] = red[1][0]; clock[3] = red[2][0]; clock[4] = red[3][0];
    clock[5] = clock[5] + 1.0;
    clock[6] = (!(clock[1] < d.t_end) || !(clock[5] < d.max_steps)) ? 1.0 : 0.0;
  }
}

}  // namespace rb
