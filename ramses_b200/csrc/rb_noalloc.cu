// rb_noalloc.cu -- CFL reduction (courant_fine's time step and totals) that
// allocates no memory: its per-block scratch is a fixed file-scope device
// array instead of a cudaMalloc'd buffer.
//
// Who needs it: callers that cannot call cudaMalloc/cudaFree in the middle of
// their work. Those calls block until the whole device is idle, so a host loop
// that keeps several problems in flight on one stream, or code running under a
// fixed device-memory budget owned by another allocator (a Fortran host with
// its own pool), must not trigger them. This entry point only launches
// kernels on the caller's stream.
//
// Limits and sharing: the scratch holds one partial per 256 cells, for at most
// RB_NOALLOC_MAX_CELLS cells; larger inputs are rejected. Every GPU that loads
// the library holds the array (2 MiB) until the process exits. All calls share
// it and it keeps the last call's partials; every call overwrites exactly the
// partials it reads, so nothing needs clearing, but calls that overlap on the
// GPU (two streams at once) race on it. The first call on each device looks up
// the array's device address (cudaGetSymbolAddress) and should come before any
// stream capture.
// Compiled with --fmad=false like the rest of the FP64 code.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/ramses_b200.h"
#include "hydro_core.cuh"
#include "rb_error.h"

#define RB_NOALLOC_NT 256
#define RB_NOALLOC_MAX_BLOCKS 65536

static __device__ __align__(256) double g_cfl_scratch[RB_NOALLOC_MAX_BLOCKS * 4];

namespace {

constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_mu;

// one (CFL dt, mass, E, eint) partial per block of RB_NOALLOC_NT cells
__global__ void __launch_bounds__(RB_NOALLOC_NT) noalloc_cfl_partial(const double* __restrict__ u, int64_t n,
                                                                     int64_t stride, double dx, rb_hydro_params hp,
                                                                     double* __restrict__ partial) {
  using namespace rb;
  const double vol = dx * dx * dx;
  double smax = 0.0, mass = 0.0, etot = 0.0, eint = 0.0;
  const int64_t i = blockIdx.x * (int64_t)RB_NOALLOC_NT + threadIdx.x;
  if (i < n) {
    double c[5];
    for (int v = 0; v < 5; v++) c[v] = u[v * stride + i];
    mass = c[0] * vol;
    etot = c[4] * vol;
    double ei = c[4] * vol;
    for (int d = 1; d <= 3; d++) ei = ei - 0.5 * (c[d] * c[d]) / fmx(c[0], hp.smallr) * vol;
    eint = ei;
    smax = cfl_speed(c, hp);
  }
  __shared__ double red[4][RB_NOALLOC_NT / 32];
  for (int o = 16; o > 0; o >>= 1) {
    smax = fmx(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    mass += __shfl_xor_sync(0xffffffffu, mass, o);
    etot += __shfl_xor_sync(0xffffffffu, etot, o);
    eint += __shfl_xor_sync(0xffffffffu, eint, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { red[0][w] = smax; red[1][w] = mass; red[2][w] = etot; red[3][w] = eint; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < RB_NOALLOC_NT / 32; k++) {
      smax = fmx(smax, red[0][k]); mass += red[1][k]; etot += red[2][k]; eint += red[3][k];
    }
    partial[blockIdx.x * 4 + 0] = smax > 0.0 ? cfl_dt_from_speed(smax, dx, hp.courant_factor) : 1.0e300;
    partial[blockIdx.x * 4 + 1] = mass;
    partial[blockIdx.x * 4 + 2] = etot;
    partial[blockIdx.x * 4 + 3] = eint;
  }
}

// fixed-order reduction of the partials; out = (dt, mass, E, eint) with
// dt = min(dt_in, courant_factor*dx/smallc, min cell dt) as courant_fine
__global__ void __launch_bounds__(1024) noalloc_cfl_final(const double* __restrict__ partial, int nblk,
                                                          double dt_in, double dt0, double* __restrict__ out) {
  using namespace rb;
  __shared__ double red[4][1024];
  double dtm = 1.0e300, mass = 0.0, etot = 0.0, eint = 0.0;
  for (int k = threadIdx.x; k < nblk; k += 1024) {
    dtm = fmn(dtm, partial[k * 4 + 0]);
    mass += partial[k * 4 + 1];
    etot += partial[k * 4 + 2];
    eint += partial[k * 4 + 3];
  }
  red[0][threadIdx.x] = dtm; red[1][threadIdx.x] = mass; red[2][threadIdx.x] = etot; red[3][threadIdx.x] = eint;
  __syncthreads();
  for (int h = 512; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      red[0][threadIdx.x] = fmn(red[0][threadIdx.x], red[0][threadIdx.x + h]);
      red[1][threadIdx.x] += red[1][threadIdx.x + h];
      red[2][threadIdx.x] += red[2][threadIdx.x + h];
      red[3][threadIdx.x] += red[3][threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = fmn(dt_in, fmn(dt0, red[0][0]));
    out[1] = red[1][0];
    out[2] = red[2][0];
    out[3] = red[3][0];
  }
}

}  // namespace

extern "C" int rb_courant_cells_noalloc(const rb_hydro_params* hp, const double* d_u, int64_t ncell,
                                        int64_t stride, double dx, double dt_in, double* d_out, void* stream) {
  using rbi::fail;
  if (!hp || !d_u || !d_out) return fail(RB_ERR_INVALID, "rb_courant_cells_noalloc: null argument");
  if (ncell < 1 || stride < ncell || !(dx > 0.0))
    return fail(RB_ERR_INVALID, "rb_courant_cells_noalloc: need ncell >= 1, stride >= ncell and dx > 0 "
                "(ncell=%lld, stride=%lld, dx=%g)", (long long)ncell, (long long)stride, dx);
  if (ncell > RB_NOALLOC_MAX_CELLS)
    return fail(RB_ERR_CAPACITY, "rb_courant_cells_noalloc: %lld cells exceed the fixed scratch capacity of %lld "
                "cells", (long long)ncell, (long long)RB_NOALLOC_MAX_CELLS);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return fail(RB_ERR_NO_DEVICE, "rb_courant_cells_noalloc: no usable current CUDA device");
  }
  double* scratch;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
      // the host-side name g_cfl_scratch is not a device address: look it up
      // once per device, with that device current
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_cfl_scratch);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return fail(RB_ERR_CUDA, "rb_courant_cells_noalloc: cudaGetSymbolAddress of the scratch array failed: %s",
                    cudaGetErrorString(e));
      }
      g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nblk = (int)((ncell + RB_NOALLOC_NT - 1) / RB_NOALLOC_NT);
  noalloc_cfl_partial<<<nblk, RB_NOALLOC_NT, 0, s>>>(d_u, ncell, stride, dx, *hp, scratch);
  const double dt0 = hp->courant_factor * dx / hp->smallc;
  noalloc_cfl_final<<<1, 1024, 0, s>>>(scratch, nblk, dt_in, dt0, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(RB_ERR_CUDA, "rb_courant_cells_noalloc: launch failed: %s", cudaGetErrorString(e));
  return RB_OK;
}
