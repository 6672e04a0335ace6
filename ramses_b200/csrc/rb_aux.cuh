// rb_aux.cuh -- FP64 kernels around the godunov tile kernel: coarse-to-fine
// prolongation, deterministic fine-to-coarse flux correction, the CFL
// reduction, set_unew/set_uold, restriction, and layout permutations between
// the Fortran arrays and the device layout.
//
// Device layout: variable-major, then oct-major: u[v*ncell + dc] with
// dc = icell-1 for the ncoarse coarse cells and dc = ncoarse + 8*(igrid-1) +
// (ind-1) for child slot ind of oct igrid, so an oct's 8 cells of one
// variable are one 64-byte row.
#pragma once
#include <cstdint>

#include "hydro_core.cuh"

namespace rb {

// early exit of a level kernel when the device clock says the run is over
#define RB_GATE(g)                                \
  do {                                            \
    if ((g) != nullptr && *(g) != 0.0) return;    \
  } while (0)

__device__ __forceinline__ int64_t dev_cell_of_fortran(int64_t icell /*1-based*/, int32_t ncoarse,
                                                       int32_t ngridmax) {
  if (icell <= ncoarse) return icell - 1;
  const int64_t r = icell - 1 - ncoarse;
  const int64_t ind = r / ngridmax, ig = r % ngridmax;  // ig = igrid-1
  return ncoarse + ig * 8 + ind;
}

// Fortran uold(ncell,5) -> device layout. The coarse cells keep their index;
// oct cell ncoarse + ind*ngridmax + ig in Fortran (ind the child, ig =
// igrid-1) is device cell ncoarse + ig*8 + ind. The loop runs in device
// order, so a warp (4 octs x 8 children) writes 256 contiguous device bytes
// and reads one 32-byte sector in each of the 8 Fortran rows; the nvar values
// of a cell are in flight together.
static __global__ void permute_f2d_kernel(const double* __restrict__ f, double* __restrict__ d, int64_t ncell,
                                          int32_t ncoarse, int32_t ngridmax, int nvar) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ncell; i += stride) {
    int64_t fi = i;
    if (i >= ncoarse) {
      const int64_t r = i - ncoarse;
      fi = ncoarse + (r & 7) * (int64_t)ngridmax + (r >> 3);
    }
    double x[5];
#pragma unroll
    for (int v = 0; v < 5; v++)
      if (v < nvar) x[v] = f[v * ncell + fi];
#pragma unroll
    for (int v = 0; v < 5; v++)
      if (v < nvar) d[v * ncell + i] = x[v];
  }
}
// Device layout -> Fortran: Fortran order (whole Fortran rows written), one
// value per iteration; the device reads of a warp hit 32 octs' cells of one
// child, and the other children's warps find those sectors in L2.
static __global__ void permute_d2f_kernel(const double* __restrict__ d, double* __restrict__ f, int64_t ncell,
                                          int32_t ncoarse, int32_t ngridmax, int nvar) {
  const int64_t n = ncell * nvar;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = i / ncell, icell = i % ncell + 1;
    f[i] = d[v * ncell + dev_cell_of_fortran(icell, ncoarse, ngridmax)];
  }
}
// The cells of one level's octs between the staging copy of uold in the
// Fortran layout (f) and the device layout (d): thread i handles cell ind =
// i % 8 of the oct act[i / 8] (igrid-1), so the device side is contiguous
// and the Fortran side reads whole sectors of consecutive igrids.
template <bool F2D>
static __global__ void permute_level_kernel(double* __restrict__ f, double* __restrict__ d,
                                            const int32_t* __restrict__ act, int64_t noct, int64_t ncell,
                                            int32_t ncoarse, int32_t ngridmax) {
  const int64_t n = noct * 8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = act[i >> 3];
    const int ind = (int)(i & 7);
    const int64_t fi = ncoarse + (int64_t)ind * ngridmax + g, di = ncoarse + 8 * g + ind;
#pragma unroll
    for (int v = 0; v < 5; v++) {
      if (F2D) d[v * ncell + di] = f[v * ncell + fi];
      else f[v * ncell + fi] = d[v * ncell + di];
    }
  }
}
// d[idx[i]] = v[i]: the son entries that changed in a tree re-sync
static __global__ void scatter_son_kernel(int32_t* __restrict__ d, const int64_t* __restrict__ idx,
                                          const int32_t* __restrict__ v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[idx[i]] = v[i];
}

static __global__ void permute_son_kernel(const int32_t* __restrict__ f, int32_t* __restrict__ d, int64_t ncell,
                                   int32_t ncoarse, int32_t ngridmax) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ncell; i += (int64_t)gridDim.x * blockDim.x)
    d[dev_cell_of_fortran(i + 1, ncoarse, ngridmax)] = f[i];
}

// Internal energy E - d/2 (u^2+v^2+w^2), d = max(rho, smallr), u = m/d, of
// set_unew, add_pdv_source_terms and set_uold's pressure fix
// (godunov_fine.f90:75-81, 396-401, 208-213).
__device__ __forceinline__ double pf_eint(const double u[5], double smallr) {
  const double d = fmx(u[0], smallr);
  const double uu = u[1] / d, vv = u[2] / d, ww = u[3] / d;
  return u[4] - 0.5 * d * (uu * uu + vv * vv + ww * ww);
}

// pressure fix of one cell (godunov_fine.f90:203-227, hexp = 0) on its new
// state u: E = enew + ekin where E - ekin < beta_fix d (|divu| dx/dt)^2.
__device__ __forceinline__ void pf_fix_cell(double u[5], double divu, double enew, double dx, double dt,
                                            double smallr, double beta_fix) {
  const double hexp = 0.0;
  const double d = fmx(u[0], smallr);
  const double uu = u[1] / d, vv = u[2] / d, ww = u[3] / d;
  const double e_kin = 0.5 * d * (uu * uu + vv * vv + ww * ww);
  const double e_cons = u[4] - e_kin;
  const double div = fabs(divu) * dx / dt;
  const double mx = fmx(div, 3.0 * hexp * dx);
  const double e_trunc = beta_fix * d * (mx * mx);
  if (e_cons < e_trunc) u[4] = enew + e_kin;
}

// pressure_fix part of set_unew (godunov_fine.f90:71-86): divu = 0 and enew
// = the internal energy of uold, for every cell of the active octs.
static __global__ void pf_set_unew_kernel(const double* __restrict__ uold, double* __restrict__ divu,
                                          double* __restrict__ enew, const int32_t* __restrict__ active,
                                          int32_t noct, int64_t ncell, int32_t ncoarse, double smallr,
                                          const double* __restrict__ gate) {
  RB_GATE(gate);
  const int64_t n = (int64_t)noct * 8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t dc = ncoarse + (int64_t)active[i >> 3] * 8 + (i & 7);
    double u[5];
    for (int v = 0; v < 5; v++) u[v] = uold[v * ncell + dc];
    divu[dc] = 0.0;
    enew[dc] = pf_eint(u, smallr);
  }
}

// add_pdv_source_terms (godunov_fine.f90:287-432): enew -= (gamma-1) eold
// div(u) dt, with div(u) = sum over directions of (v_right - v_left) /
// (dx_left + dx_right) from the uold velocities of the neighbouring cells;
// a neighbour whose oct does not exist is its coarse father cell at 1.5 dx.
// nres6[p*6 + j] resolves nbor(igrid, j+1) of the level's oct p: >= 0 the
// device cell of child 0 of the neighbouring oct at this level, else
// -(device cell of the coarse neighbour) - 1. dt: *dt_dev if non-null, else
// dt_val. dx_pow2: dx_loc is a power of two, so the quotient by 2 dx_loc is
// the product with its exact reciprocal.
static __global__ void pdv_kernel(const double* __restrict__ uold, const int32_t* __restrict__ active,
                                  const int64_t* __restrict__ nres6, int32_t noct, int64_t ncell,
                                  int32_t ncoarse, double dx_loc, int dx_pow2, const double* __restrict__ dt_dev,
                                  double dt_val, rb_hydro_params hp, double* __restrict__ enew,
                                  const double* __restrict__ gate) {
  RB_GATE(gate);
  const double dt = dt_dev ? *dt_dev : dt_val;
  const double inv_2dx = 1.0 / (dx_loc + dx_loc);
  const int64_t n = (int64_t)noct * 8;
  // 8 consecutive lanes hold one oct's cells: a neighbour inside the oct
  // hands over its velocity by a shuffle (the same IEEE quotient the
  // reference forms again); the loop bound keeps whole warps in it
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x; i0 < n; i0 += nthreads) {
    const int64_t i = i0 + threadIdx.x;
    const bool live = i < n;
    const int64_t p = live ? i >> 3 : 0;
    const int ind = (int)(i & 7);
    const int64_t g = live ? active[p] : 0;
    const int64_t dc = ncoarse + g * 8 + ind;
    double u[5] = {1.0, 0.0, 0.0, 0.0, 1.0};
    if (live)
      for (int v = 0; v < 5; v++) u[v] = uold[v * ncell + dc];
    const double d0 = fmx(u[0], hp.smallr);
    const double own[3] = {u[1] / d0, u[2] / d0, u[3] / d0};
    double divu_loc = 0.0;
    for (int d = 0; d < 3; d++) {
      const int bit = (ind >> d) & 1, jnd = ind ^ (1 << d);
      // the velocity of the neighbour inside the oct (lane ^ (1 << d))
      const double inner = __shfl_xor_sync(0xffffffffu, own[d], 1 << d);
      // the other neighbour along d: left if bit == 0, right if bit == 1
      const int64_t r = live ? nres6[p * 6 + 2 * d + bit] : 0;
      const bool coarse = r < 0;
      const int64_t nb = coarse ? -r - 1 : r + jnd;
      const double outer = uold[(int64_t)(1 + d) * ncell + nb] / fmx(uold[nb], hp.smallr);
      const double dx_out = coarse ? dx_loc * 1.5 : dx_loc;
      const double vl = bit ? inner : outer, vr = bit ? outer : inner;
      const double den = bit ? dx_loc + dx_out : dx_out + dx_loc;
      const double diff = vr - vl;
      divu_loc = divu_loc + ((dx_pow2 && !coarse) ? diff * inv_2dx : diff / den);
    }
    // eold = E - d/2 (u^2+v^2+w^2) with the velocities above
    const double eold = u[4] - 0.5 * d0 * (own[0] * own[0] + own[1] * own[1] + own[2] * own[2]);
    if (live) enew[dc] = enew[dc] - (hp.gamma - 1.0) * eold * divu_loc * dt;
  }
}

// pressure fix of set_uold (godunov_fine.f90:203-227, hexp = 0: no
// cosmology): where the conservative internal energy E - ekin falls below
// beta_fix * d * (|divu| dx/dt)^2, E = enew + ekin. Runs on uold after the
// copy from unew; skip_split leaves the split cells alone (upload_fine has
// overwritten them with the restriction, which in the reference follows
// the fix).
static __global__ void pf_fix_kernel(double* __restrict__ uold, const double* __restrict__ divu,
                                     const double* __restrict__ enew, const int32_t* __restrict__ son,
                                     const int32_t* __restrict__ active, int32_t noct, int64_t ncell,
                                     int32_t ncoarse, double dx, const double* __restrict__ dt_dev, double dt_val,
                                     double smallr, double beta_fix, int skip_split,
                                     const double* __restrict__ gate) {
  RB_GATE(gate);
  const double dt = dt_dev ? *dt_dev : dt_val;
  const int64_t n = (int64_t)noct * 8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t dc = ncoarse + (int64_t)active[i >> 3] * 8 + (i & 7);
    if (skip_split && son[dc] > 0) continue;
    double u[5];
    for (int v = 0; v < 5; v++) u[v] = uold[v * ncell + dc];
    pf_fix_cell(u, divu[dc], enew[dc], dx, dt, smallr, beta_fix);
    uold[4 * ncell + dc] = u[4];
  }
}

// set_unew / set_uold (godunov_fine.f90:40-130, 135-232): copy the 8x5
// values of every active oct. active[] holds igrid-1.
static __global__ void copy_octs_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                 const int32_t* __restrict__ active, int32_t noct, int64_t ncell,
                                 int32_t ncoarse, const double* __restrict__ gate) {
  RB_GATE(gate);
  const int64_t n = (int64_t)noct * 8;  // one cell per iteration, its 5 variables in flight together
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t dc = ncoarse + (int64_t)active[r >> 3] * 8 + (r & 7);
    double u[5];
#pragma unroll
    for (int v = 0; v < 5; v++) u[v] = src[v * ncell + dc];
#pragma unroll
    for (int v = 0; v < 5; v++) dst[v * ncell + dc] = u[v];
  }
}

// coarse-to-fine prolongation of the level's missing neighbour blocks
// (interpol_hydro, called from godunov_fine.f90:584-592). cells7[e*7+j]: device
// cell of the father cell (j=0) and of its 6 neighbour (or neighbour-father)
// cells, as getnborfather (nbors_utils.f90:404-525) returns them.
static __global__ void interp_blocks_kernel(const double* __restrict__ uold, const int32_t* __restrict__ cells7,
                                     int32_t nentry, int64_t ncell, double* __restrict__ out,
                                     rb_hydro_params hp, const double* __restrict__ gate) {
  RB_GATE(gate);
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nentry) return;
  double u1[7][5], u2[8][5];
  for (int j = 0; j < 7; j++) {
    const int64_t dc = cells7[(int64_t)e * 7 + j];
    for (int v = 0; v < 5; v++) u1[j][v] = uold[v * ncell + dc];
  }
  interp_children(u1, hp, u2);
  const int64_t stride = (int64_t)nentry * 8;
  for (int ind = 0; ind < 8; ind++)
    for (int v = 0; v < 5; v++) out[v * stride + (int64_t)e * 8 + ind] = u2[ind][v];
}

// The state of octs created by refinement (make_grid_fine,
// amr/refine_utils.f90:590-948, through interpol_hydro,
// hydro/interpol_hydro.f90:268-444): the 8 children of each new oct prolonged
// from its father cell and that cell's 6 getnborfather neighbours
// (cells7[e][0..6], device cell indices) and written into the oct's cells.
// Father cells are one level coarser than the new octs, so no thread reads a
// cell another thread writes.
static __global__ void prolong_new_octs_kernel(double* __restrict__ uold, const int32_t* __restrict__ cells7,
                                               const int32_t* __restrict__ octs, int32_t n, int64_t ncell,
                                               int64_t ncoarse, rb_hydro_params hp) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double u1[7][5], u2[8][5];
  for (int j = 0; j < 7; j++) {
    const int64_t dc = cells7[(int64_t)e * 7 + j];
    for (int v = 0; v < 5; v++) u1[j][v] = uold[v * ncell + dc];
  }
  interp_children(u1, hp, u2);
  const int64_t base = ncoarse + 8 * (int64_t)octs[e];   // octs[e] = igrid - 1
  for (int ind = 0; ind < 8; ind++)
    for (int v = 0; v < 5; v++) uold[v * ncell + base + ind] = u2[ind][v];
}

// Fine-to-coarse correction (godunov_fine.f90:798-908), applied target by
// target with the contributions in the reference's sweep order: by vector
// batch of the contributing oct, then direction, then left before right, and
// within one face its 4 fine cells in (k3,j3,i3) order.
// contrib[k] = slot*6 + face (face 0..5 = -x,+x,-y,+y,-z,+z).
// With pressure_fix (divu non-null) divu and enew get the same corrections
// from corr_tmp[slot][face][4][2] (godunov_fine.f90:831-856, 883-906).
static __global__ void apply_corrections_kernel(double* __restrict__ unew, const int32_t* __restrict__ tgt,
                                         const int32_t* __restrict__ off, const int32_t* __restrict__ contrib,
                                         int32_t ntgt, const double* __restrict__ corr_flux, int64_t ncell,
                                         const double* __restrict__ gate, double* __restrict__ divu = nullptr,
                                         double* __restrict__ enew = nullptr,
                                         const double* __restrict__ corr_tmp = nullptr) {
  RB_GATE(gate);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntgt) return;
  const int64_t dc = tgt[t];
  const double oneontwotondim = 1.0 / 8.0;
  for (int v = 0; v < 5; v++) {
    double u = unew[v * ncell + dc];
    for (int k = off[t]; k < off[t + 1]; k++) {
      const int slot = contrib[k] / 6, face = contrib[k] % 6;
      const double* fl = corr_flux + (int64_t)slot * 120 + face * 20;
      if ((face & 1) == 0) {
        for (int c = 0; c < 4; c++) u = u - fl[c * 5 + v] * oneontwotondim;
      } else {
        for (int c = 0; c < 4; c++) u = u + fl[c * 5 + v] * oneontwotondim;
      }
    }
    unew[v * ncell + dc] = u;
  }
  if (divu) {
    for (int t2 = 0; t2 < 2; t2++) {
      double* arr = t2 == 0 ? divu : enew;
      double u = arr[dc];
      for (int k = off[t]; k < off[t + 1]; k++) {
        const int slot = contrib[k] / 6, face = contrib[k] % 6;
        const double* tl = corr_tmp + (int64_t)slot * 48 + face * 8;
        if ((face & 1) == 0) {
          for (int c = 0; c < 4; c++) u = u - tl[c * 2 + t2] * oneontwotondim;
        } else {
          for (int c = 0; c < 4; c++) u = u + tl[c * 2 + t2] * oneontwotondim;
        }
      }
      arr[dc] = u;
    }
  }
}

// courant_fine (courant_fine.f90:1-159): per-block partial (min dt, mass,
// total energy, internal energy) over the leaf cells of the level's octs.
// A second single-block pass reduces the partials in a fixed order. With
// unew non-null the kernel also does the set_unew that follows courant_fine
// in amr_step (godunov_fine.f90:40-130): unew = uold for every cell.
// FAST (FP32-mixed contexts): the wave speed of cfl_speed_fast.
template <int NT, bool FAST = false>
static __global__ void __launch_bounds__(NT) courant_partial_kernel(const double* __restrict__ uold,
                                                             const int32_t* __restrict__ son,
                                                             const int32_t* __restrict__ active, int32_t noct,
                                                             int64_t ncell, int32_t ncoarse, double dx,
                                                             rb_hydro_params hp, double* __restrict__ partial,
                                                             const double* __restrict__ gate,
                                                             double* __restrict__ unew = nullptr,
                                                             double* __restrict__ divu = nullptr,
                                                             double* __restrict__ enew = nullptr) {
  RB_GATE(gate);
  const double vol = dx * dx * dx;
  double smax = 0.0, mass = 0.0, etot = 0.0, eint = 0.0;
  const int64_t n = (int64_t)noct * 8;
  for (int64_t i = blockIdx.x * (int64_t)NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    const int64_t dc = ncoarse + (int64_t)active[i >> 3] * 8 + (i & 7);
    const bool leaf = son[dc] == 0;
    if (!leaf && !unew) continue;
    double u[5];
    for (int v = 0; v < 5; v++) u[v] = uold[v * ncell + dc];
    // set_unew fused in (it follows courant_fine in amr_step): every cell
    if (unew)
      for (int v = 0; v < 5; v++) unew[v * ncell + dc] = u[v];
    if (divu) {  // pressure_fix (godunov_fine.f90:71-86)
      divu[dc] = 0.0;
      enew[dc] = pf_eint(u, hp.smallr);
    }
    if (!leaf) continue;
    mass = mass + u[0] * vol;
    etot = etot + u[4] * vol;
    double ei = u[4] * vol;
    if (FAST) {
      const double ir = __drcp_rn(fmx(u[0], hp.smallr));
      for (int d = 1; d <= 3; d++) ei = ei - 0.5 * (u[d] * u[d]) * ir * vol;
    } else {
      for (int d = 1; d <= 3; d++) ei = ei - 0.5 * (u[d] * u[d]) / fmx(u[0], hp.smallr) * vol;
    }
    eint = eint + ei;
    smax = fmx(smax, FAST ? cfl_speed_fast(u, hp) : cfl_speed(u, hp));
  }
  __shared__ double red[4][NT / 32];
  for (int o = 16; o > 0; o >>= 1) {
    smax = fmx(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    mass += __shfl_xor_sync(0xffffffffu, mass, o);
    etot += __shfl_xor_sync(0xffffffffu, etot, o);
    eint += __shfl_xor_sync(0xffffffffu, eint, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { red[0][w] = smax; red[1][w] = mass; red[2][w] = etot; red[3][w] = eint; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < NT / 32; k++) {
      smax = fmx(smax, red[0][k]); mass += red[1][k]; etot += red[2][k]; eint += red[3][k];
    }
    partial[blockIdx.x * 4 + 0] = smax > 0.0 ? cfl_dt_from_speed(smax, dx, hp.courant_factor) : 1.0e300;
    partial[blockIdx.x * 4 + 1] = mass;
    partial[blockIdx.x * 4 + 2] = etot;
    partial[blockIdx.x * 4 + 3] = eint;
  }
}

// Deterministic reduction of per-block partials (min dt, mass, E, eint) by
// one CTA of RB_RED_NT threads in a fixed order.
// mode 0 (courant_fine, courant_fine.f90:33,123-127,154): out[0] = dt_in if the
//   level has no leaf cell, else min(dt_in, min(courant_factor*dx/smallc,
//   min cell dt)); out[1..3] = mass, E, eint.
// mode 1 (device clock of the uniform stepper): out[1] += out[0] (time
//   advanced by the step just taken), out[0] = the next step's dt as
//   newdt_fine + courant_fine give it, out[2..4] = totals, out[5] += 1.
#define RB_RED_NT 1024
// Fixed-order reduction of n partials [n][4] (min dt, sums of mass, E, eint)
// by one CTA of RB_RED_NT threads; the totals end up in red[0..3][0].
__device__ __forceinline__ void reduce4_block(const double* __restrict__ partial, int n,
                                              double (*red)[RB_RED_NT]) {
  double dtm = 1.0e300, mass = 0.0, etot = 0.0, eint = 0.0;
  for (int k = threadIdx.x; k < n; k += RB_RED_NT) {
    dtm = fmn(dtm, partial[k * 4 + 0]);
    mass += partial[k * 4 + 1];
    etot += partial[k * 4 + 2];
    eint += partial[k * 4 + 3];
  }
  red[0][threadIdx.x] = dtm; red[1][threadIdx.x] = mass; red[2][threadIdx.x] = etot; red[3][threadIdx.x] = eint;
  __syncthreads();
  for (int h = RB_RED_NT / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      red[0][threadIdx.x] = fmn(red[0][threadIdx.x], red[0][threadIdx.x + h]);
      red[1][threadIdx.x] += red[1][threadIdx.x + h];
      red[2][threadIdx.x] += red[2][threadIdx.x + h];
      red[3][threadIdx.x] += red[3][threadIdx.x + h];
    }
    __syncthreads();
  }
}

static __global__ void __launch_bounds__(RB_RED_NT) reduce_partials_kernel(const double* __restrict__ partial, int n,
                                                                    double dt_in, double dt_cmpdt0, int any_leaf,
                                                                    double* __restrict__ out, int mode) {
  __shared__ double red[4][RB_RED_NT];
  reduce4_block(partial, n, red);
  if (threadIdx.x == 0) {
    const double dt_lev = fmn(dt_cmpdt0, red[0][0]);
    if (mode == 0) {
      out[0] = any_leaf ? fmn(dt_in, dt_lev) : dt_in;
      out[1] = red[1][0]; out[2] = red[2][0]; out[3] = red[3][0];
    } else {
      out[1] = out[1] + out[0];
      out[0] = fmn(dt_in, dt_lev);
      out[2] = red[1][0]; out[3] = red[2][0]; out[4] = red[3][0];
      out[5] = out[5] + 1.0;
    }
  }
}

// ---- device-resident amr_step clock ----------------------------------------
// The scalar bookkeeping of amr_step (amr/amr_step.f90:320-331,571-576),
// newdt_fine (pm/newdt_fine.f90:47-51,173) and update_time's t/nstep advance
// (amr/update_time.f90:330-331) runs in single-thread kernels on one array
// `s`, so a sequence of coarse steps needs no host round trip and can be
// captured into a CUDA graph. Every level kernel of a coarse step takes
// gate = s + RB_S_DONE and returns at once when the run is over (t >= t_end or
// the requested number of coarse steps done), so a graph of K coarse steps
// stops exactly where a host loop would.
#define RB_NLV (RB_MAXLEVEL + 2)
#define RB_S_DTNEW 0
#define RB_S_DTOLD RB_NLV
#define RB_S_T (2 * RB_NLV)
#define RB_S_NSTEP (2 * RB_NLV + 1)
#define RB_S_MASS (2 * RB_NLV + 2)
#define RB_S_EKIN (2 * RB_NLV + 3)
#define RB_S_EINT (2 * RB_NLV + 4)
#define RB_S_DONE (2 * RB_NLV + 5)
#define RB_S_TEND (2 * RB_NLV + 6)
#define RB_S_MAXC (2 * RB_NLV + 7)
#define RB_S_COARSE (2 * RB_NLV + 8)
#define RB_S_SIZE (2 * RB_NLV + 16)

// start of a coarse step: decide whether it runs; reset the level totals
static __global__ void sched_gate_kernel(double* __restrict__ s) {
  const bool done = !(s[RB_S_T] < s[RB_S_TEND]) || !(s[RB_S_COARSE] < s[RB_S_MAXC]);
  s[RB_S_DONE] = done ? 1.0 : 0.0;
  if (!done) s[RB_S_MASS] = s[RB_S_EKIN] = s[RB_S_EINT] = 0.0;
}

// newdt_fine + courant_fine of level l from the level's CFL partials:
// dtold(l)=dtnew(l); dtnew(l)=min(boxlen/smallc, courant); for l>levelmin
// dtnew(l)=min(dtnew(l-1)/nsubcycle(l-1), dtnew(l)); level totals accumulated.
static __global__ void __launch_bounds__(RB_RED_NT) sched_courant_kernel(const double* __restrict__ partial, int n, int l,
                                                                  int levelmin, double dt_cmpdt0, int any_leaf,
                                                                  double dt_max, double nsub_prev,
                                                                  double* __restrict__ s) {
  if (s[RB_S_DONE] != 0.0) return;
  __shared__ double red[4][RB_RED_NT];
  reduce4_block(partial, n, red);
  if (threadIdx.x == 0) {
    s[RB_S_DTOLD + l] = s[RB_S_DTNEW + l];
    const double dt_lev = fmn(dt_cmpdt0, red[0][0]);
    const double dt_all = any_leaf ? fmn(dt_max, dt_lev) : dt_max;
    s[RB_S_MASS] = s[RB_S_MASS] + red[1][0];
    s[RB_S_EKIN] = s[RB_S_EKIN] + red[2][0];
    s[RB_S_EINT] = s[RB_S_EINT] + red[3][0];
    double dtn = fmn(dt_max, dt_all);
    if (l > levelmin) dtn = fmn(s[RB_S_DTNEW + l - 1] / nsub_prev, dtn);
    s[RB_S_DTNEW + l] = dtn;
  }
}

// the finest level of this step is l: advance t and nstep; when the next
// level exists but holds no oct (mode 1) also set its dtold/dtnew
static __global__ void sched_advance_kernel(double* __restrict__ s, int l, int mode, double nsub_l) {
  if (s[RB_S_DONE] != 0.0) return;
  if (mode == 1) {
    s[RB_S_DTOLD + l + 1] = s[RB_S_DTNEW + l] / nsub_l;
    s[RB_S_DTNEW + l + 1] = s[RB_S_DTNEW + l] / nsub_l;
  }
  s[RB_S_T] = s[RB_S_T] + s[RB_S_DTNEW + l];
  s[RB_S_NSTEP] = s[RB_S_NSTEP] + 1.0;
}

// end of amr_step(l, icount) for l > levelmin (amr_step.f90:571-576)
static __global__ void sched_end_kernel(double* __restrict__ s, int l, int nsub_prev_is_one, int icount) {
  if (s[RB_S_DONE] != 0.0) return;
  if (nsub_prev_is_one) s[RB_S_DTNEW + l - 1] = s[RB_S_DTNEW + l];
  if (icount == 2) s[RB_S_DTNEW + l - 1] = s[RB_S_DTOLD + l] + s[RB_S_DTNEW + l];
}

static __global__ void sched_finish_kernel(double* __restrict__ s) {
  if (s[RB_S_DONE] != 0.0) return;
  s[RB_S_COARSE] = s[RB_S_COARSE] + 1.0;
}

// hydro_refine (godunov_utils.f90:125-263) for one cell along one direction:
// ug, um, ud are the conservative states of the left neighbour, the cell and
// the right neighbour; they are converted to primitives in place as the
// reference does, then the relative density, pressure and velocity gradients
// are compared with their thresholds. Operation order as in the reference.
__device__ __forceinline__ bool hydro_refine_cell(double ug[5], double um[5], double ud[5],
                                                  const rb_hydro_params& hp, const rb_refine_params& rp) {
  const double half = 0.5, one = 1.0, zero = 0.0;
  ug[0] = fmx(ug[0], hp.smallr);
  um[0] = fmx(um[0], hp.smallr);
  ud[0] = fmx(ud[0], hp.smallr);
  for (int d = 1; d <= 3; d++) {
    ug[d] = ug[d] / ug[0];
    um[d] = um[d] / um[0];
    ud[d] = ud[d] / ud[0];
  }
  double eking = zero, ekinm = zero, ekind = zero;
  for (int d = 1; d <= 3; d++) {
    eking = eking + half * ug[0] * (ug[d] * ug[d]);
    ekinm = ekinm + half * um[0] * (um[d] * um[d]);
    ekind = ekind + half * ud[0] * (ud[d] * ud[d]);
  }
  ug[4] = (hp.gamma - one) * (ug[4] - eking);
  um[4] = (hp.gamma - one) * (um[4] - ekinm);
  ud[4] = (hp.gamma - one) * (ud[4] - ekind);
  bool ok = false;
  if (rp.err_grad_d >= 0.0) {
    const double dg = ug[0], dm = um[0], dd = ud[0];
    const double error = 2.0 * fmx(fabs((dd - dm) / (dd + dm + rp.floor_d)), fabs((dm - dg) / (dm + dg + rp.floor_d)));
    ok = ok || error > rp.err_grad_d;
  }
  if (rp.err_grad_p >= 0.0) {
    const double pg = ug[4], pm = um[4], pd = ud[4];
    const double error = 2.0 * fmx(fabs((pd - pm) / (pd + pm + rp.floor_p)), fabs((pm - pg) / (pm + pg + rp.floor_p)));
    ok = ok || error > rp.err_grad_p;
  }
  if (rp.err_grad_u >= 0.0) {
    for (int d = 1; d <= 3; d++) {
      const double vg = ug[d], vm = um[d], vd = ud[d];
      const double f2 = rp.floor_u * rp.floor_u;
      const double cg = sqrt(fmx(hp.gamma * ug[4] / ug[0], f2));
      const double cm = sqrt(fmx(hp.gamma * um[4] / um[0], f2));
      const double cd = sqrt(fmx(hp.gamma * ud[4] / ud[0], f2));
      const double error = 2.0 * fmx(fabs((vd - vm) / (cd + cm + fabs(vd) + fabs(vm) + rp.floor_u)),
                                     fabs((vm - vg) / (cm + cg + fabs(vm) + fabs(vg) + rp.floor_u)));
      ok = ok || error > rp.err_grad_u;
    }
  }
  return ok;
}

// hydro_flag (hydro_flag.f90:1-180): out[i] = 1 when cell i of the level's
// octs (oct i>>3, child slot i&7) meets a criterion towards its face
// neighbours along any direction. A face neighbour is the adjacent child of
// the same oct, or of the neighbouring oct (getnborgrids/getnborcells,
// nbors_utils.f90:363-399: the child slot with that direction's bit flipped),
// or, where that oct does not exist, the coarser neighbour cell
// nbor(igrid,j) itself (hydro_flag.f90:110-116). nbor6[oct*6 + j] is the
// device cell of nbor(igrid, j+1), j = 0..5 = -x,+x,-y,+y,-z,+z.
static __global__ void hydro_flag_kernel(const double* __restrict__ uold, const int32_t* __restrict__ son,
                                         const int32_t* __restrict__ active, const int32_t* __restrict__ nbor6,
                                         int32_t noct, int64_t ncell, int32_t ncoarse, rb_hydro_params hp,
                                         rb_refine_params rp, uint8_t* __restrict__ out) {
  const int64_t n = (int64_t)noct * 8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t oct = i >> 3;
    const int ch = (int)(i & 7);
    const int64_t base = ncoarse + (int64_t)active[oct] * 8;
    bool ok = false;
    for (int d = 0; d < 3; d++) {
      const int bit = 1 << d;
      int64_t cell[2];
      for (int side = 0; side < 2; side++) {  // 0: minus neighbour, 1: plus neighbour
        const bool same_oct = side == 0 ? (ch & bit) != 0 : (ch & bit) == 0;
        if (same_oct) {
          cell[side] = base + (ch ^ bit);
        } else {
          const int64_t fc = nbor6[oct * 6 + 2 * d + side];
          const int g = son[fc];
          cell[side] = g > 0 ? ncoarse + (int64_t)(g - 1) * 8 + (ch ^ bit) : fc;
        }
      }
      double ug[5], um[5], ud[5];
      for (int v = 0; v < 5; v++) {
        ug[v] = uold[v * ncell + cell[0]];
        um[v] = uold[v * ncell + base + ch];
        ud[v] = uold[v * ncell + cell[1]];
      }
      ok = hydro_refine_cell(ug, um, ud, hp, rp) || ok;
    }
    out[i] = ok ? 1 : 0;
  }
}

// upload_fine / upl (interpol_hydro.f90:5-263): restriction of every split
// cell of the level's active octs from its 8 children.
// Restriction of one split cell dc from its 8 children (oct gs).
__device__ __forceinline__ void restrict_cell(double* __restrict__ uold, int64_t dc, int gs, int64_t ncell,
                                              int32_t ncoarse, const rb_hydro_params& hp) {
  {
    const int64_t c0 = ncoarse + (int64_t)(gs - 1) * 8;
    double getx = 0.0;
    for (int is = 0; is < 8; is++) getx = getx + fmx(uold[c0 + is], hp.smallr);
    uold[dc] = getx / 8.0;
    for (int v = 1; v < 5; v++) {
      getx = 0.0;
      for (int is = 0; is < 8; is++) getx = getx + uold[v * ncell + c0 + is];
      uold[v * ncell + dc] = getx / 8.0;
    }
    if (hp.interpol_var == 1 || hp.interpol_var == 2) {
      getx = 0.0;
      for (int is = 0; is < 8; is++) {
        const int64_t sc = c0 + is;
        double ekin = 0.0;
        for (int d = 1; d <= 3; d++)
          ekin = ekin + 0.5 * (uold[d * ncell + sc] * uold[d * ncell + sc]) / fmx(uold[sc], hp.smallr);
        const double erad = 0.0;
        getx = getx + uold[4 * ncell + sc] - ekin - erad;
      }
      double ekin = 0.0;
      for (int d = 1; d <= 3; d++)
        ekin = ekin + 0.5 * (uold[d * ncell + dc] * uold[d * ncell + dc]) / fmx(uold[dc], hp.smallr);
      const double erad = 0.0;
      uold[4 * ncell + dc] = getx / 8.0 + ekin + erad;
    }
  }
}

static __global__ void upload_fine_kernel(double* __restrict__ uold, const int32_t* __restrict__ son,
                                   const int32_t* __restrict__ active, int32_t noct, int64_t ncell,
                                   int32_t ncoarse, rb_hydro_params hp, const double* __restrict__ gate) {
  RB_GATE(gate);
  const int64_t n = (int64_t)noct * 8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t dc = ncoarse + (int64_t)active[i >> 3] * 8 + (i & 7);
    const int gs = son[dc];
    if (gs > 0) restrict_cell(uold, dc, gs, ncell, ncoarse, hp);
  }
}

// set_uold followed by upload_fine on the same level (amr_step.f90:424,442),
// in one pass: set_uold copies unew to uold for every cell and upload_fine
// then overwrites every variable of the split cells with the restriction of
// their children, so each cell's final uold is written once. do_upload = 0
// where upload_fine does nothing (finest level, or no split cell). With
// pressure_fix (divu non-null) the copied cells get set_uold's energy fix
// (dt: *dt_dev if non-null, else dt_val); the split cells' fix would be
// overwritten by the restriction.
static __global__ void set_uold_upload_kernel(double* __restrict__ uold, const double* __restrict__ unew,
                                              const int32_t* __restrict__ son, const int32_t* __restrict__ active,
                                              int32_t noct, int64_t ncell, int32_t ncoarse, rb_hydro_params hp,
                                              int do_upload, const double* __restrict__ gate,
                                              const double* __restrict__ divu = nullptr,
                                              const double* __restrict__ enew = nullptr, double dx = 0.0,
                                              const double* __restrict__ dt_dev = nullptr, double dt_val = 0.0) {
  RB_GATE(gate);
  const double dt = dt_dev ? *dt_dev : dt_val;
  const int64_t n = (int64_t)noct * 8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t dc = ncoarse + (int64_t)active[i >> 3] * 8 + (i & 7);
    const int gs = do_upload ? son[dc] : 0;
    if (gs > 0) {
      restrict_cell(uold, dc, gs, ncell, ncoarse, hp);
    } else {
      double u[5];
#pragma unroll
      for (int v = 0; v < 5; v++) u[v] = unew[v * ncell + dc];
      if (divu) pf_fix_cell(u, divu[dc], enew[dc], dx, dt, hp.smallr, hp.beta_fix);
#pragma unroll
      for (int v = 0; v < 5; v++) uold[v * ncell + dc] = u[v];
    }
  }
}

// ---------------------------------------------------------------------------
// unsplit with the reference's own Fortran array layout (umuscl.f90:22-38):
// uin(nvector,-1:4,-1:4,-1:4,5), gravin(nvector,-1:4,-1:4,-1:4,3),
// flux(nvector,1:3,1:3,1:3,5,3), tmp(nvector,1:3,1:3,1:3,2,3).
// One CTA per oct (grid index l); the 32 traced cells and 36 faces the
// fluxes depend on are computed from the 6x6x6 stencil in shared memory.
// ---------------------------------------------------------------------------
static __global__ void __launch_bounds__(64) unsplit_fortran_kernel(const double* __restrict__ uin,
                                                             const double* __restrict__ gravin,
                                                             double* __restrict__ flux, double* __restrict__ tmp,
                                                             double dx, double dy, double dz, double dt,
                                                             int ngrid, int nvector, rb_hydro_params hp) {
  const int l = blockIdx.x;
  if (l >= ngrid) return;
  __shared__ double q[5][216];
  __shared__ double qm[5][3][64], qp[5][3][64];  // indexed [v][dir][cell 4x4x4 over 0..3]
  const Consts<double> c = make_consts<double>(hp);
  const int64_t nv = nvector;
  auto S6 = [&](int i, int j, int k) { return (int64_t)l + nv * ((i + 1) + 6 * ((j + 1) + 6 * (k + 1))); };
  const int64_t st = nv * 216;
  const double dtxhalf = dt * 0.5;
  for (int s = threadIdx.x; s < 216; s += 64) {
    const int i = s % 6 - 1, j = (s / 6) % 6 - 1, k = s / 36 - 1;
    double u[5];
    for (int v = 0; v < 5; v++) u[v] = uin[S6(i, j, k) + st * v];
    // ctoprim including the gravity predictor with the caller's gravin
    const double gamma = hp.gamma;
    const double smalle = hp.smallc * hp.smallc / gamma / (gamma - 1.0);
    double q1 = fmx(u[0], hp.smallr);
    double oneoverrho = 1.0 / q1;
    double q2 = u[1] * oneoverrho, q3 = u[2] * oneoverrho, q4 = u[3] * oneoverrho;
    double eken = 0.5 * q2 * q2;
    eken = eken + 0.5 * q3 * q3;
    eken = eken + 0.5 * q4 * q4;
    const double erad = 0.0;
    double eint = fmx(u[4] * oneoverrho - eken - erad, smalle);
    double q5 = (gamma - 1.0) * q1 * eint;
    q2 = q2 + gravin[S6(i, j, k)] * dtxhalf;
    q3 = q3 + gravin[S6(i, j, k) + st] * dtxhalf;
    q4 = q4 + gravin[S6(i, j, k) + 2 * st] * dtxhalf;
    q[0][s] = q1; q[1][s] = q2; q[2][s] = q3; q[3][s] = q4; q[4][s] = q5;
  }
  __syncthreads();
  const double dtd[3] = {dt / dx, dt / dy, dt / dz};
  for (int cidx = threadIdx.x; cidx < 64; cidx += 64) {
    const int i = cidx % 4, j = (cidx / 4) % 4, k = cidx / 16;  // cells 0..3
    const int s = (i + 1) + 6 * ((j + 1) + 6 * (k + 1));
    double dq[5][3];
    Prim<double> q0;
    q0.r = q[0][s]; q0.u = q[1][s]; q0.v = q[2][s]; q0.w = q[3][s]; q0.p = q[4][s];
    if (hp.slope_type == 0) {
      for (int v = 0; v < 5; v++) dq[v][0] = dq[v][1] = dq[v][2] = 0.0;
    } else if (hp.slope_type != 3) {
      const int stp[3] = {1, 6, 36};
      for (int v = 0; v < 5; v++)
        for (int d = 0; d < 3; d++)
          dq[v][d] = slope1<double>(q[v][s - stp[d]], q[v][s], q[v][s + stp[d]], hp.slope_type, hp.slope_theta);
    } else {
      for (int v = 0; v < 5; v++) {
        const double qc = q[v][s];
        double vmin = 0, vmax = 0;
        bool first = true;
        for (int kk = -1; kk <= 1; kk++)
          for (int ii = -1; ii <= 1; ii++)
            for (int jj = -1; jj <= 1; jj++) {
              const double d = q[v][s + ii + 6 * jj + 36 * kk] - qc;
              if (first) { vmin = d; vmax = d; first = false; }
              else { vmin = fmn(vmin, d); vmax = fmx(vmax, d); }
            }
        const double dfx = 0.5 * (q[v][s + 1] - q[v][s - 1]);
        const double dfy = 0.5 * (q[v][s + 6] - q[v][s - 6]);
        const double dfz = 0.5 * (q[v][s + 36] - q[v][s - 36]);
        const double dff = 0.5 * (fabs(dfx) + fabs(dfy) + fabs(dfz));
        double slop;
        if (dff > 0.0) slop = fmn(1.0, fmn(fabs(vmin), fabs(vmax)) / dff);
        else slop = 1.0;
        dq[v][0] = slop * dfx; dq[v][1] = slop * dfy; dq[v][2] = slop * dfz;
      }
    }
    Prim<double> sp[3], sm[3];
    trace_sel<double, 0>(q0, dq, c, dtd, sp, sm, 7u);
    for (int d = 0; d < 3; d++) {
      qm[0][d][cidx] = sm[d].r; qm[1][d][cidx] = sm[d].u; qm[2][d][cidx] = sm[d].v;
      qm[3][d][cidx] = sm[d].w; qm[4][d][cidx] = sm[d].p;
      qp[0][d][cidx] = sp[d].r; qp[1][d][cidx] = sp[d].u; qp[2][d][cidx] = sp[d].v;
      qp[3][d][cidx] = sp[d].w; qp[4][d][cidx] = sp[d].p;
    }
  }
  __syncthreads();
  const double ddd[3] = {dx, dy, dz};
  for (int f = threadIdx.x; f < 36; f += 64) {
    const int d = f / 12, r = f % 12;
    // face (i,j,k) in 1..3 along d, 1..2 across; left cell = face - e_d
    int i, j, k;
    if (d == 0) { i = 1 + r % 3; j = 1 + (r / 3) % 2; k = 1 + r / 6; }
    else if (d == 1) { i = 1 + r % 2; j = 1 + (r / 2) % 3; k = 1 + r / 6; }
    else { i = 1 + r % 2; j = 1 + (r / 2) % 2; k = 1 + r / 4; }
    const int cr = i + 4 * (j + 4 * k);
    const int cl = cr - (d == 0 ? 1 : d == 1 ? 4 : 16);
    Prim<double> L, Rr;
    L.r = qm[0][d][cl]; L.u = qm[1][d][cl]; L.v = qm[2][d][cl]; L.w = qm[3][d][cl]; L.p = qm[4][d][cl];
    Rr.r = qp[0][d][cr]; Rr.u = qp[1][d][cr]; Rr.v = qp[2][d][cr]; Rr.w = qp[3][d][cr]; Rr.p = qp[4][d][cr];
    double ql[5], qr[5], fg[6], fo[5];
    to_face(L, d, ql);
    to_face(Rr, d, qr);
    riemann<double>(ql, qr, c, fg);
    from_face(fg, d, fo);
    const int64_t base = (int64_t)l + nv * ((i - 1) + 3 * ((j - 1) + 3 * (k - 1)));
    const int64_t s3 = nv * 27;
    for (int v = 0; v < 5; v++) flux[base + s3 * (v + 5 * d)] = fo[v] * dt / ddd[d];
    if (hp.difmag > 0.0) {
      // consup (uplmde.f90:769-866): + dt*difmag*min(0, div1)*(u_i - u_{i-1}),
      // div1 from the face's four corner divergences (cmpdivu, :702-764)
      const double factorx = 0.5 * 0.5 / dx, factory = 0.5 * 0.5 / dy, factorz = 0.5 * 0.5 / dz;
      auto Q = [&](int ii, int jj, int kk, int v) { return q[v][(ii + 1) + 6 * ((jj + 1) + 6 * (kk + 1))]; };
      auto DV = [&](int ii, int jj, int kk) {  // corner (ii-1/2, jj-1/2, kk-1/2)
        double ux = 0.0, vy = 0.0, wz = 0.0;
        ux = ux + factorx * (Q(ii, jj, kk, 1) - Q(ii - 1, jj, kk, 1));
        ux = ux + factorx * (Q(ii, jj - 1, kk, 1) - Q(ii - 1, jj - 1, kk, 1));
        vy = vy + factory * (Q(ii, jj, kk, 2) - Q(ii, jj - 1, kk, 2) + Q(ii - 1, jj, kk, 2) - Q(ii - 1, jj - 1, kk, 2));
        ux = ux + factorx * (Q(ii, jj, kk - 1, 1) - Q(ii - 1, jj, kk - 1, 1) + Q(ii, jj - 1, kk - 1, 1) -
                             Q(ii - 1, jj - 1, kk - 1, 1));
        vy = vy + factory * (Q(ii, jj, kk - 1, 2) - Q(ii, jj - 1, kk - 1, 2) + Q(ii - 1, jj, kk - 1, 2) -
                             Q(ii - 1, jj - 1, kk - 1, 2));
        wz = wz + factorz * (Q(ii, jj, kk, 3) - Q(ii, jj, kk - 1, 3) + Q(ii, jj - 1, kk, 3) - Q(ii, jj - 1, kk - 1, 3) +
                             Q(ii - 1, jj, kk, 3) - Q(ii - 1, jj, kk - 1, 3) + Q(ii - 1, jj - 1, kk, 3) -
                             Q(ii - 1, jj - 1, kk - 1, 3));
        return ux + vy + wz;
      };
      const double factor = 0.5 * 0.5;
      double div1;
      if (d == 0) {
        div1 = factor * DV(i, j, k);
        div1 = div1 + factor * DV(i, j + 1, k);
        div1 = div1 + factor * (DV(i, j, k + 1) + DV(i, j + 1, k + 1));
      } else if (d == 1) {
        div1 = 0.0;
        div1 = div1 + factor * (DV(i, j, k) + DV(i + 1, j, k));
        div1 = div1 + factor * (DV(i, j, k + 1) + DV(i + 1, j, k + 1));
      } else {
        div1 = factor * (DV(i, j, k) + DV(i + 1, j, k) + DV(i, j + 1, k) + DV(i + 1, j + 1, k));
      }
      div1 = hp.difmag * fmn(0.0, div1);
      const int di = d == 0, dj = d == 1, dk = d == 2;
      for (int v = 0; v < 5; v++)
        flux[base + s3 * (v + 5 * d)] = flux[base + s3 * (v + 5 * d)] +
                                        dt * div1 * (uin[S6(i, j, k) + st * v] - uin[S6(i - di, j - dj, k - dk) + st * v]);
    }
    tmp[base + s3 * (0 + 2 * d)] = 0.5 * (ql[1] + qr[1]) * dt / ddd[d];
    tmp[base + s3 * (1 + 2 * d)] = fg[5] * dt / ddd[d];
  }
}

// Oct layout <-> dense Cartesian array of one complete level.
// cbase[i]: dense index of child 0 of the level's i-th active oct.
static __global__ void oct_to_dense_kernel(const double* __restrict__ u, double* __restrict__ d,
                                    const int32_t* __restrict__ active, const int64_t* __restrict__ cbase,
                                    int32_t noct, int64_t ncell, int32_t oct0, int32_t nx, int32_t ny,
                                    int64_t vstr) {
  const int64_t n = (int64_t)noct * 8;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = r >> 3;
    const int ch = (int)(r & 7);
    const int64_t di = cbase[o] + (ch & 1) + (int64_t)nx * (((ch >> 1) & 1) + (int64_t)ny * (ch >> 2));
    const int64_t oc = oct0 + (int64_t)active[o] * 8 + ch;
    double x[5];
#pragma unroll
    for (int v = 0; v < 5; v++) x[v] = u[v * ncell + oc];
#pragma unroll
    for (int v = 0; v < 5; v++) d[v * vstr + di] = x[v];
  }
}
static __global__ void dense_to_oct_kernel(const double* __restrict__ d, double* __restrict__ u,
                                    const int32_t* __restrict__ active, const int64_t* __restrict__ cbase,
                                    int32_t noct, int64_t ncell, int32_t oct0, int32_t nx, int32_t ny,
                                    int64_t vstr) {
  const int64_t n = (int64_t)noct * 8;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = r >> 3;
    const int ch = (int)(r & 7);
    const int64_t di = cbase[o] + (ch & 1) + (int64_t)nx * (((ch >> 1) & 1) + (int64_t)ny * (ch >> 2));
    const int64_t oc = oct0 + (int64_t)active[o] * 8 + ch;
    double x[5];
#pragma unroll
    for (int v = 0; v < 5; v++) x[v] = d[v * vstr + di];
#pragma unroll
    for (int v = 0; v < 5; v++) u[v * ncell + oc] = x[v];
  }
}

// make_boundary_hydro for one boundary region (hydro/hydro_boundary.f90:
// 118-208), one (boundary oct, cell) per grid-stride iteration. Boundary type bt: side
// dir = bt % 10 (1..6 = -x,+x,-y,+y,-z,+z), walls bt < 10, free boundaries
// 11..16. Cell ind of the boundary oct takes cell ind_ref of the reference oct:
// the mirror cell across the face (walls) or the cell of the reference oct
// next to the face (free), :57-76. Phase 0 stages the reference values in buf
// (walls: the normal momentum negated; free: E - ekin), phase 1 writes them
// (free: E + ekin of the written state, :194-202). The two launches keep the
// region's outer layers, whose reference octs lie in the same region, free of
// thread order.
static __global__ void boundary_fill_kernel(double* __restrict__ u, const int32_t* __restrict__ pairs, int64_t n,
                                     int64_t ncell, int32_t ncoarse, int bt, double smallr,
                                     double* __restrict__ buf, int phase, const double* __restrict__ gate) {
  RB_GATE(gate);
  const int a = (bt % 10 - 1) >> 1;  // axis of the face
  const bool wall = bt < 10;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * 8; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i >> 3;
    const int ind = (int)(i & 7);  // ind - 1
    double q[5];
    double* b = buf + (size_t)i * 5;
    if (phase == 0) {
      const int side = (bt % 10 - 1) & 1;  // 0: lower face, 1: upper face
      const int ind_ref = wall ? (ind ^ (1 << a)) : (side ? (ind | (1 << a)) : (ind & ~(1 << a)));
      const int64_t rc = ncoarse + 8 * (int64_t)pairs[2 * p + 1] + ind_ref;
#pragma unroll
      for (int v = 0; v < 5; v++) q[v] = u[v * ncell + rc];
      if (wall) {
        q[1 + a] = q[1 + a] * -1.0;
      } else {
        double ekin = 0.0;
        const double d = fmx(q[0], smallr);
        for (int idim = 1; idim <= 3; idim++) {
          const double vel = q[idim] / d;
          ekin = ekin + 0.5 * d * (vel * vel);
        }
        q[4] = q[4] - ekin;
      }
#pragma unroll
      for (int v = 0; v < 5; v++) b[v] = q[v];
    } else {
      const int64_t gc = ncoarse + 8 * (int64_t)pairs[2 * p] + ind;
#pragma unroll
      for (int v = 0; v < 5; v++) q[v] = b[v];
      if (!wall) {
        double ekin = 0.0;
        const double d = fmx(q[0], smallr);
        for (int idim = 1; idim <= 3; idim++) {
          const double vel = q[idim] / d;
          ekin = ekin + 0.5 * d * (vel * vel);
        }
        q[4] = q[4] + ekin;
      }
#pragma unroll
      for (int v = 0; v < 5; v++) u[v * ncell + gc] = q[v];
    }
  }
}

}  // namespace rb
