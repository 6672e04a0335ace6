// stream_kernel.cuh -- godunov_fine + set_uold + courant_fine for one complete
// (uniform) level held as a dense Cartesian array, as a z-streaming stencil.
//
// A CTA owns a TX x TY column of cells and a z range [z0, z0+hz). One thread
// owns one column (cx, cy) of the trace region (TX+2) x (TY+2) and marches in
// z. The conservative state of the planes ahead is prefetched with 16-byte
// cp.async into a 5-plane shared ring. The primitive state of planes k-1..k+2
// of its own column lives in registers, so the z slopes, the z face states
// and the z Riemann problems need no shared memory; the x and y neighbours
// read a 3-plane shared buffer of primitive planes. Per trace plane k
// (two CTA barriers):
//   A. ctoprim of plane k+2 (own column -> registers, every stencil column ->
//      shared buffer);
//   B. slopes + MUSCL-Hancock trace of plane k; publish the x/y left states;
//      -- barrier --; prefetch plane k+4;
//   C. Riemann: x face left of the column, y face below, z face k-1/2;
//      publish Fx, Fy; wait for plane k+3; -- barrier --
//   D. unew(k-1) = ((uold + dFx) + dFy) + dFz and the CFL wave speed of the
//      new state; partial update of plane k.
// Every face flux and cell update is the same function of the same stencil as
// in godunov_fine/unsplit, so with R = double (no FMA contraction) the result
// is bit-identical to the reference operation order.
#pragma once
#include <cstdint>

#include "cp_async.cuh"
#include "hydro_core.cuh"

namespace rb {

struct StreamArgs {
  const double* __restrict__ uin;   // [5][Nz][Ny][Nx] state at t
  double* __restrict__ uout;        // [5][Nz][Ny][Nx] state at t+dt
  double* __restrict__ partial;     // [nitems][4] (CFL dt, 0, 0, 0)
  const double* __restrict__ dt_dev;
  int32_t nx, ny, nz;               // cells per dimension (multiples of TX, TY, hz; even)
  int32_t hz;                       // z extent of one work item
  int32_t dx_pow2;
  int32_t outflow;                  // bit d: outflow (zero-gradient) boundaries along axis d, else periodic
  double dx, inv_dx;
  rb_hydro_params hp;
};

template <typename R, int TX, int TY>
struct StreamGeom {
  static constexpr int SX = TX + 4, SY = TY + 4;        // stencil plane
  static constexpr int CX = TX + 2, CY = TY + 2;        // trace columns
  static constexpr int NC = CX * CY;                    // threads owning a column
  static constexpr int NT = (NC + 31) / 32 * 32;        // launched threads (whole warps)
  static constexpr int NS = SX * SY;
  static constexpr int NEXTRA = NS - NC;                // q-only outer ring columns
  static constexpr int NRAW = 5;                        // raw planes in flight
  static constexpr int NQ = 2;                          // primitive planes in shared memory
  static constexpr int PAIRS = SY * (SX / 2);           // 16-byte (2-cell) pieces of one variable's plane
  static_assert(PAIRS <= NT, "one plane piece per thread");
  static constexpr size_t RAW_BYTES = sizeof(double) * NRAW * 5 * NS;
  static constexpr size_t Q_BYTES = sizeof(R) * NQ * 5 * NS;
  // Fx, Fy (face fluxes times dt/dx, FP64: in the mixed path the FP32
  // product is widened once, by the face's owner) and qm_x, qm_y
  static constexpr size_t X_BYTES = sizeof(double) * 2 * 5 * NC + sizeof(R) * 2 * 5 * NC;
  static constexpr size_t SMEM = RAW_BYTES + Q_BYTES + X_BYTES;
  static constexpr int NIN = TX * TY;                   // interior columns (threads 0..NIN-1)
  static_assert(NIN % 32 == 0, "interior columns fill whole warps");
  static_assert((RAW_BYTES + Q_BYTES) % 16 == 0, "flux buffers start 16-byte aligned");
  static_assert(NEXTRA <= NT - NIN, "the outer ring is converted by the threads after the interior");
  static_assert(TX % 2 == 0 && TY % 2 == 0, "even tile");
};

__device__ __forceinline__ int pmod(int a, int m) { return ((a % m) + m) % m; }

// One work item (TX x TY column, z range) of one problem. RS (Riemann solver)
// and ST (slope type) fix the scheme at compile time; RS = 0 / ST = -1 read it
// from a.hp at run time.
template <typename R, int TX, int TY, int RS, int ST>
__device__ __forceinline__ void stream_step_body(const StreamArgs& a, const int item) {
  using G = StreamGeom<R, TX, TY>;
  constexpr int SX = G::SX, SY = G::SY, CX = G::CX, NS = G::NS, NC = G::NC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* raw = reinterpret_cast<double*>(smem_raw);                      // [NRAW][5][NS]
  R* qb = reinterpret_cast<R*>(smem_raw + G::RAW_BYTES);                  // [NQ][5][NS]
  double* fxs = reinterpret_cast<double*>(qb + G::NQ * 5 * NS);           // [5][NC] Fx (left face)
  double* fys = fxs + 5 * NC;                                             // [5][NC] Fy (lower face)
  R* xm = reinterpret_cast<R*>(fys + 5 * NC);                             // [5][NC] qm_x
  R* ym = xm + 5 * NC;                                                    // [5][NC] qm_y
  __shared__ double red[G::NT / 32];

  // Thread -> column map. Threads 0..NIN-1 own the interior columns (they
  // solve x, y and z faces and update). The trace ring follows in the order
  // right column, top row (the ring columns with an x or a y face to solve),
  // left column, bottom row, top corners (nothing to solve), so the solve and
  // update predicates are uniform over most warps. Shared arrays are indexed
  // by the column's slot (cx+1) + CX*(cy+1), independent of this map.
  const int tid = threadIdx.x;
  const bool valid = tid < NC;                       // padding threads own no column
  int cx = -1, cy = -1;
  if (valid) {
    if (tid < G::NIN) {
      cx = tid % TX; cy = tid / TX;
    } else {
      int r = tid - G::NIN;
      if (r < TY) { cx = TX; cy = r; }
      else if ((r -= TY) < TX) { cx = r; cy = TY; }
      else if ((r -= TX) < TY) { cx = -1; cy = r; }
      else if ((r -= TY) < TX + 2) { cx = r - 1; cy = -1; }
      else { r -= TX + 2; cx = r ? TX : -1; cy = TY; }
    }
  }
  const int slot = valid ? (cx + 1) + CX * (cy + 1) : 0;
  const bool inner = valid && tid < G::NIN;
  const int nxt = a.nx / TX, nyt = a.ny / TY;
  const int tx0 = (item % nxt) * TX, ty0 = ((item / nxt) % nyt) * TY, z0 = (item / (nxt * nyt)) * a.hz;
  const int zend = z0 + a.hz;                        // planes [z0, zend) are updated
  const int64_t plane = (int64_t)a.nx * a.ny;
  const int64_t vstr = plane * a.nz;
  const Consts<R> c = make_consts<R>(a.hp);
  const double dt = *a.dt_dev;
  const int slope_type = ST >= 0 ? ST % 10 : a.hp.slope_type;
  const R dtdx = (R)(dt / a.dx);
  const R dtd[3] = {dtdx, dtdx, dtdx};

  // extra (q-only) column of this thread, if any: the outer stencil ring
  int ex = 0, ey = 0;
  const bool has_extra = tid >= G::NIN && tid - G::NIN < G::NEXTRA;
  if (has_extra) {
    int r = tid - G::NIN;
    if (r < SX) { ex = r; ey = 0; }
    else if ((r -= SX) < SX) { ex = r; ey = SY - 1; }
    else if ((r -= SX) < SY - 2) { ex = 0; ey = 1 + r; }
    else { r -= SY - 2; ex = SX - 1; ey = 1 + r; }
  }
  const int s_own = valid ? (cx + 2) + SX * (cy + 2) : 0;
  const int s_ext = ex + SX * ey;

  // every plane index used below is >= z0-2, so ring slots come from a
  // non-negative offset and constant moduli; periodic wraps need one step
  const int zbase = z0 - 2;
  // cell index along axis d outside [0, n): periodic wrap (one step is
  // enough, every index is within 2 cells of the box), or with outflow
  // boundaries the nearest interior cell, the zero-gradient ghost value that
  // make_boundary_hydro gives (hydro/hydro_boundary.f90:80-85)
  auto bnd = [&](int v, int n, int d) {
    if (a.outflow & (1 << d)) return v < 0 ? 0 : (v >= n ? n - 1 : v);
    return v < 0 ? v + n : (v >= n ? v - n : v);
  };
  // Plane loads: thread tid < PAIRS owns the 2-cell (16-byte) piece (row, j)
  // of the stencil plane for all 5 variables; its offsets inside a plane do
  // not change along z, so they are computed once here.
  // A piece starts at an even x and so lies wholly inside or wholly outside
  // the box; with outflow in x an outside piece is two copies of the edge cell.
  const bool loader = tid < G::PAIRS;
  int piece_s = 0;
  int64_t piece_g = 0;
  bool piece_dup = false;
  if (loader) {
    const int j = tid % (SX / 2), row = tid / (SX / 2);
    const int x0 = tx0 - 2 + 2 * j;
    piece_s = row * SX + 2 * j;
    piece_dup = (a.outflow & 1) && (x0 < 0 || x0 >= a.nx);
    piece_g = (int64_t)bnd(ty0 - 2 + row, a.ny, 1) * a.nx + bnd(x0, a.nx, 0);
  }
  auto issue_plane = [&](int zp) {
    if (!loader) return;
    double* dst = raw + ((unsigned)(zp - zbase) % G::NRAW) * 5 * NS + piece_s;
    const double* src = a.uin + (int64_t)bnd(zp, a.nz, 2) * plane + piece_g;
    if (piece_dup) {
#pragma unroll
      for (int v = 0; v < 5; v++) {
        cp_async8(dst + v * NS, src + v * vstr);
        cp_async8(dst + v * NS + 1, src + v * vstr);
      }
    } else {
#pragma unroll
      for (int v = 0; v < 5; v++) cp_async16(dst + v * NS, src + v * vstr);
    }
  };
  auto load_u = [&](int zp, int s, double u[5]) {
    const double* p = raw + ((unsigned)(zp - zbase) % G::NRAW) * 5 * NS + s;
#pragma unroll
    for (int v = 0; v < 5; v++) u[v] = p[v * NS];
  };
  auto to_q = [&](int zp, int s) {
    double u[5];
    load_u(zp, s, u);
    return ctoprim_cell<R>(u, a.hp);
  };
  auto put_q = [&](int zp, int s, const Prim<R>& q) {
    R* p = qb + ((unsigned)(zp - zbase) % G::NQ) * 5 * NS + s;
    p[0] = q.r; p[NS] = q.u; p[2 * NS] = q.v; p[3 * NS] = q.w; p[4 * NS] = q.p;
  };

  // ---- prologue: planes z0-2 .. z0+2 in flight; q(z0-2..z0) converted ----
  for (int zp = z0 - 2; zp <= z0 + 2; zp++) { issue_plane(zp); cp_async_commit(); }
  cp_async_wait<1>();
  __syncthreads();
  Prim<R> q_m1 = to_q(z0 - 2, s_own);
  Prim<R> q_0 = to_q(z0 - 1, s_own);
  Prim<R> q_p1 = to_q(z0, s_own);
  Prim<R> q_p2 = q_p1;
  if (valid) { put_q(z0 - 1, s_own, q_0); put_q(z0, s_own, q_p1); }
  if (has_extra) { put_q(z0 - 1, s_ext, to_q(z0 - 1, s_ext)); put_q(z0, s_ext, to_q(z0, s_ext)); }
  cp_async_wait<0>();
  __syncthreads();

  Prim<R> qmz_prev;                  // qm_z of the plane below (left state of face k-1/2)
  qmz_prev.r = qmz_prev.u = qmz_prev.v = qmz_prev.w = qmz_prev.p = (R)0;
  double upd[5] = {0, 0, 0, 0, 0};   // uold + dFx + dFy of the pending plane
  double fzb[5] = {0, 0, 0, 0, 0};   // flux through the pending plane's lower face
  double smax = 0.0;
  const int64_t col = inner ? (int64_t)(ty0 + cy) * a.nx + (tx0 + cx) : 0;

  for (int k = z0 - 1; k <= zend; k++) {
    const bool upd_plane = (k >= z0) && (k < zend);  // x/y fluxes and partial update at k
    // B. slopes and trace of plane k
    const R* qk = qb + ((unsigned)(k - zbase) % G::NQ) * 5 * NS;
    R dq[5][3];
    {
      const R own[5] = {q_0.r, q_0.u, q_0.v, q_0.w, q_0.p};
      const R zm[5] = {q_m1.r, q_m1.u, q_m1.v, q_m1.w, q_m1.p};
      const R zp[5] = {q_p1.r, q_p1.u, q_p1.v, q_p1.w, q_p1.p};
      const int sxm = valid ? s_own - 1 : 0, sxp = valid ? s_own + 1 : 0;
      const int sym = valid ? s_own - SX : 0, syp = valid ? s_own + SX : 0;
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const R* qv = qk + v * NS;
        dq[v][0] = slope1<R>(qv[sxm], own[v], qv[sxp], slope_type, c.slope_theta);
        dq[v][1] = slope1<R>(qv[sym], own[v], qv[syp], slope_type, c.slope_theta);
        dq[v][2] = slope1<R>(zm[v], own[v], zp[v], slope_type, c.slope_theta);
      }
    }
    // the ring columns (whole warps after the interior ones) solve no z face
    Prim<R> sp[3], sm[3];
    trace_sel<R, RS, ST>(q_0, dq, c, dtd, sp, sm, inner ? 7u : 3u);
    if (valid) {
      const int o = slot;
      xm[o] = sm[0].r; xm[NC + o] = sm[0].u; xm[2 * NC + o] = sm[0].v; xm[3 * NC + o] = sm[0].w; xm[4 * NC + o] = sm[0].p;
      ym[o] = sm[1].r; ym[NC + o] = sm[1].u; ym[2 * NC + o] = sm[1].v; ym[3 * NC + o] = sm[1].w; ym[4 * NC + o] = sm[1].p;
    }
    __syncthreads();
    if (k + 4 <= zend + 1) issue_plane(k + 4);
    cp_async_commit();
    // A. ctoprim of plane k+2, into the primitive slot of plane k, which
    // every thread has finished reading at the barrier above; plane k+2 landed
    // at the previous iteration's wait
    if (k + 2 <= zend + 1) {
      q_p2 = to_q(k + 2, s_own);
      if (valid) put_q(k + 2, s_own, q_p2);
      if (has_extra) put_q(k + 2, s_ext, to_q(k + 2, s_ext));
    }
    // C. Riemann problems
    R fx[5] = {0, 0, 0, 0, 0}, fy[5] = {0, 0, 0, 0, 0}, fz[5] = {0, 0, 0, 0, 0};
    const bool xface = upd_plane && valid && cx >= 0 && cy >= 0 && cy < TY;
    const bool yface = upd_plane && valid && cy >= 0 && cx >= 0 && cx < TX;
    if (xface) {
      const int o = slot - 1;  // column (cx-1, cy)
      Prim<R> L;
      L.r = xm[o]; L.u = xm[NC + o]; L.v = xm[2 * NC + o]; L.w = xm[3 * NC + o]; L.p = xm[4 * NC + o];
      R ql[5], qr[5], fg[6];
      to_face(L, 0, ql);
      to_face(sp[0], 0, qr);
      riemann_sel<R, RS>(ql, qr, c, fg);
      from_face(fg, 0, fx);
    }
    if (yface) {
      const int o = slot - CX;  // column (cx, cy-1)
      Prim<R> L;
      L.r = ym[o]; L.u = ym[NC + o]; L.v = ym[2 * NC + o]; L.w = ym[3 * NC + o]; L.p = ym[4 * NC + o];
      R ql[5], qr[5], fg[6];
      to_face(L, 1, ql);
      to_face(sp[1], 1, qr);
      riemann_sel<R, RS>(ql, qr, c, fg);
      from_face(fg, 1, fy);
    }
    if (inner && k >= z0) {
      R ql[5], qr[5], fg[6];
      to_face(qmz_prev, 2, ql);
      to_face(sp[2], 2, qr);
      riemann_sel<R, RS>(ql, qr, c, fg);
      from_face(fg, 2, fz);
    }
    if (inner) qmz_prev = sm[2];
    // flux*dt/dx evaluated as (fx*dt)/dx (umuscl.f90:101-163); dividing by an
    // exact power-of-two dx equals multiplying by its reciprocal
    // Each face flux is rounded to FP64 once, by the face's owner, so that the
    // FP64 accumulation below telescopes exactly (conservation to FP64
    // roundoff in both precisions).
    auto scale = [&](R f) -> R {
      if (sizeof(R) == 8) {
        const double t = (double)f * dt;
        return (R)(a.dx_pow2 ? t * a.inv_dx : t / a.dx);
      }
      return f * dtdx;
    };
    double fzd[5];
    if (upd_plane && valid) {
#pragma unroll
      for (int v = 0; v < 5; v++) {
        fxs[v * NC + slot] = (double)scale(fx[v]);
        fys[v * NC + slot] = (double)scale(fy[v]);
      }
    }
    if (inner && k >= z0) {
#pragma unroll
      for (int v = 0; v < 5; v++) fzd[v] = (double)scale(fz[v]);
    }
    cp_async_wait<1>();  // plane k+3 (converted at the next A) has landed
    __syncthreads();
    // D. finish plane k-1, partial update of plane k
    if (inner) {
      if (k - 1 >= z0) {
        double un[5];
        const int64_t zo = (int64_t)(k - 1) * plane;  // k-1 in [z0, zend) lies inside the box
#pragma unroll
        for (int v = 0; v < 5; v++) {
          un[v] = upd[v] + (fzb[v] - fzd[v]);
          a.uout[v * vstr + zo + col] = un[v];
        }
        if constexpr (sizeof(R) == 8) smax = fmx(smax, cfl_speed(un, a.hp));
        else smax = fmax(smax, cfl_speed_fast(un, a.hp));
      }
      if (upd_plane) {
        double uo[5];
        load_u(k, s_own, uo);
#pragma unroll
        for (int v = 0; v < 5; v++) {
          double u = uo[v];
          u = u + (fxs[v * NC + slot] - fxs[v * NC + slot + 1]);
          u = u + (fys[v * NC + slot] - fys[v * NC + slot + CX]);
          upd[v] = u;
          fzb[v] = fzd[v];
        }
      }
    }
    q_m1 = q_0;
    q_0 = q_p1;
    q_p1 = q_p2;
  }
  cp_async_wait<0>();

  // ---- CFL partial of this work item (max wave speed -> min dt) ----
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) smax = fmx(smax, __shfl_xor_sync(0xffffffffu, smax, o));
  if ((tid & 31) == 0) red[tid >> 5] = smax;
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < G::NT / 32; w++) smax = fmx(smax, red[w]);
    a.partial[(int64_t)item * 4 + 0] = smax > 0.0 ? cfl_dt_from_speed(smax, a.dx, a.hp.courant_factor) : 1.0e300;
    a.partial[(int64_t)item * 4 + 1] = 0.0;
    a.partial[(int64_t)item * 4 + 2] = 0.0;
    a.partial[(int64_t)item * 4 + 3] = 0.0;
  }
}

// One step of one problem: one CTA per work item.
// MINB: CTAs per SM the register allocation must allow (the register budget
// knob of the autotuner).
template <typename R, int TX, int TY, int MINB, int RS, int ST>
__global__ void __launch_bounds__(StreamGeom<R, TX, TY>::NT, MINB) stream_step_kernel(StreamArgs a) {
  stream_step_body<R, TX, TY, RS, ST>(a, blockIdx.x);
}

// Problem descriptor of the batched (serving) step. The problem's device
// clock holds (dt, t, -, -, -, steps, done, -): the kernel reads dt from it,
// picks the current buffer from the step parity and skips finished problems.
struct BatchDesc {
  StreamArgs a;          // geometry, partial slice and parameters of the problem
  double* dense[2];      // the two state buffers
  double* clock;         // [8]
  double t_end;          // stop rule: t >= t_end or steps >= max_steps
  double max_steps;
  double dt_max, dt0;    // boxlen/smallc and courant_factor*dx/smallc
  int32_t parity0;       // buffer holding the state when the clock read 0 steps
  int32_t nitems;
};

// One round of the serving engine: the work items of every active problem in
// one launch. item_off[p] .. item_off[p+1]-1 are problem p's items.
template <typename R, int TX, int TY, int MINB, int RS, int ST>
__global__ void __launch_bounds__(StreamGeom<R, TX, TY>::NT, MINB)
    stream_batch_kernel(const BatchDesc* __restrict__ desc, const int32_t* __restrict__ item_off, int nprob) {
  const int b = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {  // last p with item_off[p] <= b
    const int mid = (lo + hi + 1) >> 1;
    if (item_off[mid] <= b) lo = mid; else hi = mid - 1;
  }
  const BatchDesc& d = desc[lo];
  if (d.clock[6] != 0.0) return;  // finished: the state stays where it is
  StreamArgs a = d.a;
  const int cur = (d.parity0 + (int)d.clock[5]) & 1;
  a.uin = d.dense[cur];
  a.uout = d.dense[cur ^ 1];
  a.dt_dev = d.clock;
  stream_step_body<R, TX, TY, RS, ST>(a, b - item_off[lo]);
}

}  // namespace rb
