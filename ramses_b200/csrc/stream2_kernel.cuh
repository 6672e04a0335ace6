// stream2_kernel.cuh -- the FP32-mixed z-streaming step of a complete level
// (godunov_fine + set_uold + courant_fine on the dense [v][z][y][x] mirror),
// laid out for B200 issue throughput.
//
// Same stencil and the same arithmetic as stream_kernel.cuh in FP32-mixed
// (slopes, trace and HLLC in FP32; ctoprim's floors, E - rho v^2/2, the
// conservative accumulation and the CFL reduction in FP64), organised so that
// every warp of a CTA carries about the same work between the two barriers of
// a plane:
//   * threads 0..NIN-1 own the TX x TY interior columns: own ctoprim, slopes
//     and trace of x, y, z, the x face to their left, the z face below, and
//     the FP64 update;
//   * the ring group (threads NIN..NT-1) traces the 2(TX+TY) ring columns
//     (x and y only; the 4 corners need no trace), converts the 64 q-only
//     columns of the stencil plane, and solves the y faces and the x faces of
//     the right ring column, several rounds per plane.
// Shared memory is packed for 128-bit accesses: primitive planes as
// (rho,u,v,w) float4 + p, face states as five float4 per column, fluxes
// (already times dt/dx) as FP32, widened exactly to FP64 by both cells that
// share the face so that the FP64 accumulation telescopes. A 4-plane raw ring
// (cp.async, one plane of prefetch distance) keeps the CTA at ~70 KB, three
// CTAs per SM.
//
// HLLC with minmod (ST = 1) or moncen (ST = 2) slopes, MUSCL-Hancock
// predictor; other schemes and the FP64 drop-in use stream_kernel.cuh.
// References: ctoprim umuscl.f90:861-965, uslope :1241-1327, trace3d
// :483-708, cmpflxm :714-856, riemann_hllc godunov_utils.f90:988-1209,
// update godunov_fine.f90:751-792, cmpdt godunov_utils.f90:5-120.
#pragma once
#include <cstdint>

#include "cp_async.cuh"
#include "hydro_core.cuh"
#include "stream_kernel.cuh"

namespace rb {

template <int TX, int TY>
struct S2Geom {
  static constexpr int SX = TX + 4, SY = TY + 4, NS = SX * SY;   // stencil plane
  static constexpr int SXP = SX + 1;                              // padded row of the q planes
  static constexpr int NQS = SXP * SY;                            // q-plane slots
  static constexpr int CX = TX + 2, CY = TY + 2, NC = CX * CY;   // trace columns
  static constexpr int NIN = TX * TY;
  static constexpr int NRING = 2 * (TX + TY);
  static constexpr int NTRACE = NIN + NRING;
  static constexpr int NEXTRA = NS - NTRACE;                      // q-only columns
  static constexpr int NRG0 = NRING > NEXTRA ? NRING : NEXTRA;
  static constexpr int NT = NIN + (NRG0 + 31) / 32 * 32;
  static constexpr int NRG = NT - NIN;                            // ring-group threads
  static constexpr int NRAW = 4;                                  // raw planes in the ring
  static constexpr int PAIRS = SY * (SX / 2);                     // 16-byte pieces of a variable's plane
  static constexpr int NRF = TX * (TY + 1) + TY;                  // faces of the ring group
  static constexpr int ROUNDS = (NRF + NRG - 1) / NRG;
  static constexpr size_t RAW_BYTES = sizeof(double) * NRAW * 5 * NS;
  static constexpr size_t Q4_BYTES = 16 * 2 * NQS;
  static constexpr size_t QP_BYTES = 4 * 2 * NQS;
  static constexpr size_t FS_BYTES = 80 * NC;                     // 5 float4 per trace column
  static constexpr size_t FL_BYTES = 20 * NC;                     // one face flux (float4 + float) per column
  static constexpr size_t SMEM = RAW_BYTES + Q4_BYTES + QP_BYTES + FS_BYTES + 2 * FL_BYTES;
  static_assert(NIN % 32 == 0, "interior columns fill whole warps");
  static_assert(PAIRS <= NT, "one plane piece per thread");
  static_assert(NEXTRA <= NRG, "one q-only column per ring-group thread");
  static_assert(TX % 2 == 0 && TY % 2 == 0, "even tile");
  static_assert(RAW_BYTES % 16 == 0 && Q4_BYTES % 16 == 0 && QP_BYTES % 16 == 0, "16-byte aligned sections");
};

// Half slope dq/2 of one variable in one direction (uslope, umuscl.f90:1241-1327):
// ST = 1 minmod, ST = 2 moncen, in FP32 with the sign applied last.
template <int ST>
__device__ __forceinline__ float hslope(float qm1, float q0, float qp1) {
  const float a = q0 - qm1, b = qp1 - q0;
  const float m = fminf(fabsf(a), fabsf(b));
  float s;
  if (ST == 1) {
    s = copysignf(0.5f * m, a);
  } else {
    const float t = a + b;
    s = copysignf(fminf(m, 0.25f * fabsf(t)), t);
  }
  return a * b <= 0.0f ? 0.0f : s;
}

// Half slope from the two one-sided differences a = q0 - q(-1), b = q(+1) - q0.
template <int ST>
__device__ __forceinline__ float hslope_ab(float a, float b) {
  const float m = fminf(fabsf(a), fabsf(b));
  float s;
  if (ST == 1) {
    s = copysignf(0.5f * m, a);
  } else {
    const float t = a + b;
    s = copysignf(fminf(m, 0.25f * fabsf(t)), t);
  }
  return a * b <= 0.0f ? 0.0f : s;
}

// ctoprim (umuscl.f90:861-965) for the FP32-mixed kernels. The density
// floor, the internal energy E - |m|^2/(2 rho) and the pressure floor are
// FP64; the reciprocal of rho is the FP32 one refined by one Newton step in
// FP64, and the velocities are FP32. With
// P = (gamma-1) rho max(E/rho - v^2/2, smalle) and
// smalle = smallc^2/gamma/(gamma-1): P = max((gamma-1)(E - |m|^2/(2 rho)), rho smallc^2/gamma).
__device__ __forceinline__ Prim<float> ctoprim_mixed(const double u[5], double smallr, double gm1, double pfc) {
  const double rho = fmax(u[0], smallr);
  const float rf = (float)rho;
  const float irf = __fdividef(1.0f, rf);
  const double ir = fma((double)irf, fma(-rho, (double)irf, 1.0), (double)irf);
  const double ke = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
  const double p = fmax(gm1 * fma(-0.5 * ke, ir, u[4]), pfc * rho);
  Prim<float> q;
  q.r = rf;
  q.u = (float)u[1] * irf;
  q.v = (float)u[2] * irf;
  q.w = (float)u[3] * irf;
  q.p = (float)p;
  return q;
}

// HLLC flux (riemann_hllc, godunov_utils.f90:988-1209) in FP32 for the mixed
// path, times dt/dx. Face frame (rho, u_n, P, u_t1, u_t2) in, flux of (mass,
// normal momentum, energy, t1 momentum, t2 momentum) out. The larger of the
// two fast sound speeds is formed with one reciprocal and one square root,
// and the sampled state's side is chosen before its energy is formed.
__device__ __forceinline__ void hllc_f32(const float ql[5], const float qr[5], const Consts<float>& c,
                                         float smallc2, float dtdx, float f[5]) {
  const float rl = fmaxf(ql[0], c.smallr), ul = ql[1], Pl = fmaxf(ql[2], rl * c.smallp);
  const float rr = fmaxf(qr[0], c.smallr), ur = qr[1], Pr = fmaxf(qr[2], rr * c.smallp);
  // max(gamma Pl/rl, gamma Pr/rr, smallc^2), rl, rr > 0
  const float a2 = fmaxf(fmaxf(Pl * rr, Pr * rl) * (c.gamma * __fdividef(1.0f, rl * rr)), smallc2);
  const float cmax = sqrtf(a2);
  const float SL = fminf(ul, ur) - cmax, SR = fmaxf(ul, ur) + cmax;
  const float rcl = rl * (ul - SL), rcr = rr * (SR - ur);
  const float inv = __fdividef(1.0f, rcr + rcl);
  const float ustar = (rcr * ur + rcl * ul + (Pl - Pr)) * inv;
  const float Pstar = (rcr * Pl + rcl * Pr + rcl * rcr * (ul - ur)) * inv;
  // sampling at x/t = 0: outer left if SL > 0, left star if ustar > 0, right
  // star if SR > 0, else outer right
  const bool outl = SL > 0.0f, lft = ustar > 0.0f;
  const bool side = outl || lft;
  const bool star = !outl && (lft || SR > 0.0f);
  const float rs = side ? rl : rr, us = side ? ul : ur, Ss = side ? SL : SR, Ps = side ? Pl : Pr;
  const float t1 = side ? ql[3] : qr[3], t2 = side ? ql[4] : qr[4];
  const float num = Ss - us, iden = __fdividef(1.0f, Ss - ustar);
  const float ratio = star ? num * iden : 1.0f;
  const float ro = rs * ratio;
  const float uo = star ? ustar : us;
  const float Po = star ? Pstar : Ps;
  const float ets = Ps * c.entho + 0.5f * rs * (us * us + t1 * t1 + t2 * t2);
  const float eto = star ? (num * ets - Ps * us + Pstar * ustar) * iden : ets;
  const float uos = uo * dtdx;
  const float mo = ro * uos;
  f[0] = mo;
  f[1] = mo * uo + Po * dtdx;
  f[2] = (eto + Po) * uos;
  f[3] = mo * t1;
  f[4] = mo * t2;
}

// MUSCL-Hancock half-step state of a cell for the FP32 path: h = q + s dt/(2dx)
// with the source terms of trace3d (umuscl.f90:576-580), equal in every
// direction on a cubic cell. hd[v][d] are half slopes; th = dt/dx (the factor
// 1/2 of the half step cancels the 2 of the full slope).
__device__ __forceinline__ void half_step(const Prim<float>& q, const float hd[5][3], float gamma, float th,
                                          float h[5]) {
  const float r = q.r, u = q.u, v = q.v, w = q.w, p = q.p;
  const float divv = hd[1][0] + hd[2][1] + hd[3][2];
  const float ir = __fdividef(1.0f, r);
  h[0] = r - th * (u * hd[0][0] + v * hd[0][1] + w * hd[0][2] + divv * r);
  h[4] = p - th * (u * hd[4][0] + v * hd[4][1] + w * hd[4][2] + divv * (gamma * p));
  h[1] = u - th * (u * hd[1][0] + v * hd[1][1] + w * hd[1][2] + hd[4][0] * ir);
  h[2] = v - th * (u * hd[2][0] + v * hd[2][1] + w * hd[2][2] + hd[4][1] * ir);
  h[3] = w - th * (u * hd[3][0] + v * hd[3][1] + w * hd[3][2] + hd[4][2] * ir);
}

// face states of direction d: right state at the lower face P = h - hd,
// left state at the upper face M = h + hd, density floored to the cell's
// (trace3d: if (q < smallr) q = r)
__device__ __forceinline__ void face_pair(const float h[5], const float hd[5][3], int d, float r, float smallr,
                                          float P[5], float M[5]) {
#pragma unroll
  for (int v = 0; v < 5; v++) { P[v] = h[v] - hd[v][d]; M[v] = h[v] + hd[v][d]; }
  if (P[0] < smallr) P[0] = r;
  if (M[0] < smallr) M[0] = r;
}

// (rho, u, v, w, p) -> face frame of direction d (cmpflxm's permutation)
__device__ __forceinline__ void face_frame(const float s[5], int d, float o[5]) {
  o[0] = s[0];
  o[2] = s[4];
  if (d == 0) { o[1] = s[1]; o[3] = s[2]; o[4] = s[3]; }
  else if (d == 1) { o[1] = s[2]; o[3] = s[1]; o[4] = s[3]; }
  else { o[1] = s[3]; o[3] = s[1]; o[4] = s[2]; }
}
// face-frame flux -> (rho, mx, my, mz, E)
__device__ __forceinline__ void flux_back(const float f[5], int d, float o[5]) {
  o[0] = f[0];
  o[4] = f[2];
  if (d == 0) { o[1] = f[1]; o[2] = f[3]; o[3] = f[4]; }
  else if (d == 1) { o[2] = f[1]; o[1] = f[3]; o[3] = f[4]; }
  else { o[3] = f[1]; o[1] = f[3]; o[2] = f[4]; }
}

// One work item (TX x TY column, z range [z0, z0+hz)) of one problem.
template <int TX, int TY, int ST>
__device__ __forceinline__ void stream2_step_body(const StreamArgs& a, const int item) {
  using G = S2Geom<TX, TY>;
  constexpr int SX = G::SX, SY = G::SY, NS = G::NS, SXP = G::SXP, NQS = G::NQS, CX = G::CX, NIN = G::NIN;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* raw = reinterpret_cast<double*>(smem_raw);                                   // [NRAW][5][NS]
  float4* q4 = reinterpret_cast<float4*>(smem_raw + G::RAW_BYTES);                     // [2][NQS]
  float* qpl = reinterpret_cast<float*>(smem_raw + G::RAW_BYTES + G::Q4_BYTES);        // [2][NQS]
  // face states [5][NC]: qm_x, qp_x, qm_y, qp_y as (rho,u,v,w), then their four p
  float4* fs = reinterpret_cast<float4*>(smem_raw + G::RAW_BYTES + G::Q4_BYTES + G::QP_BYTES);
  // face fluxes times dt/dx: x face left of / y face below a column, (f0..f3) + f4
  float4* fx4 = fs + 5 * G::NC;
  float4* fy4 = fx4 + G::NC;
  float* fx1 = reinterpret_cast<float*>(fy4 + G::NC);
  float* fy1 = fx1 + G::NC;
  __shared__ double red[G::NT / 32];

  const int tid = threadIdx.x;
  // ---- roles ----
  const bool inner = tid < NIN;
  const bool ringt = tid >= NIN && tid < G::NTRACE;
  const bool tracer = tid < G::NTRACE;
  int cx = 0, cy = 0;
  if (inner) {
    cx = tid % TX; cy = tid / TX;
  } else if (ringt) {
    int r = tid - NIN;
    if (r < TY) { cx = TX; cy = r; }
    else if ((r -= TY) < TX) { cx = r; cy = TY; }
    else if ((r -= TX) < TY) { cx = -1; cy = r; }
    else { cx = r - TY; cy = -1; }
  }
  const int slot = (cx + 1) + CX * (cy + 1);          // trace-column slot (face states, fluxes)
  const int s_own = (cx + 2) + SX * (cy + 2);         // raw plane index
  const int sq_own = (cx + 2) + SXP * (cy + 2);       // q plane index
  // q-only column of a ring-group thread: the outer stencil ring, then the
  // four corners of the trace region
  const int e = tid - NIN;
  const bool has_extra = e >= 0 && e < G::NEXTRA;
  int ex = 0, ey = 0;
  if (has_extra) {
    int r = e;
    if (r < SX) { ex = r; ey = 0; }
    else if ((r -= SX) < SX) { ex = r; ey = SY - 1; }
    else if ((r -= SX) < SY - 2) { ex = 0; ey = 1 + r; }
    else if ((r -= SY - 2) < SY - 2) { ex = SX - 1; ey = 1 + r; }
    else { r -= SY - 2; ex = (r & 1) ? SX - 2 : 1; ey = (r & 2) ? SY - 2 : 1; }
  }
  const int s_ext = ex + SX * ey, sq_ext = ex + SXP * ey;

  const int nxt = a.nx / TX, nyt = a.ny / TY;
  const int tx0 = (item % nxt) * TX, ty0 = ((item / nxt) % nyt) * TY, z0 = (item / (nxt * nyt)) * a.hz;
  const int zend = z0 + a.hz;
  const int64_t plane = (int64_t)a.nx * a.ny;
  const int64_t vstr = plane * a.nz;
  const Consts<float> c = make_consts<float>(a.hp);
  const float smallc2 = c.smallc * c.smallc;
  const double dt = *a.dt_dev;
  const float dtdx = (float)(dt / a.dx);
  const float th = dtdx;                   // half step times 2: the slopes are halves

  auto bnd = [&](int v, int n, int d) {
    if (a.outflow & (1 << d)) return v < 0 ? 0 : (v >= n ? n - 1 : v);
    return v < 0 ? v + n : (v >= n ? v - n : v);
  };
  // plane loads: one 16-byte piece (2 cells) of the stencil plane per thread
  // for all 5 variables; offsets fixed along z
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
  const int zbase = z0 - 2;
  auto rawp = [&](int zp) { return raw + ((zp - zbase) & (G::NRAW - 1)) * (5 * NS); };
  auto issue_plane = [&](int zp) {
    if (!loader) return;
    double* dst = rawp(zp) + piece_s;
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
  const double gm1 = a.hp.gamma - 1.0, pfc = a.hp.smallc * a.hp.smallc / a.hp.gamma;
  auto to_q = [&](const double* rp, int s) {
    double u[5];
#pragma unroll
    for (int v = 0; v < 5; v++) u[v] = rp[v * NS + s];
    return ctoprim_mixed(u, a.hp.smallr, gm1, pfc);
  };
  auto put_q = [&](int zp, int sq, const Prim<float>& q) {
    const int o = ((zp - zbase) & 1) * NQS + sq;
    q4[o] = make_float4(q.r, q.u, q.v, q.w);
    qpl[o] = q.p;
  };

  // ---- prologue: raw planes z0-2 .. z0+1; q(z0-2 .. z0) ----
  for (int zp = z0 - 2; zp <= z0 + 1; zp++) { issue_plane(zp); cp_async_commit(); }
  cp_async_wait<1>();
  __syncthreads();
  Prim<float> q_m1, q_0, q_p1, q_p2;
  q_m1.r = q_m1.u = q_m1.v = q_m1.w = q_m1.p = 0.0f;
  q_0 = q_p1 = q_p2 = q_m1;
  if (tracer) {
    q_m1 = to_q(rawp(z0 - 2), s_own);
    q_0 = to_q(rawp(z0 - 1), s_own);
    q_p1 = to_q(rawp(z0), s_own);
    put_q(z0 - 1, sq_own, q_0);
    put_q(z0, sq_own, q_p1);
  }
  if (has_extra) {
    put_q(z0 - 1, sq_ext, to_q(rawp(z0 - 1), s_ext));
    put_q(z0, sq_ext, to_q(rawp(z0), s_ext));
  }
  __syncthreads();                         // q planes z0-1, z0 visible
  float qmz[5] = {0, 0, 0, 0, 0};          // left state of the face below the plane being traced
  // q(z0-1) - q(z0-2): the lower z difference of the first traced plane
  float dzl[5] = {q_0.r - q_m1.r, q_0.u - q_m1.u, q_0.v - q_m1.v, q_0.w - q_m1.w, q_0.p - q_m1.p};
  double pend[5] = {0, 0, 0, 0, 0};        // uold + dFx + dFy + Fz(lower) of the pending plane
  double smax = 0.0;
  const int64_t col = inner ? (int64_t)(ty0 + cy) * a.nx + (tx0 + cx) : 0;

  for (int k = z0 - 1; k <= zend; k++) {
    const bool upd_plane = (k >= z0) && (k < zend);
    // ---- P1: slopes and trace of plane k ----
    float zP[5], zM[5];                   // z face states of the own column (inner)
    if (tracer) {
      const int qo = ((k - zbase) & 1) * NQS + sq_own;
      const float4 xm = q4[qo - 1], xp = q4[qo + 1], ym = q4[qo - SXP], yp = q4[qo + SXP];
      const float pxm = qpl[qo - 1], pxp = qpl[qo + 1], pym = qpl[qo - SXP], pyp = qpl[qo + SXP];
      float hd[5][3];
      hd[0][0] = hslope<ST>(xm.x, q_0.r, xp.x); hd[0][1] = hslope<ST>(ym.x, q_0.r, yp.x);
      hd[1][0] = hslope<ST>(xm.y, q_0.u, xp.y); hd[1][1] = hslope<ST>(ym.y, q_0.u, yp.y);
      hd[2][0] = hslope<ST>(xm.z, q_0.v, xp.z); hd[2][1] = hslope<ST>(ym.z, q_0.v, yp.z);
      hd[3][0] = hslope<ST>(xm.w, q_0.w, xp.w); hd[3][1] = hslope<ST>(ym.w, q_0.w, yp.w);
      hd[4][0] = hslope<ST>(pxm, q_0.p, pxp);   hd[4][1] = hslope<ST>(pym, q_0.p, pyp);
      // z: the lower difference is the upper one of the plane below
      const float bz[5] = {q_p1.r - q_0.r, q_p1.u - q_0.u, q_p1.v - q_0.v, q_p1.w - q_0.w, q_p1.p - q_0.p};
#pragma unroll
      for (int v = 0; v < 5; v++) {
        hd[v][2] = hslope_ab<ST>(dzl[v], bz[v]);
        dzl[v] = bz[v];
      }
      float h[5];
      half_step(q_0, hd, c.gamma, th, h);
      float P[5], M[5];
      face_pair(h, hd, 0, q_0.r, c.smallr, P, M);
      fs[slot] = make_float4(M[0], M[1], M[2], M[3]);
      fs[G::NC + slot] = make_float4(P[0], P[1], P[2], P[3]);
      const float mxp = M[4], pxp_ = P[4];
      face_pair(h, hd, 1, q_0.r, c.smallr, P, M);
      fs[2 * G::NC + slot] = make_float4(M[0], M[1], M[2], M[3]);
      fs[3 * G::NC + slot] = make_float4(P[0], P[1], P[2], P[3]);
      fs[4 * G::NC + slot] = make_float4(mxp, pxp_, M[4], P[4]);
      if (inner) face_pair(h, hd, 2, q_0.r, c.smallr, zP, zM);
    }
    cp_async_wait<0>();                    // raw plane k+2 (own copies) has landed
    __syncthreads();                       // B1: face states and raw plane k+2 visible
    // ---- P2: prefetch, ctoprim of plane k+2, Riemann problems ----
    if (k + 3 <= zend + 1) issue_plane(k + 3);
    cp_async_commit();
    // interior columns convert their own column of plane k+2 here; the ring
    // group does its conversions after the second barrier, which balances
    // the two phases
    if (inner && k + 2 <= zend + 1) {
      q_p2 = to_q(rawp(k + 2), s_own);
      put_q(k + 2, sq_own, q_p2);
    }
    double fzd[5] = {0, 0, 0, 0, 0};
    if (inner) {
      if (upd_plane) {                     // x face left of the own column
        const float4 L4 = fs[slot - 1], R4 = fs[G::NC + slot];
        const float Lp = fs[4 * G::NC + slot - 1].x, Rp = fs[4 * G::NC + slot].y;
        const float L[5] = {L4.x, L4.y, L4.z, L4.w, Lp}, R[5] = {R4.x, R4.y, R4.z, R4.w, Rp};
        float ql[5], qr[5], ff[5], fo[5];
        face_frame(L, 0, ql);
        face_frame(R, 0, qr);
        hllc_f32(ql, qr, c, smallc2, dtdx, ff);
        flux_back(ff, 0, fo);
        fx4[slot] = make_float4(fo[0], fo[1], fo[2], fo[3]);
        fx1[slot] = fo[4];
      }
      if (k >= z0) {                       // z face below plane k
        float ql[5], qr[5], ff[5], fo[5];
        face_frame(qmz, 2, ql);
        face_frame(zP, 2, qr);
        hllc_f32(ql, qr, c, smallc2, dtdx, ff);
        flux_back(ff, 2, fo);
#pragma unroll
        for (int v = 0; v < 5; v++) fzd[v] = (double)fo[v];
      }
#pragma unroll
      for (int v = 0; v < 5; v++) qmz[v] = zM[v];
    } else if (upd_plane) {
      // ring group: y faces below (cx, cy), cx in [0,TX), cy in [0,TY], then
      // the x faces left of the right ring column
#pragma unroll
      for (int rd = 0; rd < G::ROUNDS; rd++) {
        const int fidx = rd * G::NRG + e;
        if (fidx < G::NRF) {
          const bool yf = fidx < TX * (TY + 1);
          const int fcx = yf ? fidx % TX : TX, fcy = yf ? fidx / TX : fidx - TX * (TY + 1);
          const int fsl = (fcx + 1) + CX * (fcy + 1);
          const int lsl = yf ? fsl - CX : fsl - 1;
          const float4 L4 = fs[(yf ? 2 : 0) * G::NC + lsl], R4 = fs[(yf ? 3 : 1) * G::NC + fsl];
          const float4 Lp4 = fs[4 * G::NC + lsl], Rp4 = fs[4 * G::NC + fsl];
          const float L[5] = {L4.x, L4.y, L4.z, L4.w, yf ? Lp4.z : Lp4.x};
          const float R[5] = {R4.x, R4.y, R4.z, R4.w, yf ? Rp4.w : Rp4.y};
          const int d = yf ? 1 : 0;
          float ql[5], qr[5], ff[5], fo[5];
          face_frame(L, d, ql);
          face_frame(R, d, qr);
          hllc_f32(ql, qr, c, smallc2, dtdx, ff);
          flux_back(ff, d, fo);
          (yf ? fy4 : fx4)[fsl] = make_float4(fo[0], fo[1], fo[2], fo[3]);
          (yf ? fy1 : fx1)[fsl] = fo[4];
        }
      }
    }
    __syncthreads();                       // B2: fluxes visible
    // ---- P3: ring-group conversions of plane k+2; update (interior columns) ----
    if (!inner && k + 2 <= zend + 1) {
      const double* rp = rawp(k + 2);
      if (tracer) {
        q_p2 = to_q(rp, s_own);
        put_q(k + 2, sq_own, q_p2);
      }
      if (has_extra) put_q(k + 2, sq_ext, to_q(rp, s_ext));
    }
    if (inner) {
      if (k - 1 >= z0) {
        double un[5];
        const int64_t zo = (int64_t)(k - 1) * plane;
#pragma unroll
        for (int v = 0; v < 5; v++) {
          un[v] = pend[v] - fzd[v];
          a.uout[v * vstr + zo + col] = un[v];
        }
        smax = fmax(smax, cfl_speed_fast(un, a.hp));
      }
      if (upd_plane) {
        const double* rp = rawp(k) + s_own;
        const float4 xl = fx4[slot], xr = fx4[slot + 1], yl = fy4[slot], yr = fy4[slot + CX];
        const float xl4 = fx1[slot], xr4 = fx1[slot + 1], yl4 = fy1[slot], yr4 = fy1[slot + CX];
        const float fxl[5] = {xl.x, xl.y, xl.z, xl.w, xl4}, fxr[5] = {xr.x, xr.y, xr.z, xr.w, xr4};
        const float fyl[5] = {yl.x, yl.y, yl.z, yl.w, yl4}, fyr[5] = {yr.x, yr.y, yr.z, yr.w, yr4};
#pragma unroll
        for (int v = 0; v < 5; v++) {
          double u = rp[v * NS];
          u = u + ((double)fxl[v] - (double)fxr[v]);
          u = u + ((double)fyl[v] - (double)fyr[v]);
          pend[v] = u + fzd[v];
        }
      }
    }
    q_0 = q_p1;
    q_p1 = q_p2;
  }
  cp_async_wait<0>();

  // ---- CFL partial of this work item (max wave speed -> min dt) ----
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
  if ((tid & 31) == 0) red[tid >> 5] = smax;
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < G::NT / 32; w++) smax = fmax(smax, red[w]);
    a.partial[(int64_t)item * 4 + 0] = smax > 0.0 ? cfl_dt_from_speed(smax, a.dx, a.hp.courant_factor) : 1.0e300;
    a.partial[(int64_t)item * 4 + 1] = 0.0;
    a.partial[(int64_t)item * 4 + 2] = 0.0;
    a.partial[(int64_t)item * 4 + 3] = 0.0;
  }
}

// One step of one problem: one CTA per work item. MINB: CTAs per SM the
// register allocation is bounded for.
template <int TX, int TY, int MINB, int ST>
__global__ void __launch_bounds__(S2Geom<TX, TY>::NT, MINB) stream2_step_kernel(StreamArgs a) {
  stream2_step_body<TX, TY, ST>(a, blockIdx.x);
}

// One round of the serving engine over the work items of every active
// problem (the BatchDesc protocol of stream_batch_kernel).
template <int TX, int TY, int MINB, int ST>
__global__ void __launch_bounds__(S2Geom<TX, TY>::NT, MINB)
    stream2_batch_kernel(const BatchDesc* __restrict__ desc, const int32_t* __restrict__ item_off, int nprob) {
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
  stream2_step_body<TX, TY, ST>(a, b - item_off[lo]);
}

}  // namespace rb

