// hydro_core.cuh -- per-cell and per-face arithmetic of RAMSES's unsplit
// MUSCL-Hancock scheme (NDIM=3, nvar=5), as device functions templated on
// the compute type R.
//
// R = double: the FP64 drop-in. Every expression keeps the operation order of
// the reference Fortran, and the translation units that instantiate it are
// compiled with --fmad=false so that no multiply-add is contracted; results
// are then bit-identical to the FP64 CPU restatement.
// R = float: the FP32-mixed path. Slopes, trace and Riemann fluxes run in
// FP32; conservative->primitive (density floor, E - 1/2 rho v^2, pressure
// floor) stays FP64 and is rounded to FP32 on output.
#pragma once
#include <cstdint>

#include "rb_types.h"

namespace rb {

// Fortran MAX/MIN with a fixed tie rule (first argument wins on equality),
// used identically by the CPU restatement so that signed zeros agree.
template <typename R> __device__ __forceinline__ R fmx(R a, R b) { return a > b ? a : (b > a ? b : a); }
template <typename R> __device__ __forceinline__ R fmn(R a, R b) { return a < b ? a : (b < a ? b : a); }
// The FP32-mixed path needs no signed-zero tie rule: one native min/max.
template <> __device__ __forceinline__ float fmx<float>(float a, float b) { return fmaxf(a, b); }
template <> __device__ __forceinline__ float fmn<float>(float a, float b) { return fminf(a, b); }

template <typename R> struct Prim { R r, u, v, w, p; };

// Hydro constants in compute precision.
template <typename R> struct Consts {
  R gamma, smallr, smallc, smallp, entho, half, slope_theta, courant;
  int slope_type, riemann, niter_riemann, scheme;
};

template <typename R>
__device__ __forceinline__ Consts<R> make_consts(const rb_hydro_params& hp) {
  Consts<R> c;
  c.gamma = (R)hp.gamma;
  c.smallr = (R)hp.smallr;
  c.smallc = (R)hp.smallc;
  // smallp = smallc**2/gamma ; entho = one/(gamma-one) (godunov_utils.f90:1019-1020)
  c.smallp = (R)(hp.smallc * hp.smallc / hp.gamma);
  c.entho = (R)(1.0 / (hp.gamma - 1.0));
  c.half = (R)0.5;
  c.slope_theta = (R)hp.slope_theta;
  c.courant = (R)hp.courant_factor;
  c.slope_type = hp.slope_type;
  c.riemann = hp.riemann;
  c.niter_riemann = hp.niter_riemann;
  c.scheme = hp.scheme;
  return c;
}

// ---------------------------------------------------------------------------
// ctoprim for one cell (umuscl.f90:861-965), conservative FP64 input.
// The sound speed of ctoprim is only used by the PLMDE trace, which forms it
// from the primitive state.
// ---------------------------------------------------------------------------
// FP64 reciprocal for the FP32-mixed path: the FP32 reciprocal of x refined
// by one Newton-Raphson step r <- r + r(1 - xr) in FP64, which squares the
// relative error (~1e-7 -> ~1e-14). Valid for x inside the normal FP32 range
// (1.2e-38 .. 3.4e38), which holds for densities floored at smallr.
__device__ __forceinline__ double rcp_newton(double x) {
  const double r = (double)(1.0f / (float)x);
  return fma(r, fma(-x, r, 1.0), r);
}

template <typename R>
__device__ __forceinline__ Prim<R> ctoprim_cell(const double u[5], const rb_hydro_params& hp) {
  const double gamma = hp.gamma;
  const double smalle = hp.smallc * hp.smallc / gamma / (gamma - 1.0);
  double q1 = fmx(u[0], hp.smallr);
  if constexpr (sizeof(R) == 4) {
    // FP32-mixed: velocities, E/rho - v^2/2 and its floor in FP64 from a
    // Newton-refined reciprocal; the zero gravity predictor is dropped (it
    // only changes the sign of a zero velocity)
    const double ir = rcp_newton(q1);
    const double q2 = u[1] * ir, q3 = u[2] * ir, q4 = u[3] * ir;
    const double eint = fmx(u[4] * ir - 0.5 * (q2 * q2 + q3 * q3 + q4 * q4), smalle);
    Prim<R> q;
    q.r = (R)q1; q.u = (R)q2; q.v = (R)q3; q.w = (R)q4; q.p = (R)((gamma - 1.0) * q1 * eint);
    return q;
  }
  // FP64 path: IEEE division as the reference
  double oneoverrho = 1.0 / q1;
  double q2 = u[1] * oneoverrho;
  double q3 = u[2] * oneoverrho;
  double q4 = u[3] * oneoverrho;
  double eken = 0.5 * q2 * q2;
  eken = eken + 0.5 * q3 * q3;
  eken = eken + 0.5 * q4 * q4;
  const double erad = 0.0;
  double eint = fmx(u[4] * oneoverrho - eken - erad, smalle);
  double q5 = (gamma - 1.0) * q1 * eint;
  // gravity predictor with the zero gravity field of a pure-hydro run:
  // q + 0*dt/2 == q + 0.0 (turns a negative zero positive, as the reference)
  q2 = __dadd_rn(q2, 0.0);
  q3 = __dadd_rn(q3, 0.0);
  q4 = __dadd_rn(q4, 0.0);
  Prim<R> q;
  q.r = (R)q1; q.u = (R)q2; q.v = (R)q3; q.w = (R)q4; q.p = (R)q5;
  return q;
}

// ---------------------------------------------------------------------------
// One-direction limited slope (uslope, umuscl.f90:1241-1473) for slope types
// 1 (minmod), 2 (moncen), 7 (van Leer), 8 (generalised moncen).
// ---------------------------------------------------------------------------
// FP32 form of the same limiters for the mixed path: the values of the
// expressions below, with the factors of two moved out of the min/max
// (exact scalings) and the sign applied last; a zero slope is +0.
__device__ __forceinline__ float slope1_f32(float qm1, float q0, float qp1, int st, float theta) {
  const float a = q0 - qm1, b = qp1 - q0;
  const float m = fminf(fabsf(a), fabsf(b));
  float s;
  if (st == 1) s = copysignf(m, a);
  else if (st == 2) { const float cen = 0.5f * (a + b); s = copysignf(fminf(2.0f * m, fabsf(cen)), cen); }
  else if (st == 7) s = __fdividef(2.0f * a * b, a + b);
  else if (st == 8) { const float cen = 0.5f * (a + b); s = copysignf(fminf(theta * m, fabsf(cen)), cen); }
  else return 0.0f;
  return a * b <= 0.0f ? 0.0f : s;
}

template <typename R>
__device__ __forceinline__ R slope1(R qm1, R q0, R qp1, int st, R theta) {
  if constexpr (sizeof(R) == 4) return slope1_f32(qm1, q0, qp1, st, theta);
  const R zero = (R)0, half = (R)0.5, one = (R)1;
  // minmod and van Leer are written as selects, not early returns: the same
  // values, without divergent branches inside a warp
  if (st == 1) {
    R dlft = q0 - qm1;
    R drgt = qp1 - q0;
    const R lim = dlft > 0 ? fmn(dlft, drgt) : fmx(dlft, drgt);
    return (dlft * drgt) <= zero ? zero : lim;
  } else if (st == 2) {
    const R two = (R)2;
    R dlft = two * (q0 - qm1);
    R drgt = two * (qp1 - q0);
    R dcen = half * (dlft + drgt) / two;
    R dsgn = copysign(one, dcen);
    R slop = fmn(fabs(dlft), fabs(drgt));
    R dlim = slop;
    if ((dlft * drgt) <= zero) dlim = zero;
    return dsgn * fmn(dlim, (R)fabs(dcen));
  } else if (st == 7) {
    R dlft = (q0 - qm1);
    R drgt = (qp1 - q0);
    const R vl = ((R)2 * dlft * drgt / (dlft + drgt));  // unused (0/0 at worst) where the product is <= 0
    return (dlft * drgt) <= zero ? zero : vl;
  } else if (st == 8) {
    R dlft = (q0 - qm1);
    R drgt = (qp1 - q0);
    R dcen = half * (dlft + drgt);
    R dsgn = copysign(one, dcen);
    R slop = fmn(theta * (R)fabs(dlft), theta * (R)fabs(drgt));
    R dlim = slop;
    if ((dlft * drgt) <= zero) dlim = zero;
    return dsgn * fmn(dlim, (R)fabs(dcen));
  }
  return zero;  // slope_type 0
}

// MUSCL-Hancock predictor for one cell (trace3d, umuscl.f90:483-708):
// given the cell state q and its 15 slopes dq[var][dir], produce the face
// states qp[dir] (right state at the left interface) and qm[dir] (left state
// at the right interface). Variables are ordered (r, u, v, w, p).
template <typename R>
__device__ __forceinline__ void trace_cell(const Prim<R>& q, const R dq[5][3], R gamma, R smallr,
                                           const R dtd[3], Prim<R> qp[3], Prim<R> qm[3],
                                           unsigned dirmask = 7u) {
  const R half = (R)0.5;
  const R r = q.r, u = q.u, v = q.v, w = q.w, p = q.p;
  const R drx = dq[0][0], dry = dq[0][1], drz = dq[0][2];
  const R dux = dq[1][0], duy = dq[1][1], duz = dq[1][2];
  const R dvx = dq[2][0], dvy = dq[2][1], dvz = dq[2][2];
  const R dwx = dq[3][0], dwy = dq[3][1], dwz = dq[3][2];
  const R dpx = dq[4][0], dpy = dq[4][1], dpz = dq[4][2];
  if constexpr (sizeof(R) == 4) {
    // FP32-mixed: the same predictor with the half-step source term
    // s*dt/(2dx), equal in every direction on a cubic cell, added once:
    // q -/+ dq/2 + s*dt/(2dx) = (q + s*dt/(2dx)) -/+ dq/2
    const float th = dtd[0] * 0.5f;
    const float divv = dux + dvy + dwz;
    const float ir = 1.0f / r;
    const float hr = r - th * (u * drx + v * dry + w * drz + divv * r);
    const float hp = p - th * (u * dpx + v * dpy + w * dpz + divv * gamma * p);
    const float hu = u - th * (u * dux + v * duy + w * duz + dpx * ir);
    const float hv = v - th * (u * dvx + v * dvy + w * dvz + dpy * ir);
    const float hw = w - th * (u * dwx + v * dwy + w * dwz + dpz * ir);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      if (!(dirmask & (1u << d))) continue;
      const float dr = half * dq[0][d], du = half * dq[1][d], dv = half * dq[2][d], dw = half * dq[3][d],
                  dp = half * dq[4][d];
      Prim<R> P, M;
      P.r = hr - dr; P.u = hu - du; P.v = hv - dv; P.w = hw - dw; P.p = hp - dp;
      M.r = hr + dr; M.u = hu + du; M.v = hv + dv; M.w = hw + dw; M.p = hp + dp;
      if (P.r < smallr) P.r = r;
      if (M.r < smallr) M.r = r;
      qp[d] = P;
      qm[d] = M;
    }
    return;
  }
  // source terms (:576-580)
  const R sr0 = -(u * drx) - v * dry - w * drz - (dux + dvy + dwz) * r;
  const R sp0 = -(u * dpx) - v * dpy - w * dpz - (dux + dvy + dwz) * gamma * p;
  const R su0 = -(u * dux) - v * duy - w * duz - (dpx) / r;
  const R sv0 = -(u * dvx) - v * dvy - w * dvz - (dpy) / r;
  const R sw0 = -(u * dwx) - v * dwy - w * dwz - (dpz) / r;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (!(dirmask & (1u << d))) continue;
    const R t = dtd[d];
    const R dr = dq[0][d], du = dq[1][d], dv = dq[2][d], dw = dq[3][d], dp = dq[4][d];
    Prim<R> P, M;
    P.r = r - half * dr + sr0 * t * half;
    P.p = p - half * dp + sp0 * t * half;
    P.u = u - half * du + su0 * t * half;
    P.v = v - half * dv + sv0 * t * half;
    P.w = w - half * dw + sw0 * t * half;
    if (P.r < smallr) P.r = r;
    M.r = r + half * dr + sr0 * t * half;
    M.p = p + half * dp + sp0 * t * half;
    M.u = u + half * du + su0 * t * half;
    M.v = v + half * dv + sv0 * t * half;
    M.w = w + half * dw + sw0 * t * half;
    if (M.r < smallr) M.r = r;
    qp[d] = P;
    qm[d] = M;
  }
}

// PLMDE predictor, one direction (tracexyz, uplmde.f90:470-520 for x):
// characteristic amplitudes of the slopes, each wave traced to the face only
// when it moves towards it (project_out = 1 otherwise), the sound wave speed
// zeroed where |du_n| > 3c (supersonic fix). In the face frame: r, normal
// velocity un, p, transverse velocities t1, t2 and their half-step sources s*.
// P/M = (r, un, p, t1, t2) of the right state at the lower face and of the
// left state at the upper face.
template <typename R>
__device__ __forceinline__ void plmde_dir(R r, R un, R p, R t1, R t2, R cc, R csq, R dr, R dun, R dp, R dt1,
                                          R dt2, R dtd, R sr, R sun, R sp, R st1, R st2, R smallr, R P[5],
                                          R M[5]) {
  const R half = (R)0.5, one = (R)1, zero = (R)0, three = (R)3;
  const R alpham = half * (dp / csq - dun * r / cc);
  const R alphap = half * (dp / csq + dun * r / cc);
  const R alpha0r = dr - dp / csq;
  const R ccc = ((R)fabs(dun) > three * cc) ? zero : cc;
  {
    R spminus = (un - ccc) * dtd, spplus = (un + ccc) * dtd, spzero = un * dtd;
    if ((un + ccc) > zero) spplus = -one;
    if ((un - ccc) > zero) spminus = -one;
    if (un > zero) spzero = -one;
    const R ap = half * (-one - spplus) * alphap;
    const R am = half * (-one - spminus) * alpham;
    const R azr = half * (-one - spzero) * alpha0r;
    const R az1 = half * (-one - spzero) * dt1;
    const R az2 = half * (-one - spzero) * dt2;
    P[0] = fmx<R>(smallr, r + (ap + am + azr) + sr);
    P[1] = un + (ap - am) * cc / r + sun;
    P[2] = p + (ap + am) * csq + sp;
    P[3] = t1 + az1 + st1;
    P[4] = t2 + az2 + st2;
  }
  {
    R spminus = (un - ccc) * dtd, spplus = (un + ccc) * dtd, spzero = un * dtd;
    if ((un + ccc) <= zero) spplus = one;
    if ((un - ccc) <= zero) spminus = one;
    if (un <= zero) spzero = one;
    const R ap = half * (one - spplus) * alphap;
    const R am = half * (one - spminus) * alpham;
    const R azr = half * (one - spzero) * alpha0r;
    const R az1 = half * (one - spzero) * dt1;
    const R az2 = half * (one - spzero) * dt2;
    M[0] = fmx<R>(smallr, r + (ap + am + azr) + sr);
    M[1] = un + (ap - am) * cc / r + sun;
    M[2] = p + (ap + am) * csq + sp;
    M[3] = t1 + az1 + st1;
    M[4] = t2 + az2 + st2;
  }
}

// PLMDE predictor for one cell (scheme='plmde': tracexyz, uplmde.f90:375-696),
// same interface as trace_cell. The transverse source terms are the
// reference's (:459-469), all scaled by dt/dx; the sound speed is ctoprim's
// sqrt((gamma*p)*(1/rho)) (umuscl.f90:936-937).
template <typename R>
__device__ __forceinline__ void trace_plmde_cell(const Prim<R>& q, const R dq[5][3], R gamma, R smallr,
                                                 const R dtd[3], Prim<R> qp[3], Prim<R> qm[3],
                                                 unsigned dirmask = 7u) {
  const R half = (R)0.5;
  const R r = q.r, u = q.u, v = q.v, w = q.w, p = q.p;
  R cc = gamma * p;
  cc = (R)sqrt(cc * ((R)1 / r));
  const R csq = gamma * p / r;
  const R drx = dq[0][0], dry = dq[0][1], drz = dq[0][2];
  const R dux = dq[1][0], duy = dq[1][1], duz = dq[1][2];
  const R dvx = dq[2][0], dvy = dq[2][1], dvz = dq[2][2];
  const R dwx = dq[3][0], dwy = dq[3][1], dwz = dq[3][2];
  const R dpx = dq[4][0], dpy = dq[4][1], dpz = dq[4][2];
  const R hdt = half * dtd[0];
  R P[5], M[5];
  if (dirmask & 1u) {
    const R srx = hdt * (-v * dry - w * drz - (dvy + dwz) * r);
    const R spx = hdt * (-v * dpy - w * dpz - (dvy + dwz) * gamma * p);
    const R sux = hdt * (-v * duy - w * duz);
    const R svx = hdt * (-v * dvy - w * dvz - (dpy) / r);
    const R swx = hdt * (-v * dwy - w * dwz - (dpz) / r);
    plmde_dir<R>(r, u, p, v, w, cc, csq, drx, dux, dpx, dvx, dwx, dtd[0], srx, sux, spx, svx, swx, smallr, P, M);
    qp[0].r = P[0]; qp[0].u = P[1]; qp[0].p = P[2]; qp[0].v = P[3]; qp[0].w = P[4];
    qm[0].r = M[0]; qm[0].u = M[1]; qm[0].p = M[2]; qm[0].v = M[3]; qm[0].w = M[4];
  }
  if (dirmask & 2u) {
    const R sry = hdt * (-u * drx - w * drz - (dux + dwz) * r);
    const R spy = hdt * (-u * dpx - w * dpz - (dux + dwz) * gamma * p);
    const R suy = hdt * (-u * dux - w * duz - (dpx) / r);
    const R svy = hdt * (-u * dvx - w * dvz);
    const R swy = hdt * (-u * dwx - w * dwz - (dpz) / r);
    plmde_dir<R>(r, v, p, u, w, cc, csq, dry, dvy, dpy, duy, dwy, dtd[1], sry, svy, spy, suy, swy, smallr, P, M);
    qp[1].r = P[0]; qp[1].v = P[1]; qp[1].p = P[2]; qp[1].u = P[3]; qp[1].w = P[4];
    qm[1].r = M[0]; qm[1].v = M[1]; qm[1].p = M[2]; qm[1].u = M[3]; qm[1].w = M[4];
  }
  if (dirmask & 4u) {
    const R srz = hdt * (-v * dry - u * drx - (dvy + dux) * r);
    const R spz = hdt * (-v * dpy - u * dpx - (dvy + dux) * gamma * p);
    const R suz = hdt * (-v * duy - u * dux - (dpx) / r);
    const R svz = hdt * (-v * dvy - u * dvx - (dpy) / r);
    const R swz = hdt * (-v * dwy - u * dwx);
    plmde_dir<R>(r, w, p, u, v, cc, csq, drz, dwz, dpz, duz, dvz, dtd[2], srz, swz, spz, suz, svz, smallr, P, M);
    qp[2].r = P[0]; qp[2].w = P[1]; qp[2].p = P[2]; qp[2].u = P[3]; qp[2].v = P[4];
    qm[2].r = M[0]; qm[2].w = M[1]; qm[2].p = M[2]; qm[2].u = M[3]; qm[2].v = M[4];
  }
}

// The predictor of the scheme: PLMDE in the compiled PLMDE variants
// (ST >= 10, slope type ST % 10), chosen from c.scheme in the run-time
// variant (RS == 0), MUSCL-Hancock otherwise.
template <typename R, int RS, int ST = -1>
__device__ __forceinline__ void trace_sel(const Prim<R>& q, const R dq[5][3], const Consts<R>& c, const R dtd[3],
                                          Prim<R> qp[3], Prim<R> qm[3], unsigned dirmask) {
  if constexpr (ST >= 10) {
    trace_plmde_cell<R>(q, dq, c.gamma, c.smallr, dtd, qp, qm, dirmask);
    return;
  }
  if constexpr (RS == 0) {
    if (c.scheme == RB_SCHEME_PLMDE) {
      trace_plmde_cell<R>(q, dq, c.gamma, c.smallr, dtd, qp, qm, dirmask);
      return;
    }
  }
  trace_cell<R>(q, dq, c.gamma, c.smallr, dtd, qp, qm, dirmask);
}

// ---------------------------------------------------------------------------
// Riemann solvers (godunov_utils.f90). Inputs in the face frame:
// (rho, u_normal, P, u_t1, u_t2). Output f[0..4] = (mass, normal momentum,
// energy, t1 momentum, t2 momentum) and f[5] = thermal-energy flux.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void riemann_llf(const R ql[5], const R qr[5], const Consts<R>& c, R f[6]) {
  // :660-820
  const R half = c.half;
  R rl = fmx(ql[0], c.smallr), ul = ql[1], pl = fmx(ql[2], rl * c.smallp);
  R cl = c.gamma * pl;
  cl = sqrt(cl / rl);
  R rr = fmx(qr[0], c.smallr), ur = qr[1], pr = fmx(qr[2], rr * c.smallp);
  R cr = c.gamma * pr;
  cr = sqrt(cr / rr);
  R cmax = fmx((R)fabs(ul) + cl, (R)fabs(ur) + cr);
  R uL[6], uR[6], fL[6], fR[6];
  uL[0] = ql[0]; uR[0] = qr[0];
  uL[1] = ql[0] * ql[1]; uR[1] = qr[0] * qr[1];
  uL[2] = ql[2] * c.entho + half * ql[0] * (ql[1] * ql[1]);
  uR[2] = qr[2] * c.entho + half * qr[0] * (qr[1] * qr[1]);
  uL[2] = uL[2] + half * ql[0] * (ql[3] * ql[3]);
  uR[2] = uR[2] + half * qr[0] * (qr[3] * qr[3]);
  uL[2] = uL[2] + half * ql[0] * (ql[4] * ql[4]);
  uR[2] = uR[2] + half * qr[0] * (qr[4] * qr[4]);
  uL[3] = ql[0] * ql[3]; uR[3] = qr[0] * qr[3];
  uL[4] = ql[0] * ql[4]; uR[4] = qr[0] * qr[4];
  uL[5] = ql[2] * c.entho; uR[5] = qr[2] * c.entho;
  fL[0] = ql[1] * uL[0]; fR[0] = qr[1] * uR[0];
  fL[1] = ql[1] * uL[1] + ql[2]; fR[1] = qr[1] * uR[1] + qr[2];
  fL[2] = ql[1] * (uL[2] + ql[2]); fR[2] = qr[1] * (uR[2] + qr[2]);
#pragma unroll
  for (int n = 3; n < 6; n++) { fL[n] = ql[1] * uL[n]; fR[n] = qr[1] * uR[n]; }
#pragma unroll
  for (int n = 0; n < 6; n++) f[n] = half * (fL[n] + fR[n] - cmax * (uR[n] - uL[n]));
}

template <typename R>
__device__ __forceinline__ void riemann_hll(const R ql[5], const R qr[5], const Consts<R>& c, R f[6]) {
  // :825-983
  const R half = c.half, zero = (R)0;
  R rl = fmx(ql[0], c.smallr), ul = ql[1], pl = fmx(ql[2], rl * c.smallp);
  R cl = c.gamma * pl;
  cl = sqrt(cl / rl);
  R rr = fmx(qr[0], c.smallr), ur = qr[1], pr = fmx(qr[2], rr * c.smallp);
  R cr = c.gamma * pr;
  cr = sqrt(cr / rr);
  R SL = fmn(fmn(ul, ur) - fmx(cl, cr), zero);
  R SR = fmx(fmx(ul, ur) + fmx(cl, cr), zero);
  R uL[6], uR[6], fL[6], fR[6];
  uL[0] = ql[0]; uR[0] = qr[0];
  uL[1] = ql[0] * ql[1]; uR[1] = qr[0] * qr[1];
  uL[2] = ql[2] * c.entho + half * ql[0] * (ql[1] * ql[1]);
  uR[2] = qr[2] * c.entho + half * qr[0] * (qr[1] * qr[1]);
  uL[2] = uL[2] + half * ql[0] * (ql[3] * ql[3]);
  uR[2] = uR[2] + half * qr[0] * (qr[3] * qr[3]);
  uL[2] = uL[2] + half * ql[0] * (ql[4] * ql[4]);
  uR[2] = uR[2] + half * qr[0] * (qr[4] * qr[4]);
  uL[3] = ql[0] * ql[3]; uR[3] = qr[0] * qr[3];
  uL[4] = ql[0] * ql[4]; uR[4] = qr[0] * qr[4];
  uL[5] = ql[2] * c.entho; uR[5] = qr[2] * c.entho;
  fL[0] = uL[1]; fR[0] = uR[1];
  fL[1] = ql[2] + uL[1] * ql[1]; fR[1] = qr[2] + uR[1] * qr[1];
  fL[2] = ql[1] * (uL[2] + ql[2]); fR[2] = qr[1] * (uR[2] + qr[2]);
#pragma unroll
  for (int n = 3; n < 6; n++) { fL[n] = ql[1] * uL[n]; fR[n] = qr[1] * uR[n]; }
#pragma unroll
  for (int n = 0; n < 6; n++) f[n] = (SR * fL[n] - SL * fR[n] + SR * SL * (uR[n] - uL[n])) / (SR - SL);
}

template <typename R>
__device__ __forceinline__ void riemann_hllc(const R ql[5], const R qr[5], const Consts<R>& c, R f[6]) {
  // :988-1209 (only the sampled star state is formed; the others are dead)
  if constexpr (sizeof(R) == 4) {
    // FP32-mixed: the same solver with the kinetic energy summed before the
    // product with rho/2, and the sampled state picked by one side select
    // (left if SL > 0 or ustar > 0) and one star-or-outer select
    const float rl = fmaxf(ql[0], c.smallr), ul = ql[1], Pl = fmaxf(ql[2], rl * c.smallp);
    const float rr = fmaxf(qr[0], c.smallr), ur = qr[1], Pr = fmaxf(qr[2], rr * c.smallp);
    const float el = Pl * c.entho, er = Pr * c.entho;
    const float etotl = el + 0.5f * rl * (ul * ul + ql[3] * ql[3] + ql[4] * ql[4]);
    const float etotr = er + 0.5f * rr * (ur * ur + qr[3] * qr[3] + qr[4] * qr[4]);
    const float smallc2 = c.smallc * c.smallc;
    const float cfastl = sqrtf(fmaxf(c.gamma * Pl * __fdividef(1.0f, rl), smallc2));
    const float cfastr = sqrtf(fmaxf(c.gamma * Pr * __fdividef(1.0f, rr), smallc2));
    const float cmax = fmaxf(cfastl, cfastr);
    const float SL = fminf(ul, ur) - cmax, SR = fmaxf(ul, ur) + cmax;
    const float rcl = rl * (ul - SL), rcr = rr * (SR - ur);
    const float inv = __fdividef(1.0f, rcr + rcl);
    const float ustar = (rcr * ur + rcl * ul + (Pl - Pr)) * inv;
    const float Pstar = (rcr * Pl + rcl * Pr + rcl * rcr * (ul - ur)) * inv;
    const bool outl = SL > 0.0f, lft = ustar > 0.0f;
    const bool side = outl || lft;
    const bool star = !outl && (lft || SR > 0.0f);
    const float rs = side ? rl : rr, us = side ? ul : ur, Ss = side ? SL : SR;
    const float Ps = side ? Pl : Pr, ets = side ? etotl : etotr, es = side ? el : er;
    const float num = Ss - us, iden = __fdividef(1.0f, Ss - ustar);
    const float ro = star ? rs * num * iden : rs;
    const float uo = star ? ustar : us;
    const float Po = star ? Pstar : Ps;
    const float eto = star ? (num * ets - Ps * us + Pstar * ustar) * iden : ets;
    const float eo = star ? es * num * iden : es;
    const float mo = ro * uo;
    f[0] = mo;
    f[1] = mo * uo + Po;
    f[2] = (eto + Po) * uo;
    f[3] = mo * (lft ? ql[3] : qr[3]);
    f[4] = mo * (lft ? ql[4] : qr[4]);
    f[5] = uo * eo;
    return;
  }
  const R half = c.half;
  R rl = fmx(ql[0], c.smallr);
  R Pl = fmx(ql[2], rl * c.smallp);
  R ul = ql[1];
  R el = Pl * c.entho;
  R ecinl = half * rl * ul * ul;
  ecinl = ecinl + half * rl * (ql[3] * ql[3]);
  ecinl = ecinl + half * rl * (ql[4] * ql[4]);
  R etotl = el + ecinl;
  R Ptotl = Pl;
  R rr = fmx(qr[0], c.smallr);
  R Pr = fmx(qr[2], rr * c.smallp);
  R ur = qr[1];
  R er = Pr * c.entho;
  R ecinr = half * rr * ur * ur;
  ecinr = ecinr + half * rr * (qr[3] * qr[3]);
  ecinr = ecinr + half * rr * (qr[4] * qr[4]);
  R etotr = er + ecinr;
  R Ptotr = Pr;
  const R smallc2 = c.smallc * c.smallc;
  R cfastl = c.gamma * Pl;
  cfastl = sqrt(fmx(cfastl / rl, smallc2));
  R cfastr = c.gamma * Pr;
  cfastr = sqrt(fmx(cfastr / rr, smallc2));
  R SL = fmn(ul, ur) - fmx(cfastl, cfastr);
  R SR = fmx(ul, ur) + fmx(cfastl, cfastr);
  R rcl = rl * (ul - SL);
  R rcr = rr * (SR - ur);
  R ustar, Ptotstar;
  if (sizeof(R) == 4) {  // FP32-mixed: one reciprocal for the two star quotients
    const R inv = (R)1 / (rcr + rcl);
    ustar = (rcr * ur + rcl * ul + (Ptotl - Ptotr)) * inv;
    Ptotstar = (rcr * Ptotl + rcl * Ptotr + rcl * rcr * (ul - ur)) * inv;
  } else {
    ustar = (rcr * ur + rcl * ul + (Ptotl - Ptotr)) / (rcr + rcl);
    Ptotstar = (rcr * Ptotl + rcl * Ptotr + rcl * rcr * (ul - ur)) / (rcr + rcl);
  }
  // Sampling at x/t = 0: the outer left state if SL > 0, else the left star
  // state if ustar > 0, else the right star state if SR > 0, else the outer
  // right state. Written with selects (no divergent branches): the star side
  // is picked first and one star state is formed with the same operations as
  // the reference's branch for that side.
  const bool lft = ustar > (R)0;
  const R rs = lft ? rl : rr, us = lft ? ul : ur, Ss = lft ? SL : SR;
  const R Pts = lft ? Ptotl : Ptotr, ets = lft ? etotl : etotr, es = lft ? el : er;
  const R num = Ss - us, den = Ss - ustar;
  R ro_s, etoto_s, eo_s;
  if (sizeof(R) == 4) {
    const R inv = (R)1 / den;
    ro_s = rs * num * inv;
    etoto_s = (num * ets - Pts * us + Ptotstar * ustar) * inv;
    eo_s = es * num * inv;
  } else {
    ro_s = rs * num / den;
    etoto_s = (num * ets - Pts * us + Ptotstar * ustar) / den;
    eo_s = es * num / den;
  }
  const bool outl = SL > (R)0;
  const bool star = !outl && (lft || SR > (R)0);
  const R ro = outl ? rl : (star ? ro_s : rr);
  const R uo = outl ? ul : (star ? ustar : ur);
  const R Ptoto = outl ? Ptotl : (star ? Ptotstar : Ptotr);
  const R etoto = outl ? etotl : (star ? etoto_s : etotr);
  const R eo = outl ? el : (star ? eo_s : er);
  f[0] = ro * uo;
  f[1] = ro * uo * uo + Ptoto;
  f[2] = (etoto + Ptoto) * uo;
  const R t3 = lft ? ql[3] : qr[3], t4 = lft ? ql[4] : qr[4];
  f[3] = ro * uo * t3;
  f[4] = ro * uo * t4;
  f[5] = uo * eo;
}

// Fluxes of the sampled face state q = (rho, u_n, P, u_t1, u_t2, e) of the
// acoustic and exact solvers (godunov_utils.f90:461-491, 628-655).
template <typename R>
__device__ __forceinline__ void flux_of_state(const R q[6], const Consts<R>& c, R f[6]) {
  const R half = c.half;
  f[0] = q[0] * q[1];
  f[1] = q[2] + q[0] * (q[1] * q[1]);
  R etot = q[2] * c.entho + half * q[0] * (q[1] * q[1]);
  etot = etot + half * q[0] * (q[3] * q[3]);
  etot = etot + half * q[0] * (q[4] * q[4]);
  f[2] = q[1] * (etot + q[2]);
  f[3] = f[0] * q[3];
  f[4] = f[0] * q[4];
  f[5] = f[0] * q[5];
}

template <typename R>
__device__ __forceinline__ void riemann_acoustic(const R ql[5], const R qr[5], const Consts<R>& c, R f[6]) {
  // :500-655, linearised (acoustic) star state
  const R one = (R)1, half = c.half, zero = (R)0;
  const R rl = fmx(ql[0], c.smallr), ul = ql[1], pl = fmx(ql[2], rl * c.smallp);
  const R rr = fmx(qr[0], c.smallr), ur = qr[1], pr = fmx(qr[2], rr * c.smallp);
  const R cl = sqrt(c.gamma * pl / rl), cr = sqrt(c.gamma * pr / rr);
  const R wl = cl * rl, wr = cr * rr;
  const R pstar = ((wr * pl + wl * pr) + wl * wr * (ul - ur)) / (wl + wr);
  const R ustar = ((wr * ur + wl * ul) + (pl - pr)) / (wl + wr);
  const R sgnm = copysign(one, ustar);
  const bool left = sgnm == one;
  const R ro = left ? rl : rr, uo = left ? ul : ur, po = left ? pl : pr, co = left ? cl : cr;
  R rstar = ro + (pstar - po) / (co * co);
  rstar = fmx(rstar, c.smallr);
  R cstar = sqrt(fabs(c.gamma * pstar / rstar));
  cstar = fmx(cstar, c.smallc);
  R spout = co - sgnm * uo;
  R spin = cstar - sgnm * ustar;
  R ushock = half * (spin + spout);
  ushock = fmx(ushock, -sgnm * ustar);
  if (pstar >= po) { spout = ushock; spin = spout; }
  R q[6];
  if (spout < zero) { q[0] = ro; q[1] = uo; q[2] = po; }
  else if (spin >= zero) { q[0] = rstar; q[1] = ustar; q[2] = pstar; }
  else {
    const R frac = spout / (spout - spin);
    q[0] = frac * rstar + (one - frac) * ro;
    q[1] = frac * ustar + (one - frac) * uo;
    q[2] = frac * pstar + (one - frac) * po;
  }
  q[3] = left ? ql[3] : qr[3];
  q[4] = left ? ql[4] : qr[4];
  q[5] = po / ro * c.entho;
  flux_of_state(q, c, f);
}

template <typename R>
__device__ __forceinline__ void riemann_exact(const R ql[5], const R qr[5], const Consts<R>& c, R f[6]) {
  // riemann_approx :268-495: two-shock Newton iterations for the star
  // pressure (at most niter_riemann, until |dp/p| <= 1e-6), then the exact
  // sampling with rarefaction fans
  const R one = (R)1, two = (R)2, half = c.half, zero = (R)0;
  const R smallpp = c.smallr * c.smallp;
  const R gamma6 = (c.gamma + one) / (two * c.gamma);
  const R rl = fmx(ql[0], c.smallr), ul = ql[1], pl = fmx(ql[2], rl * c.smallp);
  const R rr = fmx(qr[0], c.smallr), ur = qr[1], pr = fmx(qr[2], rr * c.smallp);
  const R cl = c.gamma * pl * rl, cr = c.gamma * pr * rr;
  R wl = sqrt(cl), wr = sqrt(cr);
  R pstar = ((wr * pl + wl * pr) + wl * wr * (ul - ur)) / (wl + wr);
  pstar = fmx(pstar, zero);
  R pold = pstar;
  for (int iter = 1; iter <= c.niter_riemann; iter++) {
    const R wwl = sqrt(cl * (one + gamma6 * (pold - pl) / pl));
    const R wwr = sqrt(cr * (one + gamma6 * (pold - pr) / pr));
    const R qlw = two * (wwl * wwl * wwl) / (wwl * wwl + cl);
    const R qrw = two * (wwr * wwr * wwr) / (wwr * wwr + cr);
    const R usl = ul - (pold - pl) / wwl;
    const R usr = ur + (pold - pr) / wwr;
    const R delp = fmx(qrw * qlw / (qrw + qlw) * (usl - usr), -pold);
    pold = pold + delp;
    if (!(fabs(delp / (pold + smallpp)) > (R)1e-06)) break;  // converged
  }
  pstar = pold;
  wl = sqrt(cl * (one + gamma6 * (pstar - pl) / pl));
  wr = sqrt(cr * (one + gamma6 * (pstar - pr) / pr));
  const R ustar = half * (ul + (pl - pstar) / wl + ur - (pr - pstar) / wr);
  const R sgnm = copysign(one, ustar);
  const bool left = sgnm == one;
  const R ro = left ? rl : rr, uo = left ? ul : ur, po = left ? pl : pr, wo = left ? wl : wr;
  const R co = fmx(c.smallc, (R)sqrt(fabs(c.gamma * po / ro)));
  R rstar;
  if (pstar >= po) rstar = ro / (one + ro * (po - pstar) / (wo * wo));
  else rstar = ro * pow(pstar / po, one / c.gamma);
  rstar = fmx(rstar, c.smallr);
  R cstar = sqrt(fabs(c.gamma * pstar / rstar));
  cstar = fmx(cstar, c.smallc);
  R spout = co - sgnm * uo;
  R spin = cstar - sgnm * ustar;
  const R ushock = wo / ro - sgnm * uo;
  if (pstar >= po) { spout = ushock; spin = spout; }
  R q[6];
  if (spout <= zero) { q[0] = ro; q[1] = uo; q[2] = po; }
  else if (spin >= zero) { q[0] = rstar; q[1] = ustar; q[2] = pstar; }
  else {
    const R frac = spout / (spout - spin);
    q[1] = frac * ustar + (one - frac) * uo;
    q[2] = frac * pstar + (one - frac) * po;
    q[0] = ro * pow(q[2] / po, one / c.gamma);
  }
  q[3] = left ? ql[3] : qr[3];
  q[4] = left ? ql[4] : qr[4];
  q[5] = po / ro * c.entho;
  flux_of_state(q, c, f);
}

template <typename R>
__device__ __forceinline__ void riemann(const R ql[5], const R qr[5], const Consts<R>& c, R f[6]) {
  if (c.riemann == RB_RIEMANN_HLLC) riemann_hllc(ql, qr, c, f);
  else if (c.riemann == RB_RIEMANN_HLL) riemann_hll(ql, qr, c, f);
  else if (c.riemann == RB_RIEMANN_ACOUSTIC) riemann_acoustic(ql, qr, c, f);
  else if (c.riemann == RB_RIEMANN_EXACT) riemann_exact(ql, qr, c, f);
  else riemann_llf(ql, qr, c, f);
}

// Riemann solver fixed at compile time (RS = RB_RIEMANN_*), or chosen at run
// time from c.riemann when RS == 0.
template <typename R, int RS>
__device__ __forceinline__ void riemann_sel(const R ql[5], const R qr[5], const Consts<R>& c, R f[6]) {
  if (RS == RB_RIEMANN_HLLC) riemann_hllc(ql, qr, c, f);
  else if (RS == RB_RIEMANN_HLL) riemann_hll(ql, qr, c, f);
  else if (RS == RB_RIEMANN_LLF) riemann_llf(ql, qr, c, f);
  else riemann(ql, qr, c, f);
}

// Face frame permutation of cmpflxm (umuscl.f90:745-790): normal velocity of
// direction d is variable 1+d; the tangential ones are the remaining two in
// ascending order.
template <typename R>
__device__ __forceinline__ void to_face(const Prim<R>& s, int d, R out[5]) {
  out[0] = s.r;
  out[2] = s.p;
  if (d == 0) { out[1] = s.u; out[3] = s.v; out[4] = s.w; }
  else if (d == 1) { out[1] = s.v; out[3] = s.u; out[4] = s.w; }
  else { out[1] = s.w; out[3] = s.u; out[4] = s.v; }
}

// Godunov flux back in (rho, mx, my, mz, E) order.
template <typename R>
__device__ __forceinline__ void from_face(const R f[6], int d, R out[5]) {
  out[0] = f[0];
  out[4] = f[2];
  if (d == 0) { out[1] = f[1]; out[2] = f[3]; out[3] = f[4]; }
  else if (d == 1) { out[2] = f[1]; out[1] = f[3]; out[3] = f[4]; }
  else { out[3] = f[1]; out[1] = f[3]; out[2] = f[4]; }
}

// ---------------------------------------------------------------------------
// Coarse-to-fine prolongation of one child (interpol_hydro,
// interpol_hydro.f90:268-637). u7[j][v]: father cell (j=0) and its 6
// neighbours (-x,+x,-y,+y,-z,+z), conservative FP64. Produces the 8
// children; called per child by the gather, results identical per child.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void interp_children(double u1[7][5], const rb_hydro_params& hp,
                                                double u2[8][5]) {
  const int ivar_ = hp.interpol_var, itype = hp.interpol_type;
  const double smallr = hp.smallr;
  if (ivar_ == 1 || ivar_ == 2) {
    for (int j = 0; j <= 6; j++) {
      double ekin = 0.0;
      for (int idim = 1; idim <= 3; idim++)
        ekin = ekin + 0.5 * (u1[j][idim] * u1[j][idim]) / fmx(u1[j][0], smallr);
      const double erad = 0.0;
      u1[j][4] = u1[j][4] - ekin - erad;
      if (ivar_ == 2)
        for (int idim = 1; idim <= 3; idim++) u1[j][idim] = u1[j][idim] / fmx(u1[j][0], smallr);
    }
  }
  for (int iv = 0; iv < 5; iv++) {
    double a[7], w[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j <= 6; j++) a[j] = u1[j][iv];
    int t = itype;
    if (itype == 4) t = (iv >= 1 && iv <= 3) ? 3 : 2;
    if (t == 1) {  // compute_limiter_minmod :449-476
      for (int idim = 1; idim <= 3; idim++) {
        double dl = 0.5 * (a[2 * idim] - a[0]);
        double dr = 0.5 * (a[0] - a[2 * idim - 1]);
        double mm;
        if (dl * dr <= 0.0) mm = 0;
        else mm = fmn(fabs(dl), fabs(dr)) * dl / fabs(dl);
        w[idim - 1] = mm;
      }
    } else if (t == 3) {  // compute_central :618-637
      for (int idim = 1; idim <= 3; idim++) w[idim - 1] = 0.25 * (a[2 * idim] - a[2 * idim - 1]);
    } else if (t == 2) {  // compute_limiter_central :481-613
      for (int idim = 1; idim <= 3; idim++) w[idim - 1] = 0.25 * (a[2 * idim] - a[2 * idim - 1]);
      double ac[8];
      for (int ind = 0; ind < 8; ind++) ac[ind] = a[0];
      for (int idim = 0; idim < 3; idim++)
        for (int ind = 0; ind < 8; ind++) {
          double xc = (double)((ind >> idim) & 1) - 0.5;
          ac[ind] = ac[ind] + 2.0 * w[idim] * xc;
        }
      double corner = ac[0];
      for (int j = 1; j < 8; j++) corner = fmx(corner, ac[j]);
      double kernel = a[1];
      for (int j = 2; j <= 6; j++) kernel = fmx(kernel, a[j]);
      double dk = a[0] - kernel, dc = a[0] - corner;
      double max_lim = 0.0;
      if (dk * dc > 0.0) max_lim = fmn(1.0, dk / dc);
      corner = ac[0];
      for (int j = 1; j < 8; j++) corner = fmn(corner, ac[j]);
      kernel = a[1];
      for (int j = 2; j <= 6; j++) kernel = fmn(kernel, a[j]);
      dk = a[0] - kernel;
      dc = a[0] - corner;
      double min_lim = 0.0;
      if (dk * dc > 0.0) min_lim = fmn(1.0, dk / dc);
      double lim = fmn(min_lim, max_lim);
      for (int idim = 0; idim < 3; idim++) w[idim] = w[idim] * lim;
    }
    for (int ind = 0; ind < 8; ind++) {
      double v = a[0];
      for (int idim = 0; idim < 3; idim++) v = v + w[idim] * ((double)((ind >> idim) & 1) - 0.5);
      u2[ind][iv] = v;
    }
  }
  if (ivar_ == 1 || ivar_ == 2) {
    if (ivar_ == 2) {
      for (int ind = 0; ind < 8; ind++)
        for (int idim = 1; idim <= 3; idim++) u2[ind][idim] = u2[ind][idim] * u2[ind][0];
      for (int idim = 1; idim <= 3; idim++) {
        double mom = 0;
        for (int ind = 0; ind < 8; ind++) mom = mom + u2[ind][idim] * 0.125;
        mom = mom - u1[0][idim] * u1[0][0];
        for (int ind = 0; ind < 8; ind++) u2[ind][idim] = u2[ind][idim] - mom;
      }
    }
    for (int ind = 0; ind < 8; ind++) {
      double ekin = 0.0;
      for (int idim = 1; idim <= 3; idim++)
        ekin = ekin + 0.5 * (u2[ind][idim] * u2[ind][idim]) / fmx(u2[ind][0], smallr);
      const double erad = 0.0;
      u2[ind][4] = u2[ind][4] + ekin + erad;
    }
  }
}

// Per-cell CFL time step (cmpdt, godunov_utils.f90:5-120) with zero gravity.
// CFL wave speed ndim*c + sum|v| of one cell in cmpdt's operation order.
__device__ __forceinline__ double cfl_speed(const double uu_in[5], const rb_hydro_params& hp) {
  const double gamma = hp.gamma, smallc = hp.smallc;
  const double smallp = smallc * smallc / gamma;
  double u1 = fmx(uu_in[0], hp.smallr);
  double v1 = uu_in[1] / u1, v2 = uu_in[2] / u1, v3 = uu_in[3] / u1;
  double e = uu_in[4];
  e = e - 0.5 * u1 * (v1 * v1);
  e = e - 0.5 * u1 * (v2 * v2);
  e = e - 0.5 * u1 * (v3 * v3);
  e = fmx((gamma - 1.0) * e, u1 * smallp);
  e = gamma * e;
  e = sqrt(e / u1);
  e = 3.0 * e;
  e = e + fabs(v1);
  e = e + fabs(v2);
  e = e + fabs(v3);
  return e;
}

// Same speed for the FP32-mixed path: the internal energy
// E - |m|^2/(2 rho) and its floor in FP64 (a Newton-refined reciprocal instead
// of four divisions), the sound speed and the velocity sum in FP32 (relative
// difference ~1e-7 from cfl_speed; the dt minimum over cells is formed from
// the maximum speed as in the FP64 path).
__device__ __forceinline__ double cfl_speed_fast(const double u[5], const rb_hydro_params& hp) {
  const double gamma = hp.gamma;
  const double rho = fmax(u[0], hp.smallr);
  const double ir = rcp_newton(rho);
  double e = u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) * ir;
  e = fmax((gamma - 1.0) * e, rho * (hp.smallc * hp.smallc / gamma));
  const float irf = (float)ir;
  const float vs = (fabsf((float)u[1]) + fabsf((float)u[2]) + fabsf((float)u[3])) * irf;
  return (double)(3.0f * sqrtf((float)(gamma * e) * irf) + vs);
}

// With zero gravity the gravity-strength ratio of cmpdt is its floor 1e-4 in
// every cell, so dt_cell = ((dx/speed)*(sqrt(1+2*C*1e-4)-1))/1e-4 is a
// monotone function of the speed: the minimum over cells is exactly
// dt_cell(maximum speed). (godunov_utils.f90:100-118)
__device__ __forceinline__ double cfl_dt_from_speed(double s, double dx, double C) {
  const double g = 0.0001;
  return dx / s * (sqrt(1.0 + 2.0 * C * g) - 1.0) / g;
}

}  // namespace rb
