// opcount.cpp -- exact floating-point operation counts of the oracle's hydro
// stages, per cell update. TEST AND MEASUREMENT INFRASTRUCTURE ONLY: it
// compiles ramses_oracle.c unchanged with every `double` replaced by a
// counting number type, runs the stages on seeded states, and prints the
// counts as JSON. Nothing in the product library links or calls it.
//
// Stages (hydro/umuscl.f90 and godunov_utils.f90, as restated by the oracle):
//   ctoprim      per cell          (umuscl.f90:861-965)
//   uslope       per cell, 15 limited slopes (umuscl.f90:1240-1478)
//   trace3d      per cell, 6 face states (umuscl.f90:483-708)
//   cmpflxm      per face: one Riemann problem (godunov_utils.f90) + the
//                tmp half sum, and unsplit's flux*dt/dx scaling (umuscl.f90:101-163)
//   update       per cell: unew += flux(i) - flux(i+1) in x, y, z
//                (godunov_fine.f90:751-792)
//   cmpdt        per cell (godunov_utils.f90:5-120)
// "algorithmic" = ctoprim + uslope + trace3d + 3 faces + update + cmpdt: every
// quantity of one cell update formed once. "reference_dense_step" is what the
// reference's godunov_fine executes per cell update on a uniform periodic grid
// (the 6^3 stencil per oct: 27x ctoprim, 8x slopes and trace, 1.5x faces).
//
// Build and run:  g++ -O1 -std=c++17 oracle/opcount.cpp -o <out> && <out> [riemann] [slope_type]
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <cmath>
#include <cstdio>
#include <random>

namespace opc {
struct Counts {
  long long add = 0, mul = 0, div = 0, sqrt = 0, pow = 0, cmp = 0, abs = 0, sgn = 0, neg = 0;
  long long flops() const { return add + mul + div + sqrt + pow; }
};
Counts g;
}  // namespace opc

// A double that counts the operations applied to it.
struct CD {
  double v;
  CD() = default;
  constexpr CD(double x) : v(x) {}
  explicit operator double() const { return v; }
  explicit operator int() const { return (int)v; }
  explicit operator long() const { return (long)v; }
  explicit operator long long() const { return (long long)v; }
};
inline CD operator+(CD a, CD b) { opc::g.add++; return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { opc::g.add++; return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { opc::g.mul++; return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { opc::g.div++; return CD(a.v / b.v); }
inline CD operator-(CD a) { opc::g.neg++; return CD(-a.v); }
inline CD operator+(CD a) { return a; }
inline CD& operator+=(CD& a, CD b) { a = a + b; return a; }
inline CD& operator-=(CD& a, CD b) { a = a - b; return a; }
inline CD& operator*=(CD& a, CD b) { a = a * b; return a; }
inline CD& operator/=(CD& a, CD b) { a = a / b; return a; }
inline bool operator<(CD a, CD b) { opc::g.cmp++; return a.v < b.v; }
inline bool operator>(CD a, CD b) { opc::g.cmp++; return a.v > b.v; }
inline bool operator<=(CD a, CD b) { opc::g.cmp++; return a.v <= b.v; }
inline bool operator>=(CD a, CD b) { opc::g.cmp++; return a.v >= b.v; }
inline bool operator==(CD a, CD b) { opc::g.cmp++; return a.v == b.v; }
inline bool operator!=(CD a, CD b) { opc::g.cmp++; return a.v != b.v; }
inline CD sqrt(CD a) { opc::g.sqrt++; return CD(std::sqrt(a.v)); }
inline CD fabs(CD a) { opc::g.abs++; return CD(std::fabs(a.v)); }
inline CD copysign(CD a, CD b) { opc::g.sgn++; return CD(std::copysign(a.v, b.v)); }
inline CD pow(CD a, CD b) { opc::g.pow++; return CD(std::pow(a.v, b.v)); }

#define double CD
#include "ramses_oracle.c"
#undef double

namespace {

orc_params params(int riemann, int slope_type) {
  orc_params p;
  memset(&p, 0, sizeof p);
  p.gamma = 1.001; p.smallr = 1e-10; p.smallc = 1e-10; p.courant_factor = 0.8; p.slope_theta = 1.5;
  p.riemann = riemann; p.slope_type = slope_type; p.interpol_var = 0; p.interpol_type = 1;
  p.niter_riemann = 10; p.difmag = 0.0; p.scheme = 0;
  return p;
}

// seeded conservative states of the turbulent-box kind: rho log-normal,
// supersonic velocities, P = 0.01 rho
void seeded_state(std::mt19937_64& rng, CD u[5]) {
  std::normal_distribution<double> n01(0.0, 1.0);
  const double rho = std::exp(n01(rng));
  const double vx = 0.5 * n01(rng), vy = 0.5 * n01(rng), vz = 0.5 * n01(rng);
  const double p = 0.01 * rho;
  u[0] = rho; u[1] = rho * vx; u[2] = rho * vy; u[3] = rho * vz;
  u[4] = p / (1.001 - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz);
}

struct Delta {
  opc::Counts c;
  double per;
};
Delta measure(opc::Counts before, double units) {
  const opc::Counts& a = opc::g;
  Delta d;
  d.c.add = a.add - before.add; d.c.mul = a.mul - before.mul; d.c.div = a.div - before.div;
  d.c.sqrt = a.sqrt - before.sqrt; d.c.pow = a.pow - before.pow; d.c.cmp = a.cmp - before.cmp;
  d.c.abs = a.abs - before.abs; d.c.sgn = a.sgn - before.sgn; d.c.neg = a.neg - before.neg;
  d.per = units;
  return d;
}
void print(const char* name, const Delta& d, bool comma) {
  const double u = d.per;
  printf("  \"%s\": {\"add\": %.4f, \"mul\": %.4f, \"div\": %.4f, \"sqrt\": %.4f, \"pow\": %.4f, \"cmp\": %.4f, "
         "\"abs\": %.4f, \"copysign\": %.4f, \"neg\": %.4f, \"flops\": %.4f}%s\n",
         name, d.c.add / u, d.c.mul / u, d.c.div / u, d.c.sqrt / u, d.c.pow / u, d.c.cmp / u, d.c.abs / u,
         d.c.sgn / u, d.c.neg / u, d.c.flops() / u, comma ? "," : "");
}
Delta sum(std::initializer_list<std::pair<const Delta*, double>> parts) {
  Delta s;
  s.per = 1.0;
  double add = 0, mul = 0, dv = 0, sq = 0, pw = 0, cmp = 0, ab = 0, sg = 0, ng = 0;
  for (auto& pr : parts) {
    const Delta& d = *pr.first;
    const double w = pr.second / d.per;
    add += w * d.c.add; mul += w * d.c.mul; dv += w * d.c.div; sq += w * d.c.sqrt; pw += w * d.c.pow;
    cmp += w * d.c.cmp; ab += w * d.c.abs; sg += w * d.c.sgn; ng += w * d.c.neg;
  }
  // stored scaled by 1e6 to keep the integer fields
  s.per = 1e6;
  s.c.add = llround(add * 1e6); s.c.mul = llround(mul * 1e6); s.c.div = llround(dv * 1e6);
  s.c.sqrt = llround(sq * 1e6); s.c.pow = llround(pw * 1e6); s.c.cmp = llround(cmp * 1e6);
  s.c.abs = llround(ab * 1e6); s.c.sgn = llround(sg * 1e6); s.c.neg = llround(ng * 1e6);
  return s;
}

}  // namespace

int main(int argc, char** argv) {
  const int riemann = argc > 1 ? atoi(argv[1]) : ORC_RIEMANN_HLLC;
  const int slope_type = argc > 2 ? atoi(argv[2]) : 2;
  orc_params p = params(riemann, slope_type);
  std::mt19937_64 rng(2024);
  const int nv = 1;
  // one oct's 6^3 stencil (nvector = 1)
  work w;
  if (work_init(&w, nv)) return 1;
  CD* uin = (CD*)malloc(sizeof(CD) * 216 * NV);
  CD* gin = (CD*)calloc(216 * 3, sizeof(CD));
  for (int c = 0; c < 216; c++) {
    CD u[5];
    seeded_state(rng, u);
    for (int v = 0; v < NV; v++) uin[c + 216 * v] = u[v];
  }
  const CD dx = 1.0 / 256, dt = 1e-4;
  opc::Counts b = opc::g;
  ctoprim(&p, uin, w.qin, w.cin, gin, dt, 1, nv);
  Delta d_ctoprim = measure(b, 216);
  b = opc::g;
  if (uslope(&p, w.qin, w.dq, 1, nv)) return 2;
  Delta d_uslope = measure(b, 64);
  b = opc::g;
  trace3d(&p, w.qin, w.dq, w.qm, w.qp, dx, dx, dx, dt, 1, nv);
  Delta d_trace = measure(b, 64);
  // faces: cmpflxm over x (3x2x2 faces) and unsplit's scaling of those faces
  b = opc::g;
  if (cmpflxm(&p, w.qm, w.qp, 1, 1, 3, 1, 2, 1, 2, w.fx, w.tx, 1, nv)) return 3;
  Delta d_riemann = measure(b, 12);
  CD* flux = (CD*)malloc(sizeof(CD) * 27 * NV * 3);
  CD* tmp = (CD*)malloc(sizeof(CD) * 27 * 2 * 3);
  b = opc::g;
  for (int i = 1; i <= 3; i++)
    for (int j = 1; j <= 2; j++)
      for (int k = 1; k <= 2; k++) {
        for (int ivar = 1; ivar <= NV; ivar++)
          flux[FI(nv, 0, i, j, k, ivar, 1)] = w.fx[QI(nv, 0, i, j, k, ivar)] * dt / dx;
        for (int ivar = 1; ivar <= 2; ivar++)
          tmp[TI(nv, 0, i, j, k, ivar, 1)] = w.tx[S6(nv, 0, i, j, k) + ST(nv) * (size_t)(ivar - 1)] * dt / dx;
      }
  Delta d_scale = measure(b, 12);
  // update of one cell: u = u + (f(i) - f(i+1)) per direction and variable
  b = opc::g;
  {
    CD u = 1.0, fl = 0.25, fr = 0.125;
    for (int d = 0; d < 3; d++)
      for (int v = 0; v < NV; v++) u = u + (fl - fr);
    (void)u;
  }
  Delta d_update = measure(b, 1);
  // cmpdt over 256 cells
  const int ncdt = 256;
  CD* uu = (CD*)malloc(sizeof(CD) * ncdt * NV);
  CD* gg = (CD*)calloc(ncdt * 3, sizeof(CD));
  for (int c = 0; c < ncdt; c++) {
    CD u[5];
    seeded_state(rng, u);
    for (int v = 0; v < NV; v++) uu[c + ncdt * v] = u[v];
  }
  b = opc::g;
  orc_cmpdt(&p, uu, gg, dx, ncdt, ncdt);
  Delta d_cmpdt = measure(b, ncdt);
  // what the reference executes per cell update: one dense periodic step
  // (courant_fine + godfine1 over every oct with its 6^3 stencil + update)
  const int n = 16;
  CD* ud = (CD*)malloc(sizeof(CD) * NV * n * n * n);
  for (int c = 0; c < n * n * n; c++) {
    CD u[5];
    seeded_state(rng, u);
    for (int v = 0; v < NV; v++) ud[c + (size_t)n * n * n * v] = u[v];
  }
  CD dt_out;
  b = opc::g;
  if (orc_dense_step(&p, ud, n, n, n, CD(1.0 / n), CD(1.0 / p.smallc), 0, 32, &dt_out)) return 4;
  Delta d_dense = measure(b, (double)n * n * n);
  Delta algo = sum({{&d_ctoprim, 1.0}, {&d_uslope, 1.0}, {&d_trace, 1.0}, {&d_riemann, 3.0}, {&d_scale, 3.0},
                    {&d_update, 1.0}, {&d_cmpdt, 1.0}});
  printf("{\n  \"riemann\": %d, \"slope_type\": %d, \"unit\": \"operations per cell (per face for riemann/scale)\",\n",
         riemann, slope_type);
  print("ctoprim_per_cell", d_ctoprim, true);
  print("uslope_per_cell", d_uslope, true);
  print("trace3d_per_cell", d_trace, true);
  print("riemann_per_face", d_riemann, true);
  print("flux_scale_per_face", d_scale, true);
  print("update_per_cell", d_update, true);
  print("cmpdt_per_cell", d_cmpdt, true);
  print("algorithmic_per_cell_update", algo, true);
  print("reference_dense_step_per_cell_update", d_dense, false);
  printf("}\n");
  work_free(&w);
  return 0;
}
