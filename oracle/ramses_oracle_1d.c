/*
 * ramses_oracle_1d.c -- TEST INFRASTRUCTURE ONLY. A CPU restatement of a
 * whole RAMSES hydro run built with NDIM=1 (nvar=3: rho, rho*u, E), one MPI
 * rank, hydro only: the initial refinement, the adaptive time loop with
 * subcycling, refinement and derefinement at every level step, wall and free
 * boundaries, and the snapshot's leaf cells at the first coarse step that
 * starts at t >= tout. It exists to pin the oracle's restatement against the
 * reference's own regression checksum (tests/hydro/sod-tube/sod-tube-ref.dat,
 * a 1D AMR run); the product library never links or calls it.
 *
 * Every routine follows the cited Fortran with NDIM=1 (twotondim = 2,
 * twondim = 2, threetondim = 3, nvector = 500), keeping the reference's
 * operation order. The Riemann solvers are the ones of the 3D restatement
 * (orc_riemann_face in ramses_oracle.c), called with zero transverse
 * velocities. Arrays are 1-based like the Fortran: cells 0..ncell with
 * icell = ncoarse + (ind-1)*ngridmax + igrid, grids 0..ngridmax; index 0 is
 * the reference's "absent" cell or grid and stays zero.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ramses_oracle.h"
#include "ramses_oracle_1d.h"

#define NV1 3      /* nvar = ndim + 2 */
#define NVEC 500   /* nvector (amr/amr_parameters.f90) */

static inline double fmaxd1(double a, double b) { return a > b ? a : (b > a ? b : a); }
static inline double fmind1(double a, double b) { return a < b ? a : (b < a ? b : a); }

typedef struct t1d {
  const orc1d_params *P;
  orc_params hp;
  int nx, ncoarse, ngridmax, ncell, nlevelmax, levelmin;
  int icoarse_min, icoarse_max;
  int nboundary, boundary_type[2], ibound_min[2], ibound_max[2];
  int32_t *son, *flag1, *flag2;  /* [ncell+1] */
  int32_t *father, *next, *prev; /* [ngridmax+1] */
  int32_t *nbor;                 /* [(ngridmax+1)*2] */
  double *xg;                    /* [ngridmax+1], coarse units */
  double *uold, *unew;           /* [(ncell+1)*3] */
  int headl[ORC_MAXLEVEL + 2], taill[ORC_MAXLEVEL + 2], numbl[ORC_MAXLEVEL + 2];
  int headb[2][ORC_MAXLEVEL + 2], tailb[2][ORC_MAXLEVEL + 2], numbb[2][ORC_MAXLEVEL + 2];
  int headf, tailf, numbf;
  double dtnew[ORC_MAXLEVEL + 2], dtold[ORC_MAXLEVEL + 2], t;
  int64_t nstep, nstep_coarse, nstep_coarse_old;
  int init;
  int err;
  char msg[160];
  int32_t *lst, *lst2;           /* scratch grid lists [ngridmax+1] */
} t1d;

#define CELL(T, g, ind) ((T)->ncoarse + ((ind) - 1) * (T)->ngridmax + (g))
#define UO(T, c, v) ((T)->uold[(size_t)(c) * NV1 + (v) - 1])
#define UN(T, c, v) ((T)->unew[(size_t)(c) * NV1 + (v) - 1])
#define NB(T, g, j) ((T)->nbor[(size_t)(g) * 2 + (j) - 1])

static void fail1(t1d *T, const char *m) {
  if (!T->err) { T->err = 1; snprintf(T->msg, sizeof T->msg, "%s", m); }
}

/* active(ilevel)%igrid and boundary(ibound,ilevel)%igrid: the level's linked
 * list in order (build_comm, amr/virtual_boundaries.f90) */
static int level_list(const t1d *T, int l, int32_t *out) {
  int n = 0;
  for (int g = T->headl[l]; g > 0 && n < T->numbl[l]; g = T->next[g]) out[n++] = g;
  return n;
}
static int bound_list(const t1d *T, int ib, int l, int32_t *out) {
  int n = 0;
  for (int g = T->headb[ib][l]; g > 0 && n < T->numbb[ib][l]; g = T->next[g]) out[n++] = g;
  return n;
}
static void list_append(t1d *T, int *head, int *tail, int *numb, int g) {
  if (*numb > 0) {
    T->next[g] = 0; T->prev[g] = *tail; T->next[*tail] = g; *tail = g; *numb += 1;
  } else {
    T->next[g] = 0; T->prev[g] = 0; *head = g; *tail = g; *numb = 1;
  }
}
static void list_remove(t1d *T, int *head, int *tail, int *numb, int g) {
  if (T->prev[g] != 0) {
    if (T->next[g] != 0) { T->next[T->prev[g]] = T->next[g]; T->prev[T->next[g]] = T->prev[g]; }
    else { T->next[T->prev[g]] = 0; *tail = T->prev[g]; }
  } else {
    if (T->next[g] != 0) { T->prev[T->next[g]] = 0; *head = T->next[g]; }
    else { *head = 0; *tail = 0; }
  }
  *numb -= 1;
}

/* ---- neighbour utilities: amr/nbors_utils.f90 (NDIM=1) ---- */
/* getnborgrids :530-555 */
static void getnborgrids(const t1d *T, int g, int igridn[3]) {
  igridn[0] = g;
  for (int j = 1; j <= 2; j++) igridn[j] = T->son[NB(T, g, j)];
}
/* getnborgrids_check (absent nbor: no grid) */
static void getnborgrids_check(const t1d *T, int g, int igridn[3]) {
  igridn[0] = g;
  for (int j = 1; j <= 2; j++) igridn[j] = NB(T, g, j) > 0 ? T->son[NB(T, g, j)] : 0;
}
/* getnborcells :363-399 with the NDIM=1 rows of ggg/hhh: left of cell 1 is
 * cell 2 of the left grid, right of cell 2 is cell 1 of the right grid */
static void getnborcells(const t1d *T, const int igridn[3], int ind, int icelln[3]) {
  static const int ggg[3][3] = {{0, 0, 0}, {0, 1, 0}, {0, 0, 2}}; /* [ind][in] */
  static const int hhh[3][3] = {{0, 0, 0}, {0, 2, 2}, {0, 1, 1}};
  for (int in = 1; in <= 2; in++) {
    int ig = ggg[ind][in], ih = hhh[ind][in];
    icelln[in] = igridn[ig] > 0 ? T->ncoarse + (ih - 1) * T->ngridmax + igridn[ig] : 0;
  }
}
/* get3cubefather :5-300: the three father-level cells around cell fcell of
 * level ilevel-1 (0 where the grid toward that side is absent) */
static void get3cubefather(const t1d *T, int fcell, int ilevel, int out[3]) {
  if (ilevel == 1) {
    int ix = fcell - 1;
    for (int i1 = 0; i1 <= 2; i1++) {
      int iix = ix + i1 - 1;
      if (iix < 0) iix = T->nx - 1;
      if (iix > T->nx - 1) iix = 0;
      out[i1] = 1 + iix;
    }
    return;
  }
  int pos = (fcell - T->ncoarse - 1) / T->ngridmax + 1;
  int g = fcell - T->ncoarse - (pos - 1) * T->ngridmax;
  int c = pos - 1;
  int side = T->son[NB(T, g, c ? 2 : 1)];
  for (int i1 = 0; i1 <= 2; i1++) {
    int cp = c + i1 - 1, gs = cp < 0 ? -1 : (cp > 1 ? 1 : 0);
    int gr = gs == 0 ? g : side;
    out[i1] = gr > 0 ? T->ncoarse + (cp - 2 * gs) * T->ngridmax + gr : 0;
  }
}
/* getnborfather :404-525: cell, then its left and right neighbours at the
 * same level, or the coarser neighbour cell nbor(grid,j) where absent */
static void getnborfather(const t1d *T, int cell, int ilevel, int f[3]) {
  f[0] = cell;
  if (ilevel == 1) {
    int ix = cell - 1;
    f[1] = ix > 0 ? cell - 1 : cell + (T->nx - 1);
    f[2] = ix < T->nx - 1 ? cell + 1 : cell - (T->nx - 1);
    return;
  }
  int pos = (cell - T->ncoarse - 1) / T->ngridmax + 1;
  int g = cell - T->ncoarse - (pos - 1) * T->ngridmax;
  int c = pos - 1;
  for (int j = 1; j <= 2; j++) {
    int inside = j == 2 ? (c == 0) : (c == 1);
    int gg = inside ? g : T->son[NB(T, g, j)];
    int icell = gg > 0 ? T->ncoarse + (1 - c) * T->ngridmax + gg : 0;
    f[j] = icell > 0 ? icell : NB(T, g, j);
  }
}

/* ---- interpol_hydro, NDIM=1, interpol_var = 0: hydro/interpol_hydro.f90:268-637 ---- */
static int interpol_hydro1(const t1d *T, double u1[3][NV1], double u2[2][NV1]) {
  const int itype = T->hp.interpol_type;
  static const double xc[2] = {-0.5, 0.5};
  if (T->hp.interpol_var != 0 || itype < 0 || itype > 3) return -1;
  for (int ivar = 1; ivar <= NV1; ivar++) {
    double a0 = u1[0][ivar - 1], a1 = u1[1][ivar - 1], a2 = u1[2][ivar - 1], w = 0.0;
    if (itype == 1) { /* compute_limiter_minmod :449-476 */
      double dl = 0.5 * (a2 - a0), dr = 0.5 * (a0 - a1);
      w = dl * dr <= 0.0 ? 0.0 : fmind1(fabs(dl), fabs(dr)) * dl / fabs(dl);
    } else if (itype == 2) { /* compute_limiter_central :481-613 */
      w = 0.25 * (a2 - a1);
      double ac[2];
      for (int ind = 0; ind < 2; ind++) ac[ind] = a0 + 2.0 * w * xc[ind];
      double corner = fmaxd1(ac[0], ac[1]), kernel = fmaxd1(a1, a2);
      double dk = a0 - kernel, dc = a0 - corner, maxl = 0.0, minl = 0.0;
      if (dk * dc > 0.0) maxl = fmind1(1.0, dk / dc);
      corner = fmind1(ac[0], ac[1]);
      kernel = fmind1(a1, a2);
      dk = a0 - kernel; dc = a0 - corner;
      if (dk * dc > 0.0) minl = fmind1(1.0, dk / dc);
      w = w * fmind1(minl, maxl);
    } else if (itype == 3) { /* compute_central :618-637 */
      w = 0.25 * (a2 - a1);
    }
    for (int ind = 0; ind < 2; ind++) u2[ind][ivar - 1] = a0 + w * xc[ind];
  }
  return 0;
}

/* ---- initial conditions: hydro/condinit.f90, region_condinit ('square') ---- */
static void condinit1(const t1d *T, double x, double u[NV1]) {
  const orc1d_params *P = T->P;
  const double gamma = T->hp.gamma;
  double q[3] = {T->hp.smallr, 0.0, T->hp.smallr * (T->hp.smallc * T->hp.smallc) / gamma};
  for (int k = 0; k < P->nregion; k++) {
    double en = P->exp_region[k];
    double xn = 2.0 * fabs(x - P->x_center[k]) / P->length_x[k];
    double r = en < 10 ? pow(pow(xn, en) + 0.0 + 0.0, 1.0 / en) : fmaxd1(fmaxd1(xn, 0.0), 0.0);
    if (r < 1.0) { q[0] = P->d_region[k]; q[1] = P->u_region[k]; q[2] = P->p_region[k]; }
  }
  u[0] = q[0];
  u[1] = q[0] * q[1];
  u[2] = 0.0;
  u[2] = u[2] + 0.5 * q[0] * (q[1] * q[1]);
  u[2] = u[2] + q[2] / (gamma - 1.0);
}

static double scale_of(const t1d *T) { return T->P->boxlen / (double)(T->icoarse_max - T->icoarse_min + 1); }

/* init_flow_fine (hydro/init_flow_fine.f90:418-456): condinit at the cell centres */
static void init_flow_fine(t1d *T, int ilevel) {
  int n = level_list(T, ilevel, T->lst);
  if (n == 0) return;
  double dx = pow(0.5, ilevel), scale = scale_of(T), skip = (double)T->icoarse_min;
  for (int ind = 1; ind <= 2; ind++) {
    double xc = ((double)(ind - 1) - 0.5) * dx;
    for (int i = 0; i < n; i++) {
      double x = (T->xg[T->lst[i]] + xc - skip) * scale, u[NV1];
      condinit1(T, x, u);
      for (int v = 1; v <= NV1; v++) UO(T, CELL(T, T->lst[i], ind), v) = u[v - 1];
    }
  }
}

/* upload_fine / upl (hydro/interpol_hydro.f90:5-150), interpol_var = 0 */
static void upload_fine(t1d *T, int ilevel) {
  if (ilevel == T->nlevelmax) return;
  int n = level_list(T, ilevel, T->lst);
  for (int ind = 1; ind <= 2; ind++)
    for (int i = 0; i < n; i++) {
      int cell = CELL(T, T->lst[i], ind), gs = T->son[cell];
      if (gs <= 0) continue;
      double getx = 0.0;
      for (int is = 1; is <= 2; is++) getx = getx + fmaxd1(UO(T, CELL(T, gs, is), 1), T->hp.smallr);
      UO(T, cell, 1) = getx / 2.0;
      for (int ivar = 2; ivar <= NV1; ivar++) {
        getx = 0.0;
        for (int is = 1; is <= 2; is++) getx = getx + UO(T, CELL(T, gs, is), ivar);
        UO(T, cell, ivar) = getx / 2.0;
      }
    }
}

/* make_boundary_hydro (hydro/hydro_boundary.f90:5-260), NDIM=1: walls
 * (types 1, 2) mirror the reference grid with u negated, free boundaries
 * (11, 12) copy the adjacent cell with E - ekin + ekin recomputed */
static void make_boundary_hydro(t1d *T, int ilevel) {
  for (int ib = 0; ib < T->nboundary; ib++) {
    const int bt = T->boundary_type[ib], dir = bt - 10 * (bt / 10);
    const int inbor = dir == 1 ? 2 : 1;
    int ind_ref[3];
    if (bt / 10 == 0) { ind_ref[1] = 2; ind_ref[2] = 1; }
    else if (dir == 1) { ind_ref[1] = 1; ind_ref[2] = 1; }
    else { ind_ref[1] = 2; ind_ref[2] = 2; }
    int n = bound_list(T, ib, ilevel, T->lst);
    for (int i0 = 0; i0 < n; i0 += NVEC) {
      int ng = n - i0 < NVEC ? n - i0 : NVEC;
      for (int ind = 1; ind <= 2; ind++)
        for (int i = 0; i < ng; i++) {
          int g = T->lst[i0 + i], gref = T->son[NB(T, g, inbor)];
          if (gref <= 0) { fail1(T, "make_boundary_hydro: boundary grid without a reference grid"); return; }
          int c = CELL(T, g, ind), cr = CELL(T, gref, ind_ref[ind]);
          double uu[NV1];
          for (int v = 1; v <= NV1; v++) uu[v - 1] = UO(T, cr, v);
          if (bt / 10 == 0) {
            UO(T, c, 1) = uu[0];
            UO(T, c, 2) = uu[1] * -1.0;
            UO(T, c, 3) = uu[2];
          } else {
            double d = fmaxd1(uu[0], T->hp.smallr), vv = uu[1] / d;
            uu[2] = uu[2] - 0.5 * d * (vv * vv);
            for (int v = 1; v <= NV1; v++) UO(T, c, v) = uu[v - 1];
            d = fmaxd1(UO(T, c, 1), T->hp.smallr);
            vv = UO(T, c, 2) / d;
            UO(T, c, 3) = UO(T, c, 3) + 0.5 * d * (vv * vv);
          }
        }
    }
  }
}

/* ---- flags: amr/flag_utils.f90, amr/virtual_boundaries.f90 ---- */
/* make_boundary_flag (virtual_boundaries.f90) */
static void make_boundary_flag(t1d *T, int ilevel) {
  for (int ib = 0; ib < T->nboundary; ib++) {
    const int bt = T->boundary_type[ib], dir = bt - 10 * (bt / 10);
    const int inbor = dir == 1 ? 2 : 1;
    int ind_ref[3];
    if (bt / 10 == 0) { ind_ref[1] = 2; ind_ref[2] = 1; }
    else if (dir == 1) { ind_ref[1] = 1; ind_ref[2] = 1; }
    else { ind_ref[1] = 2; ind_ref[2] = 2; }
    int n = bound_list(T, ib, ilevel, T->lst2);
    for (int ind = 1; ind <= 2; ind++)
      for (int i = 0; i < n; i++) {
        int g = T->lst2[i], gref = T->son[NB(T, g, inbor)];
        T->flag1[CELL(T, g, ind)] = T->flag1[T->ncoarse + (ind_ref[ind] - 1) * T->ngridmax + gref];
      }
  }
}

/* init_flag :111-163 with test_flag :168-208 */
static void init_flag(t1d *T, int ilevel) {
  int n = level_list(T, ilevel, T->lst);
  for (int ind = 1; ind <= 2; ind++)
    for (int i = 0; i < n; i++) T->flag1[CELL(T, T->lst[i], ind)] = 0;
  if (ilevel >= T->levelmin) {
    for (int ind = 1; ind <= 2; ind++)
      for (int i = 0; i < n; i++) {
        int gs = T->son[CELL(T, T->lst[i], ind)], ok = 0;
        if (gs > 0)
          for (int is = 1; is <= 2; is++) {
            int cs = CELL(T, gs, is);
            ok = ok || T->son[cs] > 0;
            ok = ok || T->flag1[cs] == 1;
          }
        if (ok) T->flag1[CELL(T, T->lst[i], ind)] = 1;
      }
  } else {
    for (int ind = 1; ind <= 2; ind++)
      for (int i = 0; i < n; i++) T->flag1[CELL(T, T->lst[i], ind)] = 1;
  }
  make_boundary_flag(T, ilevel);
}

/* smooth_fine :555-638 with count_nbors :643-677, n_nbor(1) = 1 */
static void smooth_fine(t1d *T, int ilevel) {
  if (ilevel == T->nlevelmax) return;
  int n = level_list(T, ilevel, T->lst);
  if (n == 0) return;
  T->flag1[0] = 0;
  for (int ind = 1; ind <= 2; ind++)
    for (int i = 0; i < n; i++) T->flag2[CELL(T, T->lst[i], ind)] = 0;
  for (int i = 0; i < n; i++) {
    int igridn[3];
    getnborgrids(T, T->lst[i], igridn);
    for (int ind = 1; ind <= 2; ind++) {
      int indn[3];
      getnborcells(T, igridn, ind, indn);
      int cnt = T->flag1[indn[1]] + T->flag1[indn[2]];
      if (cnt >= 1) T->flag2[CELL(T, T->lst[i], ind)] = 1;
    }
  }
  for (int ind = 1; ind <= 2; ind++)
    for (int i = 0; i < n; i++) {
      int c = CELL(T, T->lst[i], ind);
      if (T->flag1[c] == 1) T->flag2[c] = 0;
      if (T->flag2[c] == 1) T->flag1[c] = 1;
    }
  make_boundary_flag(T, ilevel);
}

/* hydro_refine (hydro/godunov_utils.f90:125-263), nvar = 3, one direction */
static int hydro_refine1d(const t1d *T, double g[NV1], double m[NV1], double d[NV1]) {
  const orc_refine *r = &T->P->refine;
  const double gamma = T->hp.gamma, half = 0.5, one = 1.0, zero = 0.0;
  g[0] = fmaxd1(g[0], T->hp.smallr);
  m[0] = fmaxd1(m[0], T->hp.smallr);
  d[0] = fmaxd1(d[0], T->hp.smallr);
  g[1] = g[1] / g[0];
  m[1] = m[1] / m[0];
  d[1] = d[1] / d[0];
  double eking = zero + half * g[0] * (g[1] * g[1]);
  double ekinm = zero + half * m[0] * (m[1] * m[1]);
  double ekind = zero + half * d[0] * (d[1] * d[1]);
  g[2] = (gamma - one) * (g[2] - eking);
  m[2] = (gamma - one) * (m[2] - ekinm);
  d[2] = (gamma - one) * (d[2] - ekind);
  int ok = 0;
  if (r->err_grad_d >= 0.) {
    double error = 2.0 * fmaxd1(fabs((d[0] - m[0]) / (d[0] + m[0] + r->floor_d)),
                                fabs((m[0] - g[0]) / (m[0] + g[0] + r->floor_d)));
    ok = ok || error > r->err_grad_d;
  }
  if (r->err_grad_p >= 0.) {
    double error = 2.0 * fmaxd1(fabs((d[2] - m[2]) / (d[2] + m[2] + r->floor_p)),
                                fabs((m[2] - g[2]) / (m[2] + g[2] + r->floor_p)));
    ok = ok || error > r->err_grad_p;
  }
  if (r->err_grad_u >= 0.) {
    double f2 = r->floor_u * r->floor_u;
    double cg = sqrt(fmaxd1(gamma * g[2] / g[0], f2));
    double cm = sqrt(fmaxd1(gamma * m[2] / m[0], f2));
    double cd = sqrt(fmaxd1(gamma * d[2] / d[0], f2));
    double error = 2.0 * fmaxd1(fabs((d[1] - m[1]) / (cd + cm + fabs(d[1]) + fabs(m[1]) + r->floor_u)),
                                fabs((m[1] - g[1]) / (cm + cg + fabs(m[1]) + fabs(g[1]) + r->floor_u)));
    ok = ok || error > r->err_grad_u;
  }
  return ok;
}

/* userflag_fine :281-427 (no geometry or Poisson criterion) -> hydro_flag
 * (hydro/hydro_flag.f90:1-180) */
static void userflag_fine(t1d *T, int ilevel) {
  if (ilevel == T->nlevelmax) return;
  int n = level_list(T, ilevel, T->lst);
  if (n == 0) return;
  const orc_refine *r = &T->P->refine;
  if (!(r->err_grad_d == -1.0 && r->err_grad_p == -1.0 && r->err_grad_u == -1.0)) {
    for (int i = 0; i < n; i++) {
      int g = T->lst[i], igridn[3];
      getnborgrids(T, g, igridn);
      for (int ind = 1; ind <= 2; ind++) {
        int cell = CELL(T, g, ind), indn[3];
        getnborcells(T, igridn, ind, indn);
        for (int j = 1; j <= 2; j++)
          if (indn[j] == 0) indn[j] = NB(T, g, j);
        double ug[NV1], um[NV1], ud[NV1];
        for (int v = 1; v <= NV1; v++) {
          ug[v - 1] = UO(T, indn[1], v);
          um[v - 1] = UO(T, cell, v);
          ud[v - 1] = UO(T, indn[2], v);
        }
        if (hydro_refine1d(T, ug, um, ud)) T->flag1[cell] = 1;
      }
    }
  }
  make_boundary_flag(T, ilevel);
}

/* ensure_ref_rules :213-276: unflag the cells of grids whose father's three
 * neighbour cells are not all refined */
static void ensure_ref_rules(t1d *T, int ilevel) {
  int n = level_list(T, ilevel, T->lst);
  for (int i = 0; i < n; i++) {
    int g = T->lst[i], nb[3], ok = 1;
    get3cubefather(T, T->father[g], ilevel, nb);
    for (int k = 0; k < 3; k++) {
      if (nb[k] == 0) ok = 0;
      if (nb[k] > 0 && T->son[nb[k]] == 0) ok = 0;
    }
    if (!ok)
      for (int ind = 1; ind <= 2; ind++) T->flag1[CELL(T, g, ind)] = 0;
  }
  make_boundary_flag(T, ilevel);
}

/* flag_fine :57-106 */
static void flag_fine(t1d *T, int ilevel, int icount) {
  if (ilevel == T->nlevelmax) return;
  if (T->numbl[ilevel] == 0) return;
  init_flag(T, ilevel);
  if (ilevel < T->levelmin) return;
  smooth_fine(T, ilevel);
  userflag_fine(T, ilevel);
  for (int ie = 1; ie <= T->P->nexpand; ie++) smooth_fine(T, ilevel);
  if (ilevel > T->levelmin && icount < T->P->nsubcycle[ilevel - 1]) ensure_ref_rules(T, ilevel);
}

/* flag_coarse :22-52 with make_boundary_coarse (virtual_boundaries.f90) */
static void flag_coarse(t1d *T) {
  for (int c = 0; c <= T->ncoarse; c++) T->flag1[c] = 0;
  for (int ix = T->icoarse_min; ix <= T->icoarse_max; ix++) T->flag1[1 + ix] = 1;
  for (int ib = 0; ib < T->nboundary; ib++) {
    int dir = T->boundary_type[ib] - 10 * (T->boundary_type[ib] / 10), iskip = dir == 1 ? +1 : -1;
    for (int i = T->ibound_min[ib]; i <= T->ibound_max[ib]; i++) T->flag1[1 + i] = T->flag1[1 + i + iskip];
  }
}

/* ---- refinement: amr/refine_utils.f90 ---- */
/* make_grid_coarse :165-327 */
static void make_grid_coarse(t1d *T, int ind_cell, int ib, int boundary_region) {
  int g = T->headf;
  T->headf = T->next[T->headf];
  T->numbf--;
  int ix = ind_cell - 1;
  T->xg[g] = (double)ix + 0.5;
  T->son[ind_cell] = g;
  T->father[g] = ind_cell;
  NB(T, g, 1) = 1 + (ix > 0 ? ix - 1 : T->nx - 1);
  NB(T, g, 2) = 1 + (ix < T->nx - 1 ? ix + 1 : 0);
  if (boundary_region) list_append(T, &T->headb[ib][1], &T->tailb[ib][1], &T->numbb[ib][1], g);
  else list_append(T, &T->headl[1], &T->taill[1], &T->numbl[1], g);
}

/* kill_grid :953-1158 */
static void kill_grid(t1d *T, int ind_cell, int ilevel, int ib, int boundary_region) {
  int g = T->son[ind_cell];
  T->son[ind_cell] = 0;
  if (boundary_region) list_remove(T, &T->headb[ib][ilevel], &T->tailb[ib][ilevel], &T->numbb[ib][ilevel], g);
  else list_remove(T, &T->headl[ilevel], &T->taill[ilevel], &T->numbl[ilevel], g);
  T->xg[g] = 0.0;
  T->father[g] = 0;
  NB(T, g, 1) = 0;
  NB(T, g, 2) = 0;
  for (int ind = 1; ind <= 2; ind++) {
    int c = CELL(T, g, ind);
    T->son[c] = 0; T->flag1[c] = 0; T->flag2[c] = 0;
    for (int v = 1; v <= NV1; v++) { UO(T, c, v) = 0.0; UN(T, c, v) = 0.0; }
  }
  T->next[T->tailf] = g;
  T->prev[g] = T->tailf;
  T->next[g] = 0;
  T->tailf = g;
  T->numbf++;
}

/* refine_coarse :25-160 with authorize_coarse */
static void refine_coarse(t1d *T) {
  T->flag2[0] = 0;
  for (int c = 1; c <= T->nx; c++) T->flag2[c] = 1;
  for (int ix = T->icoarse_min; ix <= T->icoarse_max; ix++) {
    int c = 1 + ix;
    if (T->flag2[c] == 1 && T->flag1[c] == 1 && T->son[c] == 0) make_grid_coarse(T, c, 0, 0);
  }
  for (int ib = 0; ib < T->nboundary; ib++)
    for (int i = T->ibound_min[ib]; i <= T->ibound_max[ib]; i++) {
      int c = 1 + i;
      if (T->flag2[c] == 1 && T->flag1[c] == 1 && T->son[c] == 0) make_grid_coarse(T, c, ib, 1);
    }
  for (int ix = T->icoarse_min; ix <= T->icoarse_max; ix++) {
    int c = 1 + ix;
    if (T->flag1[c] == 0 && T->son[c] > 0) kill_grid(T, c, 1, 0, 0);
  }
  for (int ib = 0; ib < T->nboundary; ib++)
    for (int i = T->ibound_min[ib]; i <= T->ibound_max[ib]; i++) {
      int c = 1 + i;
      if (T->flag1[c] == 0 && T->son[c] > 0) kill_grid(T, c, 1, ib, 1);
    }
}

/* authorize_fine (virtual_boundaries.f90:34-311, one CPU) with
 * init_boundary_fine: the boundary cells next to the box may be refined */
static void authorize_fine(t1d *T, int ilevel) {
  if (ilevel == T->nlevelmax) return;
  int n = level_list(T, ilevel, T->lst);
  for (int ind = 1; ind <= 2; ind++)
    for (int i = 0; i < n; i++) T->flag2[CELL(T, T->lst[i], ind)] = 1;
  T->flag2[0] = 0;
  for (int ib = 0; ib < T->nboundary; ib++) {
    int nb = bound_list(T, ib, ilevel, T->lst2);
    for (int ind = 1; ind <= 2; ind++)
      for (int i = 0; i < nb; i++) T->flag2[CELL(T, T->lst2[i], ind)] = 0;
  }
  /* init_boundary_fine */
  for (int ib = 0; ib < T->nboundary; ib++) {
    int nb = bound_list(T, ib, ilevel, T->lst2);
    for (int ind = 1; ind <= 2; ind++)
      for (int i = 0; i < nb; i++) T->flag2[CELL(T, T->lst2[i], ind)] = 0;
  }
  T->flag2[0] = 0;
  for (int ib = 0; ib < T->nboundary; ib++) {
    int nb = bound_list(T, ib, ilevel, T->lst2);
    for (int ind = 1; ind <= 2; ind++)
      for (int i = 0; i < nb; i++) T->flag1[CELL(T, T->lst2[i], ind)] = 0;
  }
  for (int ib = 0; ib < T->nboundary; ib++) {
    int nb = bound_list(T, ib, ilevel, T->lst2);
    for (int i = 0; i < nb; i++) {
      int igridn[3];
      getnborgrids_check(T, T->lst2[i], igridn);
      for (int ind = 1; ind <= 2; ind++) {
        int indn[3];
        getnborcells(T, igridn, ind, indn);
        if (T->flag2[indn[1]] + T->flag2[indn[2]] >= 1) T->flag1[CELL(T, T->lst2[i], ind)] = 1;
      }
    }
  }
  for (int ib = 0; ib < T->nboundary; ib++) {
    int nb = bound_list(T, ib, ilevel, T->lst2);
    for (int ind = 1; ind <= 2; ind++)
      for (int i = 0; i < nb; i++)
        if (T->flag1[CELL(T, T->lst2[i], ind)] == 1) T->flag2[CELL(T, T->lst2[i], ind)] = 1;
  }
  make_boundary_flag(T, ilevel);
}

/* make_grid_fine :590-948 for one new grid in cell ind_cell (cell ind of
 * grid ind_grid, level ilevel-1) */
static void make_grid_fine(t1d *T, int ind_grid, int ind_cell, int ind, int ilevel, int ib,
                           int boundary_region) {
  if (T->numbf <= 0) { fail1(T, "make_grid_fine: no more free memory (ngridmax)"); return; }
  int g = T->headf;
  T->headf = T->next[T->headf];
  T->numbf--;
  double dx = pow(0.5, ilevel - 1);
  double xc = ((double)(ind - 1) - 0.5) * dx;
  T->xg[g] = T->xg[ind_grid] + xc;
  T->son[ind_cell] = g;
  T->father[g] = ind_cell;
  int igridn[3], indn[3];
  getnborgrids(T, ind_grid, igridn);
  getnborcells(T, igridn, ind, indn);
  for (int j = 1; j <= 2; j++) {
    NB(T, g, j) = indn[j];
    if (indn[j] == 0 && !boundary_region) fail1(T, "make_grid_fine: father cell without a same-level neighbour");
  }
  for (int ind2 = 1; ind2 <= 2; ind2++) {
    int c = CELL(T, g, ind2);
    T->son[c] = 0; T->flag1[c] = 0; T->flag2[c] = 0;
  }
  if (boundary_region) list_append(T, &T->headb[ib][ilevel], &T->tailb[ib][ilevel], &T->numbb[ib][ilevel], g);
  else list_append(T, &T->headl[ilevel], &T->taill[ilevel], &T->numbl[ilevel], g);
  if (!T->init) {
    int fz[3] = {T->father[g], NB(T, g, 1), NB(T, g, 2)};
    double u1[3][NV1], u2[2][NV1];
    for (int j = 0; j < 3; j++)
      for (int v = 1; v <= NV1; v++) u1[j][v - 1] = fz[j] > 0 ? UO(T, fz[j], v) : 0.0;
    if (interpol_hydro1(T, u1, u2)) { fail1(T, "interpol_hydro: unsupported interpol_var/interpol_type"); return; }
    for (int ind2 = 1; ind2 <= 2; ind2++)
      for (int v = 1; v <= NV1; v++) UO(T, CELL(T, g, ind2), v) = u2[ind2 - 1][v - 1];
  }
}

/* refine_fine :332-585 (one CPU): create the sons of flagged cells of the
 * active grids, then of the boundary grids; then kill the sons of unflagged
 * cells */
static void refine_fine(t1d *T, int ilevel) {
  if (ilevel == T->nlevelmax) return;
  if (T->numbl[ilevel] == 0) return;
  authorize_fine(T, ilevel);
  for (int pass = 0; pass <= T->nboundary; pass++) {
    int ib = pass - 1, n = pass == 0 ? level_list(T, ilevel, T->lst2) : bound_list(T, ib, ilevel, T->lst2);
    for (int i0 = 0; i0 < n; i0 += NVEC) {
      int ng = n - i0 < NVEC ? n - i0 : NVEC;
      for (int ind = 1; ind <= 2; ind++)
        for (int i = 0; i < ng; i++) {
          int g = T->lst2[i0 + i], c = CELL(T, g, ind);
          if (T->flag2[c] == 1 && T->flag1[c] == 1 && T->son[c] == 0)
            make_grid_fine(T, g, c, ind, ilevel + 1, ib, pass > 0);
        }
    }
  }
  for (int pass = 0; pass <= T->nboundary; pass++) {
    int ib = pass - 1, n = pass == 0 ? level_list(T, ilevel, T->lst2) : bound_list(T, ib, ilevel, T->lst2);
    for (int i0 = 0; i0 < n; i0 += NVEC) {
      int ng = n - i0 < NVEC ? n - i0 : NVEC;
      for (int ind = 1; ind <= 2; ind++)
        for (int i = 0; i < ng; i++) {
          int c = CELL(T, T->lst2[i0 + i], ind);
          if (T->flag1[c] == 0 && T->son[c] > 0) kill_grid(T, c, ilevel + 1, ib, pass > 0);
        }
    }
  }
}

/* ---- hydro step ---- */
/* set_unew / set_uold (hydro/godunov_fine.f90:40-232, no pressure_fix) */
static void set_unew(t1d *T, int ilevel) {
  int n = level_list(T, ilevel, T->lst);
  for (int ind = 1; ind <= 2; ind++)
    for (int v = 1; v <= NV1; v++)
      for (int i = 0; i < n; i++) UN(T, CELL(T, T->lst[i], ind), v) = UO(T, CELL(T, T->lst[i], ind), v);
}
static void set_uold(t1d *T, int ilevel) {
  int n = level_list(T, ilevel, T->lst);
  for (int ind = 1; ind <= 2; ind++)
    for (int v = 1; v <= NV1; v++)
      for (int i = 0; i < n; i++) UO(T, CELL(T, T->lst[i], ind), v) = UN(T, CELL(T, T->lst[i], ind), v);
}

/* courant_fine (hydro/courant_fine.f90:1-159) with cmpdt
 * (hydro/godunov_utils.f90:5-120), NDIM=1, no gravity */
static void courant_fine(t1d *T, int ilevel) {
  const double gamma = T->hp.gamma, smallc = T->hp.smallc, C = T->hp.courant_factor;
  const double half = 0.5, one = 1.0, two = 2.0, smallp = smallc * smallc / gamma;
  double dx = pow(0.5, ilevel) * scale_of(T);
  double dt_loc = T->dtnew[ilevel];
  int n = level_list(T, ilevel, T->lst);
  for (int i0 = 0; i0 < n; i0 += NVEC) {
    int ng = n - i0 < NVEC ? n - i0 : NVEC;
    for (int ind = 1; ind <= 2; ind++) {
      int nleaf = 0;
      double dt = C * dx / smallc;
      for (int i = 0; i < ng; i++) {
        int c = CELL(T, T->lst[i0 + i], ind);
        if (T->son[c] != 0) continue;
        nleaf++;
        double d = fmaxd1(UO(T, c, 1), T->hp.smallr);
        double v = UO(T, c, 2) / d;
        double e = UO(T, c, 3) - half * d * (v * v);
        double cs = fmaxd1((gamma - one) * e, d * smallp);
        cs = gamma * cs;
        cs = sqrt(cs / d);
        cs = 1.0 * cs;
        cs = cs + fabs(v);
        double g0 = 0.0 + fabs(0.0);
        g0 = g0 * dx / (cs * cs);
        g0 = fmaxd1(g0, 0.0001);
        double dtcell = dx / cs * (sqrt(one + two * C * g0) - one) / g0;
        dt = fmind1(dt, dtcell);
      }
      if (nleaf > 0) dt_loc = fmind1(dt_loc, dt);
    }
  }
  T->dtnew[ilevel] = fmind1(T->dtnew[ilevel], dt_loc);
}

/* unsplit (hydro/umuscl.f90:22-171), NDIM=1, on one grid's stencil
 * u[i3][v], i3 = -1..4 stored at i3+1: ctoprim :861-965, uslope :970-1040,
 * trace1d :176-290, cmpflxm :714-856; flux[i][v] for faces i = 1..3 */
static int unsplit1(t1d *T, double u[6][NV1], double dx, double dt, double flux[4][NV1]) {
  const double gamma = T->hp.gamma, smallr = T->hp.smallr, half = 0.5, one = 1.0;
  const double smalle = T->hp.smallc * T->hp.smallc / gamma / (gamma - one), dtxhalf = dt * half;
  double q[6][NV1], dq[6][NV1], qm[6][NV1], qp[6][NV1];
  for (int i = 0; i < 6; i++) {
    q[i][0] = fmaxd1(u[i][0], smallr);
    double oneoverrho = one / q[i][0];
    q[i][1] = u[i][1] * oneoverrho;
    double eken = half * q[i][1] * q[i][1];
    double erad = 0.0;
    double eint = fmaxd1(u[i][2] * oneoverrho - eken - erad, smalle);
    q[i][2] = (gamma - one) * q[i][0] * eint;
    q[i][1] = q[i][1] + 0.0 * dtxhalf;
  }
  const int st = T->hp.slope_type;
  for (int i = 1; i <= 4; i++) /* cells 0..3 */
    for (int v = 0; v < NV1; v++) {
      if (st == 0) { dq[i][v] = 0.0; continue; }
      if (st < 1 || st > 3) return -1;
      const double k = (double)(st < 2 ? st : 2);
      double dlft = k * (q[i][v] - q[i - 1][v]);
      double drgt = k * (q[i + 1][v] - q[i][v]);
      double dcen = half * (dlft + drgt) / k;
      double dsgn = copysign(one, dcen);
      double slop = fmind1(fabs(dlft), fabs(drgt));
      double dlim = slop;
      if ((dlft * drgt) <= 0.0) dlim = 0.0;
      dq[i][v] = dsgn * fmind1(dlim, fabs(dcen));
    }
  const double dtdx = dt / dx;
  for (int i = 1; i <= 4; i++) {
    double r = q[i][0], uu = q[i][1], p = q[i][2];
    double drx = dq[i][0], dux = dq[i][1], dpx = dq[i][2];
    double sr0 = -uu * drx - (dux) * r;
    double sp0 = -uu * dpx - (dux) * gamma * p;
    double su0 = -uu * dux - (dpx) / r;
    qp[i][0] = r - half * drx + sr0 * dtdx * half;
    qp[i][1] = uu - half * dux + su0 * dtdx * half;
    qp[i][2] = p - half * dpx + sp0 * dtdx * half;
    if (qp[i][0] < smallr) qp[i][0] = r;
    qm[i][0] = r + half * drx + sr0 * dtdx * half;
    qm[i][1] = uu + half * dux + su0 * dtdx * half;
    qm[i][2] = p + half * dpx + sp0 * dtdx * half;
    if (qm[i][0] < smallr) qm[i][0] = r;
  }
  for (int f = 1; f <= 3; f++) { /* face f between cells f-1 and f (stored f, f+1) */
    double ql[5] = {qm[f][0], qm[f][1], qm[f][2], 0.0, 0.0};
    double qr[5] = {qp[f + 1][0], qp[f + 1][1], qp[f + 1][2], 0.0, 0.0};
    double fg[6];
    if (orc_riemann_face(&T->hp, ql, qr, fg)) return -2;
    flux[f][0] = fg[0] * dt / dx;
    flux[f][1] = fg[1] * dt / dx;
    flux[f][2] = fg[2] * dt / dx;
  }
  return 0;
}

/* godunov_fine / godfine1 (hydro/godunov_fine.f90:5-35, 486-908), NDIM=1 */
static void godunov_fine(t1d *T, int ilevel) {
  const double oneontwotondim = 1.0 / 2.0;
  double dx = pow(0.5, ilevel) * scale_of(T), dt = T->dtnew[ilevel];
  int n = level_list(T, ilevel, T->lst);
  static double flux[NVEC][4][NV1];
  for (int i0 = 0; i0 < n; i0 += NVEC) {
    int ng = n - i0 < NVEC ? n - i0 : NVEC;
    for (int i = 0; i < ng; i++) {
      int g = T->lst[i0 + i], nbf[3];
      get3cubefather(T, T->father[g], ilevel, nbf);
      double uloc[6][NV1];
      int okc[6];
      for (int i1 = 0; i1 <= 2; i1++) {
        int gn = nbf[i1] > 0 ? T->son[nbf[i1]] : 0;
        double u2[2][NV1];
        if (gn <= 0) {
          if (nbf[i1] <= 0) { fail1(T, "godunov_fine: missing father neighbour"); return; }
          int f3[3];
          getnborfather(T, nbf[i1], ilevel, f3);
          double u1[3][NV1];
          for (int j = 0; j < 3; j++)
            for (int v = 1; v <= NV1; v++) u1[j][v - 1] = UO(T, f3[j], v);
          if (interpol_hydro1(T, u1, u2)) { fail1(T, "interpol_hydro: unsupported options"); return; }
        }
        for (int i2 = 0; i2 <= 1; i2++) {
          int i3 = 1 + 2 * (i1 - 1) + i2; /* -1..4 */
          if (gn > 0) {
            int c = CELL(T, gn, 1 + i2);
            for (int v = 1; v <= NV1; v++) uloc[i3 + 1][v - 1] = UO(T, c, v);
            okc[i3 + 1] = T->son[c] > 0;
          } else {
            for (int v = 1; v <= NV1; v++) uloc[i3 + 1][v - 1] = u2[i2][v - 1];
            okc[i3 + 1] = 0;
          }
        }
      }
      if (unsplit1(T, uloc, dx, dt, flux[i])) { fail1(T, "unsplit: unsupported slope_type or Riemann solver"); return; }
      for (int f = 1; f <= 3; f++) /* refined-face zeroing :720-747 */
        if (okc[f - 1 + 1] || okc[f + 1])
          for (int v = 0; v < NV1; v++) flux[i][f][v] = 0.0;
    }
    for (int i2 = 0; i2 <= 1; i2++) /* conservative update :751-792 */
      for (int v = 1; v <= NV1; v++)
        for (int i = 0; i < ng; i++) {
          int c = CELL(T, T->lst[i0 + i], 1 + i2), i3 = 1 + i2;
          UN(T, c, v) = UN(T, c, v) + (flux[i][i3][v - 1] - flux[i][i3 + 1][v - 1]);
        }
    /* fine -> coarse corrections :798-908 */
    for (int v = 1; v <= NV1; v++)
      for (int i = 0; i < ng; i++) {
        int g = T->lst[i0 + i], nc = NB(T, g, 1);
        if (T->son[nc] == 0) UN(T, nc, v) = UN(T, nc, v) - flux[i][1][v - 1] * oneontwotondim;
      }
    for (int v = 1; v <= NV1; v++)
      for (int i = 0; i < ng; i++) {
        int g = T->lst[i0 + i], nc = NB(T, g, 2);
        if (T->son[nc] == 0) UN(T, nc, v) = UN(T, nc, v) + flux[i][3][v - 1] * oneontwotondim;
      }
  }
}

/* ---- drivers ---- */
static void flag_all(t1d *T) { /* flag (flag_utils.f90:5-17) */
  for (int l = T->nlevelmax - 1; l >= 1; l--) flag_fine(T, l, 2);
  flag_coarse(T);
}
static void refine_all(t1d *T) { /* refine (refine_utils.f90:1-20) */
  refine_coarse(T);
  for (int l = 1; l <= T->nlevelmax - 1; l++) refine_fine(T, l);
}
static void init_flow(t1d *T) { /* init_flow (hydro/init_flow_fine.f90:1-20) */
  for (int l = T->nlevelmax; l >= 1; l--) {
    if (l >= T->levelmin) init_flow_fine(T, l);
    upload_fine(T, l);
    make_boundary_hydro(T, l);
  }
}

/* update_time (amr/update_time.f90:191-380): the end test, then t += dt */
static int update_time(t1d *T, int ilevel) {
  double dt = T->dtnew[ilevel];
  int stop = 0;
  if (T->nstep_coarse != T->nstep_coarse_old)
    if (T->t >= T->P->tout) stop = 1;
  T->nstep_coarse_old = T->nstep_coarse;
  if (stop) return 1;
  T->t = T->t + dt;
  T->nstep++;
  return 0;
}

/* amr_step (amr/amr_step.f90), the hydro-only sequence; returns 1 when the
 * run ends (snapshot taken, or update_time's end test) */
static int amr_step(t1d *T, int ilevel, int icount, orc1d_result *res) {
  if (T->numbl[ilevel] == 0) return 0;
  if (T->levelmin < T->nlevelmax && (ilevel == T->levelmin || icount > 1)) { /* :41-93 */
    for (int i = ilevel; i <= T->nlevelmax; i++) {
      if (i > T->levelmin) make_boundary_hydro(T, i);
      refine_fine(T, i);
      if (T->err) return 1;
    }
  }
  if (ilevel == T->levelmin && T->t >= T->P->tout) { /* dump_all :150-176 */
    res->taken = 1;
    return 1;
  }
  T->dtold[ilevel] = T->dtnew[ilevel]; /* newdt_fine (pm/newdt_fine.f90:47-51,177) */
  T->dtnew[ilevel] = T->P->boxlen / T->hp.smallc;
  courant_fine(T, ilevel);
  if (ilevel > T->levelmin)
    T->dtnew[ilevel] = fmind1(T->dtnew[ilevel - 1] / (double)(float)T->P->nsubcycle[ilevel - 1], T->dtnew[ilevel]);
  set_unew(T, ilevel);
  if (ilevel < T->nlevelmax) {
    if (T->numbl[ilevel + 1] > 0) {
      if (T->P->nsubcycle[ilevel] == 2) {
        if (amr_step(T, ilevel + 1, 1, res)) return 1;
        if (amr_step(T, ilevel + 1, 2, res)) return 1;
      } else {
        if (amr_step(T, ilevel + 1, 1, res)) return 1;
      }
    } else {
      T->dtold[ilevel + 1] = T->dtnew[ilevel] / (double)T->P->nsubcycle[ilevel];
      T->dtnew[ilevel + 1] = T->dtnew[ilevel] / (double)T->P->nsubcycle[ilevel];
      if (update_time(T, ilevel)) return 1;
    }
  } else {
    if (update_time(T, ilevel)) return 1;
  }
  godunov_fine(T, ilevel);
  if (T->err) return 1;
  set_uold(T, ilevel);
  upload_fine(T, ilevel);
  make_boundary_hydro(T, ilevel);
  flag_fine(T, ilevel, icount);
  if (ilevel > T->levelmin) { /* :573-576 */
    if (T->P->nsubcycle[ilevel - 1] == 1) T->dtnew[ilevel - 1] = T->dtnew[ilevel];
    if (icount == 2) T->dtnew[ilevel - 1] = T->dtold[ilevel] + T->dtnew[ilevel];
  }
  return T->err;
}

static void fill_result(t1d *T, orc1d_result *res) {
  int nleaf = 0;
  double scale = scale_of(T), skip = (double)T->icoarse_min;
  for (int l = 1; l <= T->nlevelmax; l++) {
    int n = level_list(T, l, T->lst);
    double dx = pow(0.5, l);
    res->noct[l] = n;
    for (int i = 0; i < n; i++)
      for (int ind = 1; ind <= 2; ind++) {
        int c = CELL(T, T->lst[i], ind);
        if (T->son[c] != 0) continue;
        if (nleaf < res->capacity) {
          res->x[nleaf] = (T->xg[T->lst[i]] + ((double)(ind - 1) - 0.5) * dx - skip) * scale;
          res->level[nleaf] = l;
          for (int v = 1; v <= NV1; v++) res->u[(size_t)nleaf * NV1 + v - 1] = UO(T, c, v);
        }
        nleaf++;
      }
  }
  res->ncell = nleaf;
  res->t = T->t;
  res->nstep = T->nstep;
  res->nstep_coarse = T->nstep_coarse;
}

int orc1d_run(const orc1d_params *P, orc1d_result *res) {
  if (!P || !res || P->nlevelmax < 1 || P->nlevelmax > ORC_MAXLEVEL || P->levelmin < 1 ||
      P->levelmin > P->nlevelmax || P->ngridmax < 4 || P->nboundary < 0 || P->nboundary > 2)
    return -1;
  t1d T;
  memset(&T, 0, sizeof T);
  T.P = P;
  T.hp = P->hydro;
  T.nlevelmax = P->nlevelmax;
  T.levelmin = P->levelmin;
  T.ngridmax = P->ngridmax;
  /* coarse grid and boundary regions (hydro/read_hydro_params.f90:310-360) */
  T.nx = 1;
  T.nboundary = P->nboundary;
  for (int ib = 0; ib < T.nboundary; ib++) {
    T.nx += 1;
    if (P->bound_side[ib] < 0) { T.icoarse_min += 1; T.icoarse_max += 1; }
  }
  for (int ib = 0; ib < T.nboundary; ib++) {
    int left = P->bound_side[ib] < 0, bt = P->bound_type[ib];
    if (bt != 1 && bt != 2) return -1;
    T.ibound_min[ib] = T.ibound_max[ib] = left ? T.icoarse_min - 1 : T.icoarse_max + 1;
    T.boundary_type[ib] = bt == 1 ? (left ? 1 : 2) : (left ? 11 : 12);
  }
  T.ncoarse = T.nx;
  T.ncell = T.ncoarse + 2 * T.ngridmax;
  T.son = calloc((size_t)T.ncell + 1, sizeof(int32_t));
  T.flag1 = calloc((size_t)T.ncell + 1, sizeof(int32_t));
  T.flag2 = calloc((size_t)T.ncell + 1, sizeof(int32_t));
  T.father = calloc((size_t)T.ngridmax + 1, sizeof(int32_t));
  T.next = calloc((size_t)T.ngridmax + 1, sizeof(int32_t));
  T.prev = calloc((size_t)T.ngridmax + 1, sizeof(int32_t));
  T.nbor = calloc(((size_t)T.ngridmax + 1) * 2, sizeof(int32_t));
  T.xg = calloc((size_t)T.ngridmax + 1, sizeof(double));
  T.uold = calloc(((size_t)T.ncell + 1) * NV1, sizeof(double));
  T.unew = calloc(((size_t)T.ncell + 1) * NV1, sizeof(double));
  T.lst = calloc((size_t)T.ngridmax + 1, sizeof(int32_t));
  T.lst2 = calloc((size_t)T.ngridmax + 1, sizeof(int32_t));
  int rc = 0;
  if (!T.son || !T.flag1 || !T.flag2 || !T.father || !T.next || !T.prev || !T.nbor || !T.xg || !T.uold ||
      !T.unew || !T.lst || !T.lst2) {
    rc = -2;
    goto done;
  }
  /* free list (amr/init_amr.f90) */
  T.headf = 1; T.tailf = T.ngridmax; T.numbf = T.ngridmax;
  for (int g = 1; g <= T.ngridmax; g++) { T.next[g] = g < T.ngridmax ? g + 1 : 0; T.prev[g] = g - 1; }

  /* init_refine (amr/init_refine.f90:5-44) */
  T.init = 1;
  for (int l = 1; l <= T.levelmin; l++) { flag_all(&T); refine_all(&T); }
  for (int l = T.levelmin + 1; l <= T.nlevelmax && !T.err; l++) {
    init_flow(&T);
    flag_all(&T);
    refine_all(&T);
    if (T.numbl[l] == 0) break;
  }
  T.init = 0;
  init_flow(&T);
  /* init_refine_2 (:49-150) */
  for (int i = T.levelmin; i <= T.nlevelmax + 1 && !T.err; i++) {
    refine_coarse(&T);
    for (int l = 1; l <= T.nlevelmax; l++) {
      refine_fine(&T, l);
      init_flow_fine(&T, l);
    }
    for (int l = T.nlevelmax; l >= T.levelmin; l--) {
      upload_fine(&T, l);
      make_boundary_hydro(&T, l);
    }
    for (int l = T.nlevelmax; l >= 1; l--) flag_fine(&T, l, 2);
    flag_coarse(&T);
  }
  if (T.err) { rc = -3; goto done; }
  if (res->init_only) { fill_result(&T, res); goto done; }

  /* adaptive_loop (amr/adaptive_loop.f90) */
  res->taken = 0;
  T.nstep_coarse_old = T.nstep_coarse;
  for (int64_t it = 0; it < P->max_coarse_steps; it++) {
    if (T.levelmin < T.nlevelmax) {
      refine_coarse(&T);
      for (int l = 1; l <= T.levelmin; l++) {
        make_boundary_hydro(&T, l);
        if (l < T.levelmin) refine_fine(&T, l);
      }
    }
    int end = amr_step(&T, T.levelmin, 1, res);
    if (T.err) { rc = -3; goto done; }
    if (end) break;
    if (T.levelmin < T.nlevelmax) {
      for (int l = T.levelmin - 1; l >= 1; l--) { upload_fine(&T, l); make_boundary_hydro(&T, l); }
      for (int l = T.levelmin - 1; l >= 1; l--) flag_fine(&T, l, 2);
      flag_coarse(&T);
    }
    T.nstep_coarse++;
  }
  fill_result(&T, res);
done:
  if (T.err) snprintf(res->message, sizeof res->message, "%s", T.msg);
  free(T.son); free(T.flag1); free(T.flag2); free(T.father); free(T.next); free(T.prev);
  free(T.nbor); free(T.xg); free(T.uold); free(T.unew); free(T.lst); free(T.lst2);
  return rc;
}
