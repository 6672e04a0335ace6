/*
 * ramses_oracle_amr.c -- TEST INFRASTRUCTURE ONLY. A CPU restatement of a
 * whole RAMSES hydro run built with NDIM=1 or NDIM=2 (nvar = ndim+2), one
 * MPI rank, hydro only: the initial refinement, the adaptive time loop with
 * subcycling, refinement and derefinement at every level step, wall and
 * free boundaries, and the snapshot's leaf cells at the first coarse step
 * that starts at t >= tout. It exists to pin the oracle's restatement
 * against the reference's own regression checksums (tests/hydro/sod-tube,
 * a 1D AMR run, and tests/hydro/implosion, a 2D one); the product library
 * never links or calls it.
 *
 * Every routine follows the cited Fortran for the build's NDIM
 * (twotondim = 2^ndim, twondim = 2 ndim, threetondim = 3^ndim,
 * nvector = 500), keeping the reference's operation order and its nvector
 * batches where the order of accumulation depends on them. The Riemann
 * solvers are the ones of the 3D restatement (orc_riemann_face in
 * ramses_oracle.c), called with the transverse velocities the build lacks
 * set to zero. Arrays are 1-based like the Fortran: cells 0..ncell with
 * icell = ncoarse + (ind-1)*ngridmax + igrid, grids 0..ngridmax; index 0 is
 * the reference's "absent" cell or grid.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ramses_oracle.h"
#include "ramses_oracle_amr.h"

#define NVMAX 4    /* nvar of the 2D build */
#define NVEC 500   /* nvector (amr/amr_parameters.f90) */
#define NB_MAX ORC_AMR_MAXBOUND

static inline double fmaxd1(double a, double b) { return a > b ? a : (b > a ? b : a); }
static inline double fmind1(double a, double b) { return a < b ? a : (b < a ? b : a); }

typedef struct tamr {
  const orc_amr_params *P;
  orc_params hp;
  int ndim, nv, twotondim, twondim, threetondim;
  int nx, ny, ncoarse, ngridmax, ncell, nlevelmax, levelmin;
  int icoarse_min, icoarse_max, jcoarse_min, jcoarse_max;
  int nboundary, boundary_type[NB_MAX];
  int ibmin[NB_MAX], ibmax[NB_MAX], jbmin[NB_MAX], jbmax[NB_MAX];
  int32_t *son, *flag1, *flag2;  /* [ncell+1] */
  int32_t *father, *next, *prev; /* [ngridmax+1] */
  int32_t *nbor;                 /* [(ngridmax+1)*4] */
  double *xg;                    /* [(ngridmax+1)*2], coarse units */
  double *uold, *unew;           /* [(ncell+1)*NVMAX] */
  int headl[ORC_MAXLEVEL + 2], taill[ORC_MAXLEVEL + 2], numbl[ORC_MAXLEVEL + 2];
  int headb[NB_MAX][ORC_MAXLEVEL + 2], tailb[NB_MAX][ORC_MAXLEVEL + 2], numbb[NB_MAX][ORC_MAXLEVEL + 2];
  int headf, tailf, numbf;
  double dtnew[ORC_MAXLEVEL + 2], dtold[ORC_MAXLEVEL + 2], t;
  int64_t nstep, nstep_coarse, nstep_coarse_old;
  int init;
  int err;
  volatile int perr; /* error seen inside the threaded flux phase */
  char msg[160];
  int32_t *lst, *lst2;           /* scratch grid lists [ngridmax+1] */
  double (*flux)[2][4][4][NVMAX]; /* [NVEC][idim][j3][i3][v] */
  int32_t (*fok)[6][6];          /* [NVEC][j3+1][i3+1] */
} tamr;

#define CELL(T, g, ind) ((T)->ncoarse + ((ind) - 1) * (T)->ngridmax + (g))
#define UO(T, c, v) ((T)->uold[(size_t)(c) * NVMAX + (v) - 1])
#define UN(T, c, v) ((T)->unew[(size_t)(c) * NVMAX + (v) - 1])
#define NB(T, g, j) ((T)->nbor[(size_t)(g) * 4 + (j) - 1])
#define XG(T, g, d) ((T)->xg[(size_t)(g) * 2 + (d) - 1])

static void fail1(tamr *T, const char *m) {
  if (!T->err) { T->err = 1; snprintf(T->msg, sizeof T->msg, "%s", m); }
}
/* cell position ind -> (ix, iy) */
static inline int IX(int ind) { return (ind - 1) & 1; }
static inline int IY(int ind) { return ((ind - 1) >> 1) & 1; }

/* active(ilevel)%igrid and boundary(ibound,ilevel)%igrid: the level's linked
 * list in order (build_comm, amr/virtual_boundaries.f90) */
static int level_list(const tamr *T, int l, int32_t *out) {
  int n = 0;
  for (int g = T->headl[l]; g > 0 && n < T->numbl[l]; g = T->next[g]) out[n++] = g;
  return n;
}
static int bound_list(const tamr *T, int ib, int l, int32_t *out) {
  int n = 0;
  for (int g = T->headb[ib][l]; g > 0 && n < T->numbb[ib][l]; g = T->next[g]) out[n++] = g;
  return n;
}
static void list_append(tamr *T, int *head, int *tail, int *numb, int g) {
  if (*numb > 0) {
    T->next[g] = 0; T->prev[g] = *tail; T->next[*tail] = g; *tail = g; *numb += 1;
  } else {
    T->next[g] = 0; T->prev[g] = 0; *head = g; *tail = g; *numb = 1;
  }
}
static void list_remove(tamr *T, int *head, int *tail, int *numb, int g) {
  if (T->prev[g] != 0) {
    if (T->next[g] != 0) { T->next[T->prev[g]] = T->next[g]; T->prev[T->next[g]] = T->prev[g]; }
    else { T->next[T->prev[g]] = 0; *tail = T->prev[g]; }
  } else {
    if (T->next[g] != 0) { T->prev[T->next[g]] = 0; *head = T->next[g]; }
    else { *head = 0; *tail = 0; }
  }
  *numb -= 1;
}

/* ---- neighbour utilities: amr/nbors_utils.f90 ---- */
/* getnborgrids :530-555 */
static void getnborgrids(const tamr *T, int g, int igridn[5]) {
  igridn[0] = g;
  for (int j = 1; j <= T->twondim; j++) igridn[j] = T->son[NB(T, g, j)];
}
/* getnborgrids_check (an absent nbor gives no grid) */
static void getnborgrids_check(const tamr *T, int g, int igridn[5]) {
  igridn[0] = g;
  for (int j = 1; j <= T->twondim; j++) igridn[j] = NB(T, g, j) > 0 ? T->son[NB(T, g, j)] : 0;
}
/* getnborcells :363-399: neighbour in direction j of cell ind, in the same
 * grid when the move stays inside it, else in neighbour grid j (the ggg/hhh
 * tables); 0 where that grid is absent */
static void getnborcells(const tamr *T, const int igridn[5], int ind, int icelln[5]) {
  for (int in = 1; in <= T->twondim; in++) {
    int d = (in - 1) / 2, plus = (in - 1) & 1;
    int c[2] = {IX(ind), IY(ind)};
    int inside = plus ? (c[d] == 0) : (c[d] == 1);
    int ig = inside ? 0 : in;
    c[d] = 1 - c[d];
    int ih = 1 + c[0] + 2 * c[1];
    icelln[in] = igridn[ig] > 0 ? T->ncoarse + (ih - 1) * T->ngridmax + igridn[ig] : 0;
  }
}
/* get3cubefather :5-300 (with get3cubepos and getindices3cube): the 3^ndim
 * father-level cells around cell fcell of level ilevel-1, out[i1+3*j1];
 * 0 where the grid toward that side is absent */
static void get3cubefather(const tamr *T, int fcell, int ilevel, int out[9]) {
  const int jmax = T->ndim > 1 ? 2 : 0;
  if (ilevel == 1) {
    int iy = (fcell - 1) / T->nx, ix = fcell - 1 - iy * T->nx;
    for (int j1 = 0; j1 <= jmax; j1++) {
      int iiy = iy;
      if (T->ndim > 1) {
        iiy = iy + j1 - 1;
        if (iiy < 0) iiy = T->ny - 1;
        if (iiy > T->ny - 1) iiy = 0;
      }
      for (int i1 = 0; i1 <= 2; i1++) {
        int iix = ix + i1 - 1;
        if (iix < 0) iix = T->nx - 1;
        if (iix > T->nx - 1) iix = 0;
        out[i1 + 3 * j1] = 1 + iix + iiy * T->nx;
      }
    }
    return;
  }
  int pos = (fcell - T->ncoarse - 1) / T->ngridmax + 1;
  int g = fcell - T->ncoarse - (pos - 1) * T->ngridmax;
  int c[2] = {IX(pos), IY(pos)};
  int grids[4];
  for (int jj = 0; jj <= (T->ndim > 1 ? 1 : 0); jj++) {
    int g2 = g;
    if (jj > 0 && g2 > 0) g2 = T->son[NB(T, g2, c[1] ? 4 : 3)];
    for (int ii = 0; ii <= 1; ii++) {
      int g3 = g2;
      if (ii > 0 && g3 > 0) g3 = T->son[NB(T, g3, c[0] ? 2 : 1)];
      grids[ii + 2 * jj] = g3;
    }
  }
  for (int j1 = 0; j1 <= jmax; j1++)
    for (int i1 = 0; i1 <= 2; i1++) {
      int o[2] = {i1 - 1, j1 - 1}, sel = 0, cell = 0;
      for (int a = 0; a < T->ndim; a++) {
        int cp = c[a] + o[a];
        int gs = cp < 0 ? -1 : (cp > 1 ? 1 : 0);
        if (gs != 0) sel |= 1 << a;
        cell |= (cp - 2 * gs) << a;
      }
      int gr = grids[sel];
      out[i1 + 3 * j1] = gr > 0 ? T->ncoarse + cell * T->ngridmax + gr : 0;
    }
}
/* getnborfather :404-525: cell, then its 2 ndim neighbours at the same
 * level, or the coarser neighbour cell nbor(grid,j) where absent */
static void getnborfather(const tamr *T, int cell, int ilevel, int f[5]) {
  f[0] = cell;
  if (ilevel == 1) {
    int iy = (cell - 1) / T->nx, ix = cell - 1 - iy * T->nx;
    f[1] = ix > 0 ? cell - 1 : cell + (T->nx - 1);
    f[2] = ix < T->nx - 1 ? cell + 1 : cell - (T->nx - 1);
    if (T->ndim > 1) {
      f[3] = iy > 0 ? cell - T->nx : cell + (T->ny - 1) * T->nx;
      f[4] = iy < T->ny - 1 ? cell + T->nx : cell - (T->ny - 1) * T->nx;
    }
    return;
  }
  int pos = (cell - T->ncoarse - 1) / T->ngridmax + 1;
  int g = cell - T->ncoarse - (pos - 1) * T->ngridmax;
  for (int j = 1; j <= T->twondim; j++) {
    int d = (j - 1) / 2, plus = (j - 1) & 1;
    int c[2] = {IX(pos), IY(pos)};
    int inside = plus ? (c[d] == 0) : (c[d] == 1);
    int gg = inside ? g : T->son[NB(T, g, j)];
    c[d] = 1 - c[d];
    int icell = gg > 0 ? T->ncoarse + (c[0] + 2 * c[1]) * T->ngridmax + gg : 0;
    f[j] = icell > 0 ? icell : NB(T, g, j);
  }
}

/* ---- interpol_hydro, interpol_var = 0: hydro/interpol_hydro.f90:268-637 ----
 * u1[0..twondim][v] -> u2[ind-1][v] */
static int interpol_hydro(const tamr *T, double u1[5][NVMAX], double u2[4][NVMAX]) {
  const int itype = T->hp.interpol_type, nd = T->ndim, n2 = T->twotondim, nn = T->twondim;
  double xc[4][2];
  for (int ind = 1; ind <= n2; ind++) { xc[ind - 1][0] = (double)IX(ind) - 0.5; xc[ind - 1][1] = (double)IY(ind) - 0.5; }
  if (T->hp.interpol_var != 0 || itype < 0 || itype > 3) return -1;
  for (int ivar = 1; ivar <= T->nv; ivar++) {
    double a[5], w[2] = {0.0, 0.0};
    for (int j = 0; j <= nn; j++) a[j] = u1[j][ivar - 1];
    if (itype == 1) { /* compute_limiter_minmod :449-476 */
      for (int idim = 1; idim <= nd; idim++) {
        double dl = 0.5 * (a[2 * idim] - a[0]), dr = 0.5 * (a[0] - a[2 * idim - 1]);
        w[idim - 1] = dl * dr <= 0.0 ? 0.0 : fmind1(fabs(dl), fabs(dr)) * dl / fabs(dl);
      }
    } else if (itype == 2) { /* compute_limiter_central :481-613 */
      for (int idim = 1; idim <= nd; idim++) w[idim - 1] = 0.25 * (a[2 * idim] - a[2 * idim - 1]);
      double ac[4];
      for (int ind = 0; ind < n2; ind++) ac[ind] = a[0];
      for (int idim = 0; idim < nd; idim++)
        for (int ind = 0; ind < n2; ind++) ac[ind] = ac[ind] + 2.0 * w[idim] * xc[ind][idim];
      double corner = ac[0], kernel = a[1];
      for (int j = 1; j < n2; j++) corner = fmaxd1(corner, ac[j]);
      for (int j = 2; j <= nn; j++) kernel = fmaxd1(kernel, a[j]);
      double dk = a[0] - kernel, dc = a[0] - corner, maxl = 0.0, minl = 0.0;
      if (dk * dc > 0.0) maxl = fmind1(1.0, dk / dc);
      corner = ac[0];
      kernel = a[1];
      for (int j = 1; j < n2; j++) corner = fmind1(corner, ac[j]);
      for (int j = 2; j <= nn; j++) kernel = fmind1(kernel, a[j]);
      dk = a[0] - kernel; dc = a[0] - corner;
      if (dk * dc > 0.0) minl = fmind1(1.0, dk / dc);
      double lim = fmind1(minl, maxl);
      for (int idim = 0; idim < nd; idim++) w[idim] = w[idim] * lim;
    } else if (itype == 3) { /* compute_central :618-637 */
      for (int idim = 1; idim <= nd; idim++) w[idim - 1] = 0.25 * (a[2 * idim] - a[2 * idim - 1]);
    }
    for (int ind = 0; ind < n2; ind++) {
      double v = a[0];
      for (int idim = 0; idim < nd; idim++) v = v + w[idim] * xc[ind][idim];
      u2[ind][ivar - 1] = v;
    }
  }
  return 0;
}

/* ---- initial conditions: hydro/condinit.f90, region_condinit ('square') ---- */
static void condinit(const tamr *T, const double x[2], double u[NVMAX]) {
  const orc_amr_params *P = T->P;
  const double gamma = T->hp.gamma;
  const int nd = T->ndim, ip = nd + 1;
  double q[NVMAX] = {T->hp.smallr, 0.0, 0.0, 0.0};
  q[ip] = T->hp.smallr * (T->hp.smallc * T->hp.smallc) / gamma;
  for (int k = 0; k < P->nregion; k++) {
    double en = P->exp_region[k];
    double xn = 2.0 * fabs(x[0] - P->x_center[k]) / P->length_x[k], yn = 0.0, zn = 0.0;
    if (nd > 1) yn = 2.0 * fabs(x[1] - P->y_center[k]) / P->length_y[k];
    double r = en < 10 ? pow(pow(xn, en) + pow(yn, en) + pow(zn, en), 1.0 / en) : fmaxd1(fmaxd1(xn, yn), zn);
    if (r < 1.0) {
      q[0] = P->d_region[k];
      q[1] = P->u_region[k];
      if (nd > 1) q[2] = P->v_region[k];
      q[ip] = P->p_region[k];
    }
  }
  u[0] = q[0];
  for (int d = 1; d <= nd; d++) u[d] = q[0] * q[d];
  u[ip] = 0.0;
  for (int d = 1; d <= nd; d++) u[ip] = u[ip] + 0.5 * q[0] * (q[d] * q[d]);
  u[ip] = u[ip] + q[ip] / (gamma - 1.0);
}

static double scale_of(const tamr *T) { return T->P->boxlen / (double)(T->icoarse_max - T->icoarse_min + 1); }

/* cell-centre position of cell ind of grid g at level ilevel (condinit's xx) */
static void cell_pos(const tamr *T, int g, int ind, int ilevel, double x[2]) {
  double dx = pow(0.5, ilevel), scale = scale_of(T);
  double xc0 = ((double)IX(ind) - 0.5) * dx, xc1 = ((double)IY(ind) - 0.5) * dx;
  x[0] = (XG(T, g, 1) + xc0 - (double)T->icoarse_min) * scale;
  x[1] = T->ndim > 1 ? (XG(T, g, 2) + xc1 - (double)T->jcoarse_min) * scale : 0.0;
}

/* init_flow_fine (hydro/init_flow_fine.f90:418-456): condinit at the cell centres */
static void init_flow_fine(tamr *T, int ilevel) {
  int n = level_list(T, ilevel, T->lst);
  for (int ind = 1; ind <= T->twotondim; ind++)
    for (int i = 0; i < n; i++) {
      double x[2], u[NVMAX];
      cell_pos(T, T->lst[i], ind, ilevel, x);
      condinit(T, x, u);
      for (int v = 1; v <= T->nv; v++) UO(T, CELL(T, T->lst[i], ind), v) = u[v - 1];
    }
}

/* upload_fine / upl (hydro/interpol_hydro.f90:5-150), interpol_var = 0 */
static void upload_fine(tamr *T, int ilevel) {
  if (ilevel == T->nlevelmax) return;
  int n = level_list(T, ilevel, T->lst);
  const double n2 = (double)T->twotondim;
  for (int ind = 1; ind <= T->twotondim; ind++)
    for (int i = 0; i < n; i++) {
      int cell = CELL(T, T->lst[i], ind), gs = T->son[cell];
      if (gs <= 0) continue;
      double getx = 0.0;
      for (int is = 1; is <= T->twotondim; is++) getx = getx + fmaxd1(UO(T, CELL(T, gs, is), 1), T->hp.smallr);
      UO(T, cell, 1) = getx / n2;
      for (int ivar = 2; ivar <= T->nv; ivar++) {
        getx = 0.0;
        for (int is = 1; is <= T->twotondim; is++) getx = getx + UO(T, CELL(T, gs, is), ivar);
        UO(T, cell, ivar) = getx / n2;
      }
    }
}

/* boundary direction of a region (boundary_type - 10*(boundary_type/10)),
 * the reference neighbour inbor and the reference cell of each position
 * (make_boundary_hydro :57-90, make_boundary_flag) */
static void boundary_rule(const tamr *T, int ib, int *inbor, int ind_ref[5]) {
  static const int inb[7] = {0, 2, 1, 4, 3, 6, 5};
  static const int wall[3][4] = {{2, 1, 4, 3}, {3, 4, 1, 2}, {5, 6, 7, 8}};
  static const int freeb[6][4] = {{1, 1, 3, 3}, {2, 2, 4, 4}, {1, 2, 1, 2}, {3, 4, 3, 4}, {1, 2, 3, 4}, {5, 6, 7, 8}};
  const int bt = T->boundary_type[ib], dir = bt - 10 * (bt / 10);
  *inbor = inb[dir];
  for (int ind = 1; ind <= 4; ind++)
    ind_ref[ind] = bt / 10 == 0 ? wall[(dir - 1) / 2][ind - 1] : freeb[dir - 1][ind - 1];
}

/* make_boundary_hydro (hydro/hydro_boundary.f90:5-260): walls mirror the
 * reference grid with the normal velocity negated, free boundaries copy
 * the adjacent layer with E - ekin + ekin recomputed; per nvector batch
 * and cell position, the batch is gathered before it is scattered */
static void make_boundary_hydro(tamr *T, int ilevel) {
  const int nv = T->nv, nd = T->ndim;
  static double uu[NVEC][NVMAX];
  static int gref[NVEC];
  for (int ib = 0; ib < T->nboundary; ib++) {
    const int bt = T->boundary_type[ib], dir = bt - 10 * (bt / 10);
    int inbor, ind_ref[5];
    boundary_rule(T, ib, &inbor, ind_ref);
    double gs[2] = {1.0, 1.0};
    if (bt / 10 == 0) gs[(dir - 1) / 2] = -1.0;
    int n = bound_list(T, ib, ilevel, T->lst);
    for (int i0 = 0; i0 < n; i0 += NVEC) {
      int ng = n - i0 < NVEC ? n - i0 : NVEC;
      for (int i = 0; i < ng; i++) {
        gref[i] = T->son[NB(T, T->lst[i0 + i], inbor)];
        if (gref[i] <= 0) { fail1(T, "make_boundary_hydro: boundary grid without a reference grid"); return; }
      }
      for (int ind = 1; ind <= T->twotondim; ind++) {
        for (int i = 0; i < ng; i++)
          for (int v = 1; v <= nv; v++) uu[i][v - 1] = UO(T, CELL(T, gref[i], ind_ref[ind]), v);
        if (bt / 10 == 0) {
          for (int v = 1; v <= nv; v++) {
            double sw = (v > 1 && v <= nd + 1) ? gs[v - 2] : 1.0;
            for (int i = 0; i < ng; i++) UO(T, CELL(T, T->lst[i0 + i], ind), v) = uu[i][v - 1] * sw;
          }
        } else {
          for (int i = 0; i < ng; i++) {
            double ekin = 0.0, d = fmaxd1(uu[i][0], T->hp.smallr);
            for (int idim = 1; idim <= nd; idim++) {
              double vv = uu[i][idim] / d;
              ekin = ekin + 0.5 * d * (vv * vv);
            }
            uu[i][nd + 1] = uu[i][nd + 1] - ekin;
          }
          for (int v = 1; v <= nv; v++)
            for (int i = 0; i < ng; i++) UO(T, CELL(T, T->lst[i0 + i], ind), v) = uu[i][v - 1];
          for (int i = 0; i < ng; i++) {
            int c = CELL(T, T->lst[i0 + i], ind);
            double ekin = 0.0, d = fmaxd1(UO(T, c, 1), T->hp.smallr);
            for (int idim = 1; idim <= nd; idim++) {
              double vv = UO(T, c, idim + 1) / d;
              ekin = ekin + 0.5 * d * (vv * vv);
            }
            UO(T, c, nd + 2) = UO(T, c, nd + 2) + ekin;
          }
        }
      }
    }
  }
}

/* ---- flags: amr/flag_utils.f90, amr/virtual_boundaries.f90 ---- */
/* make_boundary_flag (virtual_boundaries.f90): per batch and cell
 * position, gathered before scattered */
static void make_boundary_flag(tamr *T, int ilevel) {
  static int fff[NVEC], gref[NVEC];
  for (int ib = 0; ib < T->nboundary; ib++) {
    int inbor, ind_ref[5];
    boundary_rule(T, ib, &inbor, ind_ref);
    int n = bound_list(T, ib, ilevel, T->lst2);
    for (int i0 = 0; i0 < n; i0 += NVEC) {
      int ng = n - i0 < NVEC ? n - i0 : NVEC;
      for (int i = 0; i < ng; i++) gref[i] = T->son[NB(T, T->lst2[i0 + i], inbor)];
      for (int ind = 1; ind <= T->twotondim; ind++) {
        for (int i = 0; i < ng; i++) fff[i] = T->flag1[T->ncoarse + (ind_ref[ind] - 1) * T->ngridmax + gref[i]];
        for (int i = 0; i < ng; i++) T->flag1[CELL(T, T->lst2[i0 + i], ind)] = fff[i];
      }
    }
  }
}

/* init_flag :111-163 with test_flag :168-208 */
static void init_flag(tamr *T, int ilevel) {
  int n = level_list(T, ilevel, T->lst);
  for (int ind = 1; ind <= T->twotondim; ind++)
    for (int i = 0; i < n; i++) T->flag1[CELL(T, T->lst[i], ind)] = 0;
  if (ilevel >= T->levelmin) {
    for (int ind = 1; ind <= T->twotondim; ind++)
      for (int i = 0; i < n; i++) {
        int gs = T->son[CELL(T, T->lst[i], ind)], ok = 0;
        if (gs > 0)
          for (int is = 1; is <= T->twotondim; is++) {
            int cs = CELL(T, gs, is);
            ok = ok || T->son[cs] > 0;
            ok = ok || T->flag1[cs] == 1;
          }
        if (ok) T->flag1[CELL(T, T->lst[i], ind)] = 1;
      }
  } else {
    for (int ind = 1; ind <= T->twotondim; ind++)
      for (int i = 0; i < n; i++) T->flag1[CELL(T, T->lst[i], ind)] = 1;
  }
  make_boundary_flag(T, ilevel);
}

/* smooth_fine :555-638 with count_nbors :643-677, n_nbor = (1,2,2) */
static void smooth_fine(tamr *T, int ilevel) {
  static const int n_nbor[3] = {1, 2, 2};
  if (ilevel == T->nlevelmax) return;
  int n = level_list(T, ilevel, T->lst);
  if (n == 0) return;
  T->flag1[0] = 0;
  for (int ism = 0; ism < T->ndim; ism++) {
    for (int ind = 1; ind <= T->twotondim; ind++)
      for (int i = 0; i < n; i++) T->flag2[CELL(T, T->lst[i], ind)] = 0;
    for (int i = 0; i < n; i++) {
      int igridn[5];
      getnborgrids(T, T->lst[i], igridn);
      for (int ind = 1; ind <= T->twotondim; ind++) {
        int indn[5], cnt = 0;
        getnborcells(T, igridn, ind, indn);
        for (int in = 1; in <= T->twondim; in++) cnt += T->flag1[indn[in]];
        if (cnt >= n_nbor[ism]) T->flag2[CELL(T, T->lst[i], ind)] = 1;
      }
    }
    for (int ind = 1; ind <= T->twotondim; ind++)
      for (int i = 0; i < n; i++) {
        int c = CELL(T, T->lst[i], ind);
        if (T->flag1[c] == 1) T->flag2[c] = 0;
        if (T->flag2[c] == 1) T->flag1[c] = 1;
      }
    make_boundary_flag(T, ilevel);
  }
}

/* hydro_refine (hydro/godunov_utils.f90:125-263) for one direction;
 * g, m, d are conservative states, converted in place */
static int hydro_refine(const tamr *T, double g[NVMAX], double m[NVMAX], double d[NVMAX]) {
  const orc_refine *r = &T->P->refine;
  const int nd = T->ndim, ip = nd + 1;
  const double gamma = T->hp.gamma, half = 0.5, one = 1.0, zero = 0.0;
  g[0] = fmaxd1(g[0], T->hp.smallr);
  m[0] = fmaxd1(m[0], T->hp.smallr);
  d[0] = fmaxd1(d[0], T->hp.smallr);
  for (int idim = 1; idim <= nd; idim++) {
    g[idim] = g[idim] / g[0];
    m[idim] = m[idim] / m[0];
    d[idim] = d[idim] / d[0];
  }
  double eking = zero, ekinm = zero, ekind = zero;
  for (int idim = 1; idim <= nd; idim++) {
    eking = eking + half * g[0] * (g[idim] * g[idim]);
    ekinm = ekinm + half * m[0] * (m[idim] * m[idim]);
    ekind = ekind + half * d[0] * (d[idim] * d[idim]);
  }
  g[ip] = (gamma - one) * (g[ip] - eking);
  m[ip] = (gamma - one) * (m[ip] - ekinm);
  d[ip] = (gamma - one) * (d[ip] - ekind);
  int ok = 0;
  if (r->err_grad_d >= 0.) {
    double error = 2.0 * fmaxd1(fabs((d[0] - m[0]) / (d[0] + m[0] + r->floor_d)),
                                fabs((m[0] - g[0]) / (m[0] + g[0] + r->floor_d)));
    ok = ok || error > r->err_grad_d;
  }
  if (r->err_grad_p >= 0.) {
    double error = 2.0 * fmaxd1(fabs((d[ip] - m[ip]) / (d[ip] + m[ip] + r->floor_p)),
                                fabs((m[ip] - g[ip]) / (m[ip] + g[ip] + r->floor_p)));
    ok = ok || error > r->err_grad_p;
  }
  if (r->err_grad_u >= 0.) {
    for (int idim = 1; idim <= nd; idim++) {
      double f2 = r->floor_u * r->floor_u;
      double cg = sqrt(fmaxd1(gamma * g[ip] / g[0], f2));
      double cm = sqrt(fmaxd1(gamma * m[ip] / m[0], f2));
      double cd = sqrt(fmaxd1(gamma * d[ip] / d[0], f2));
      double vg = g[idim], vm = m[idim], vd = d[idim];
      double error = 2.0 * fmaxd1(fabs((vd - vm) / (cd + cm + fabs(vd) + fabs(vm) + r->floor_u)),
                                  fabs((vm - vg) / (cm + cg + fabs(vm) + fabs(vg) + r->floor_u)));
      ok = ok || error > r->err_grad_u;
    }
  }
  return ok;
}

/* userflag_fine :281-427 (no geometry or Poisson criterion) -> hydro_flag
 * (hydro/hydro_flag.f90:1-180) */
static void userflag_fine(tamr *T, int ilevel) {
  if (ilevel == T->nlevelmax) return;
  int n = level_list(T, ilevel, T->lst);
  if (n == 0) return;
  const orc_refine *r = &T->P->refine;
  if (!(r->err_grad_d == -1.0 && r->err_grad_p == -1.0 && r->err_grad_u == -1.0)) {
    for (int i = 0; i < n; i++) {
      int g = T->lst[i], igridn[5];
      getnborgrids(T, g, igridn);
      for (int ind = 1; ind <= T->twotondim; ind++) {
        int cell = CELL(T, g, ind), indn[5], ok = 0;
        getnborcells(T, igridn, ind, indn);
        for (int j = 1; j <= T->twondim; j++)
          if (indn[j] == 0) indn[j] = NB(T, g, j);
        for (int idim = 1; idim <= T->ndim; idim++) {
          double ug[NVMAX], um[NVMAX], ud[NVMAX];
          for (int v = 1; v <= T->nv; v++) {
            ug[v - 1] = UO(T, indn[2 * idim - 1], v);
            um[v - 1] = UO(T, cell, v);
            ud[v - 1] = UO(T, indn[2 * idim], v);
          }
          if (hydro_refine(T, ug, um, ud)) ok = 1;
        }
        if (ok) T->flag1[cell] = 1;
      }
    }
  }
  make_boundary_flag(T, ilevel);
}

/* ensure_ref_rules :213-276: unflag the cells of grids whose father's
 * 3^ndim neighbour cells are not all refined */
static void ensure_ref_rules(tamr *T, int ilevel) {
  int n = level_list(T, ilevel, T->lst);
  for (int i = 0; i < n; i++) {
    int g = T->lst[i], nb[9], ok = 1;
    get3cubefather(T, T->father[g], ilevel, nb);
    for (int k = 0; k < T->threetondim; k++) {
      if (nb[k] == 0) ok = 0;
      if (nb[k] > 0 && T->son[nb[k]] == 0) ok = 0;
    }
    if (!ok)
      for (int ind = 1; ind <= T->twotondim; ind++) T->flag1[CELL(T, g, ind)] = 0;
  }
  make_boundary_flag(T, ilevel);
}

/* flag_fine :57-106 */
static void flag_fine(tamr *T, int ilevel, int icount) {
  if (ilevel == T->nlevelmax) return;
  if (T->numbl[ilevel] == 0) return;
  init_flag(T, ilevel);
  if (ilevel < T->levelmin) return;
  smooth_fine(T, ilevel);
  userflag_fine(T, ilevel);
  for (int ie = 1; ie <= T->P->nexpand[ilevel]; ie++) smooth_fine(T, ilevel);
  if (ilevel > T->levelmin && icount < T->P->nsubcycle[ilevel - 1]) ensure_ref_rules(T, ilevel);
}

/* flag_coarse :22-52 with make_boundary_coarse (virtual_boundaries.f90) */
static void flag_coarse(tamr *T) {
  for (int c = 0; c <= T->ncoarse; c++) T->flag1[c] = 0;
  for (int j = T->jcoarse_min; j <= T->jcoarse_max; j++)
    for (int i = T->icoarse_min; i <= T->icoarse_max; i++) T->flag1[1 + i + j * T->nx] = 1;
  for (int ib = 0; ib < T->nboundary; ib++) {
    int dir = T->boundary_type[ib] - 10 * (T->boundary_type[ib] / 10);
    int iskip = dir == 1 ? +1 : dir == 2 ? -1 : dir == 3 ? +T->nx : -T->nx;
    for (int j = T->jbmin[ib]; j <= T->jbmax[ib]; j++)
      for (int i = T->ibmin[ib]; i <= T->ibmax[ib]; i++) {
        int c = 1 + i + j * T->nx;
        T->flag1[c] = T->flag1[c + iskip];
      }
  }
}

/* ---- refinement: amr/refine_utils.f90 ---- */
/* make_grid_coarse :165-327 */
static void make_grid_coarse(tamr *T, int ind_cell, int ib, int boundary_region) {
  int g = T->headf;
  T->headf = T->next[T->headf];
  T->numbf--;
  int iy = (ind_cell - 1) / T->nx, ix = ind_cell - 1 - iy * T->nx;
  XG(T, g, 1) = (double)ix + 0.5;
  XG(T, g, 2) = T->ndim > 1 ? (double)iy + 0.5 : 0.0;
  T->son[ind_cell] = g;
  T->father[g] = ind_cell;
  int ixn[5] = {0, ix, ix, ix, ix}, iyn[5] = {0, iy, iy, iy, iy};
  ixn[1] = ix > 0 ? ix - 1 : T->nx - 1;
  ixn[2] = ix < T->nx - 1 ? ix + 1 : 0;
  if (T->ndim > 1) {
    iyn[3] = iy > 0 ? iy - 1 : T->ny - 1;
    iyn[4] = iy < T->ny - 1 ? iy + 1 : 0;
  }
  for (int j = 1; j <= T->twondim; j++) NB(T, g, j) = 1 + ixn[j] + iyn[j] * T->nx;
  if (boundary_region) list_append(T, &T->headb[ib][1], &T->tailb[ib][1], &T->numbb[ib][1], g);
  else list_append(T, &T->headl[1], &T->taill[1], &T->numbl[1], g);
}

/* kill_grid :953-1158 */
static void kill_grid(tamr *T, int ind_cell, int ilevel, int ib, int boundary_region) {
  int g = T->son[ind_cell];
  T->son[ind_cell] = 0;
  if (boundary_region) list_remove(T, &T->headb[ib][ilevel], &T->tailb[ib][ilevel], &T->numbb[ib][ilevel], g);
  else list_remove(T, &T->headl[ilevel], &T->taill[ilevel], &T->numbl[ilevel], g);
  XG(T, g, 1) = 0.0;
  XG(T, g, 2) = 0.0;
  T->father[g] = 0;
  for (int j = 1; j <= 4; j++) NB(T, g, j) = 0;
  for (int ind = 1; ind <= T->twotondim; ind++) {
    int c = CELL(T, g, ind);
    T->son[c] = 0; T->flag1[c] = 0; T->flag2[c] = 0;
    for (int v = 1; v <= NVMAX; v++) { UO(T, c, v) = 0.0; UN(T, c, v) = 0.0; }
  }
  T->next[T->tailf] = g;
  T->prev[g] = T->tailf;
  T->next[g] = 0;
  T->tailf = g;
  T->numbf++;
}

/* refine_coarse :25-160 with authorize_coarse */
static void refine_coarse(tamr *T) {
  T->flag2[0] = 0;
  for (int c = 1; c <= T->ncoarse; c++) T->flag2[c] = 1;
  for (int pass = 0; pass < 2; pass++) {
    for (int j = T->jcoarse_min; j <= T->jcoarse_max; j++)
      for (int i = T->icoarse_min; i <= T->icoarse_max; i++) {
        int c = 1 + i + j * T->nx;
        if (pass == 0 && T->flag2[c] == 1 && T->flag1[c] == 1 && T->son[c] == 0) make_grid_coarse(T, c, 0, 0);
        if (pass == 1 && T->flag1[c] == 0 && T->son[c] > 0) kill_grid(T, c, 1, 0, 0);
      }
    for (int ib = 0; ib < T->nboundary; ib++)
      for (int j = T->jbmin[ib]; j <= T->jbmax[ib]; j++)
        for (int i = T->ibmin[ib]; i <= T->ibmax[ib]; i++) {
          int c = 1 + i + j * T->nx;
          if (pass == 0 && T->flag2[c] == 1 && T->flag1[c] == 1 && T->son[c] == 0) make_grid_coarse(T, c, ib, 1);
          if (pass == 1 && T->flag1[c] == 0 && T->son[c] > 0) kill_grid(T, c, 1, ib, 1);
        }
  }
}

/* authorize_fine (virtual_boundaries.f90:34-311, one CPU) with
 * init_boundary_fine: the boundary cells next to the box may be refined */
static void authorize_fine(tamr *T, int ilevel) {
  static const int n_nbor[3] = {1, 2, 3};
  if (ilevel == T->nlevelmax) return;
  int n = level_list(T, ilevel, T->lst);
  for (int ind = 1; ind <= T->twotondim; ind++)
    for (int i = 0; i < n; i++) T->flag2[CELL(T, T->lst[i], ind)] = 1;
  T->flag2[0] = 0;
  for (int ib = 0; ib < T->nboundary; ib++) {
    int nb = bound_list(T, ib, ilevel, T->lst2);
    for (int ind = 1; ind <= T->twotondim; ind++)
      for (int i = 0; i < nb; i++) T->flag2[CELL(T, T->lst2[i], ind)] = 0;
  }
  /* init_boundary_fine */
  T->flag2[0] = 0;
  for (int ism = 0; ism < T->ndim; ism++) {
    for (int ib = 0; ib < T->nboundary; ib++) {
      int nb = bound_list(T, ib, ilevel, T->lst2);
      for (int ind = 1; ind <= T->twotondim; ind++)
        for (int i = 0; i < nb; i++) T->flag1[CELL(T, T->lst2[i], ind)] = 0;
    }
    for (int ib = 0; ib < T->nboundary; ib++) {
      int nb = bound_list(T, ib, ilevel, T->lst2);
      for (int i = 0; i < nb; i++) {
        int igridn[5];
        getnborgrids_check(T, T->lst2[i], igridn);
        for (int ind = 1; ind <= T->twotondim; ind++) {
          int indn[5], cnt = 0;
          getnborcells(T, igridn, ind, indn);
          for (int in = 1; in <= T->twondim; in++) cnt += T->flag2[indn[in]];
          if (cnt >= n_nbor[ism]) T->flag1[CELL(T, T->lst2[i], ind)] = 1;
        }
      }
    }
    for (int ib = 0; ib < T->nboundary; ib++) {
      int nb = bound_list(T, ib, ilevel, T->lst2);
      for (int ind = 1; ind <= T->twotondim; ind++)
        for (int i = 0; i < nb; i++)
          if (T->flag1[CELL(T, T->lst2[i], ind)] == 1) T->flag2[CELL(T, T->lst2[i], ind)] = 1;
    }
  }
  make_boundary_flag(T, ilevel);
}

/* make_grid_fine :590-948 for one new grid in cell ind_cell (cell ind of
 * grid ind_grid, level ilevel-1) */
static void make_grid_fine(tamr *T, int ind_grid, int ind_cell, int ind, int ilevel, int ib,
                           int boundary_region) {
  if (T->numbf <= 0) { fail1(T, "make_grid_fine: no more free memory (ngridmax)"); return; }
  int g = T->headf;
  T->headf = T->next[T->headf];
  T->numbf--;
  double dx = pow(0.5, ilevel - 1);
  XG(T, g, 1) = XG(T, ind_grid, 1) + ((double)IX(ind) - 0.5) * dx;
  XG(T, g, 2) = T->ndim > 1 ? XG(T, ind_grid, 2) + ((double)IY(ind) - 0.5) * dx : 0.0;
  T->son[ind_cell] = g;
  T->father[g] = ind_cell;
  int igridn[5], indn[5];
  getnborgrids(T, ind_grid, igridn);
  getnborcells(T, igridn, ind, indn);
  for (int j = 1; j <= T->twondim; j++) {
    NB(T, g, j) = indn[j];
    if (indn[j] == 0 && !boundary_region) fail1(T, "make_grid_fine: father cell without a same-level neighbour");
  }
  for (int ind2 = 1; ind2 <= T->twotondim; ind2++) {
    int c = CELL(T, g, ind2);
    T->son[c] = 0; T->flag1[c] = 0; T->flag2[c] = 0;
  }
  if (boundary_region) list_append(T, &T->headb[ib][ilevel], &T->tailb[ib][ilevel], &T->numbb[ib][ilevel], g);
  else list_append(T, &T->headl[ilevel], &T->taill[ilevel], &T->numbl[ilevel], g);
  if (!T->init) {
    int fz[5] = {T->father[g], NB(T, g, 1), NB(T, g, 2), NB(T, g, 3), NB(T, g, 4)};
    double u1[5][NVMAX], u2[4][NVMAX];
    for (int j = 0; j <= T->twondim; j++)
      for (int v = 1; v <= T->nv; v++) u1[j][v - 1] = fz[j] > 0 ? UO(T, fz[j], v) : 0.0;
    if (interpol_hydro(T, u1, u2)) { fail1(T, "interpol_hydro: unsupported interpol_var/interpol_type"); return; }
    for (int ind2 = 1; ind2 <= T->twotondim; ind2++)
      for (int v = 1; v <= T->nv; v++) UO(T, CELL(T, g, ind2), v) = u2[ind2 - 1][v - 1];
  }
}

/* refine_fine :332-585 (one CPU): create the sons of flagged cells of the
 * active grids, then of each boundary's grids, in nvector batches and cell
 * positions; then kill the sons of unflagged cells in the same order */
static void refine_fine(tamr *T, int ilevel) {
  if (ilevel == T->nlevelmax) return;
  if (T->numbl[ilevel] == 0) return;
  authorize_fine(T, ilevel);
  for (int kill = 0; kill < 2; kill++)
    for (int pass = 0; pass <= T->nboundary; pass++) {
      int ib = pass - 1, n = pass == 0 ? level_list(T, ilevel, T->lst2) : bound_list(T, ib, ilevel, T->lst2);
      for (int i0 = 0; i0 < n; i0 += NVEC) {
        int ng = n - i0 < NVEC ? n - i0 : NVEC;
        for (int ind = 1; ind <= T->twotondim; ind++)
          for (int i = 0; i < ng; i++) {
            int g = T->lst2[i0 + i], c = CELL(T, g, ind);
            if (!kill && T->flag2[c] == 1 && T->flag1[c] == 1 && T->son[c] == 0)
              make_grid_fine(T, g, c, ind, ilevel + 1, ib, pass > 0);
            if (kill && T->flag1[c] == 0 && T->son[c] > 0) kill_grid(T, c, ilevel + 1, ib, pass > 0);
          }
      }
    }
}

/* ---- hydro step ---- */
/* set_unew / set_uold (hydro/godunov_fine.f90:40-232, no pressure_fix) */
static void set_unew(tamr *T, int ilevel) {
  int n = level_list(T, ilevel, T->lst);
  for (int ind = 1; ind <= T->twotondim; ind++)
    for (int v = 1; v <= T->nv; v++)
      for (int i = 0; i < n; i++) UN(T, CELL(T, T->lst[i], ind), v) = UO(T, CELL(T, T->lst[i], ind), v);
}
static void set_uold(tamr *T, int ilevel) {
  int n = level_list(T, ilevel, T->lst);
  for (int ind = 1; ind <= T->twotondim; ind++)
    for (int v = 1; v <= T->nv; v++)
      for (int i = 0; i < n; i++) UO(T, CELL(T, T->lst[i], ind), v) = UN(T, CELL(T, T->lst[i], ind), v);
}

/* courant_fine (hydro/courant_fine.f90:1-159) with cmpdt
 * (hydro/godunov_utils.f90:5-120), no gravity */
static void courant_fine(tamr *T, int ilevel) {
  const double gamma = T->hp.gamma, smallc = T->hp.smallc, C = T->hp.courant_factor;
  const double half = 0.5, one = 1.0, two = 2.0, smallp = smallc * smallc / gamma;
  const int nd = T->ndim;
  double dx = pow(0.5, ilevel) * scale_of(T);
  double dt_loc = T->dtnew[ilevel];
  int n = level_list(T, ilevel, T->lst);
  for (int i0 = 0; i0 < n; i0 += NVEC) {
    int ng = n - i0 < NVEC ? n - i0 : NVEC;
    for (int ind = 1; ind <= T->twotondim; ind++) {
      int nleaf = 0;
      double dt = C * dx / smallc;
      for (int i = 0; i < ng; i++) {
        int c = CELL(T, T->lst[i0 + i], ind);
        if (T->son[c] != 0) continue;
        nleaf++;
        double d = fmaxd1(UO(T, c, 1), T->hp.smallr), v[2] = {0.0, 0.0};
        for (int idim = 1; idim <= nd; idim++) v[idim - 1] = UO(T, c, idim + 1) / d;
        double e = UO(T, c, nd + 2);
        for (int idim = 0; idim < nd; idim++) e = e - half * d * (v[idim] * v[idim]);
        double cs = fmaxd1((gamma - one) * e, d * smallp);
        cs = gamma * cs;
        cs = sqrt(cs / d);
        cs = (double)nd * cs;
        for (int idim = 0; idim < nd; idim++) cs = cs + fabs(v[idim]);
        double g0 = 0.0;
        for (int idim = 0; idim < nd; idim++) g0 = g0 + fabs(0.0);
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

/* unsplit (hydro/umuscl.f90:22-171) on one grid's stencil u[j3+1][i3+1][v]
 * (i3, j3 = -1..4; NDIM=1 uses row j3 = 1): ctoprim :861-965, uslope
 * :970-1130 (slope_type 0-2), trace1d :176-290 / trace2d, cmpflxm
 * :714-856; flux[idim][j][i][v] for the faces of the grid */
static int unsplit(tamr *T, double u[6][6][NVMAX], double dx, double dt, double flux[2][4][4][NVMAX]) {
  const double gamma = T->hp.gamma, smallr = T->hp.smallr, half = 0.5, one = 1.0;
  const double smalle = T->hp.smallc * T->hp.smallc / gamma / (gamma - one), dtxhalf = dt * half;
  const int nd = T->ndim, nv = T->nv, ip = nd + 1;
  const int jlo = nd > 1 ? -1 : 1, jhi = nd > 1 ? 4 : 1; /* ju1..ju2 */
  double q[6][6][NVMAX], dq[6][6][NVMAX][2], qm[6][6][NVMAX][2], qp[6][6][NVMAX][2];
  for (int j = jlo; j <= jhi; j++)
    for (int i = -1; i <= 4; i++) {
      double *uu = u[j + 1][i + 1], *qq = q[j + 1][i + 1];
      qq[0] = fmaxd1(uu[0], smallr);
      double oneoverrho = one / qq[0];
      for (int d = 1; d <= nd; d++) qq[d] = uu[d] * oneoverrho;
      double eken = half * qq[1] * qq[1];
      for (int d = 2; d <= nd; d++) eken = eken + half * qq[d] * qq[d];
      double erad = 0.0;
      double eint = fmaxd1(uu[ip] * oneoverrho - eken - erad, smalle);
      qq[ip] = (gamma - one) * qq[0] * eint;
      for (int d = 1; d <= nd; d++) qq[d] = qq[d] + 0.0 * dtxhalf;
    }
  const int st = T->hp.slope_type;
  if (st < 0 || st > (nd == 1 ? 3 : 2)) return -1;
  const int slo = nd > 1 ? 0 : 1, shi = nd > 1 ? 3 : 1; /* jlo..jhi of uslope/trace */
  for (int j = slo; j <= shi; j++)
    for (int i = 0; i <= 3; i++)
      for (int v = 0; v < nv; v++)
        for (int d = 0; d < nd; d++) {
          if (st == 0) { dq[j + 1][i + 1][v][d] = 0.0; continue; }
          const double k = (double)(st < 2 ? st : 2);
          const int di = d == 0, dj = d == 1;
          double dlft = k * (q[j + 1][i + 1][v] - q[j + 1 - dj][i + 1 - di][v]);
          double drgt = k * (q[j + 1 + dj][i + 1 + di][v] - q[j + 1][i + 1][v]);
          double dcen = half * (dlft + drgt) / k;
          double dsgn = copysign(one, dcen);
          double slop = fmind1(fabs(dlft), fabs(drgt));
          double dlim = slop;
          if ((dlft * drgt) <= 0.0) dlim = 0.0;
          dq[j + 1][i + 1][v][d] = dsgn * fmind1(dlim, fabs(dcen));
        }
  const double dtdx = dt / dx;
  for (int j = slo; j <= shi; j++)
    for (int i = 0; i <= 3; i++) {
      double *qq = q[j + 1][i + 1];
      double (*dd)[2] = dq[j + 1][i + 1];
      double (*pp)[2] = qp[j + 1][i + 1], (*mm)[2] = qm[j + 1][i + 1];
      double r = qq[0], uu = qq[1], p = qq[ip];
      if (nd == 1) {
        double drx = dd[0][0], dux = dd[1][0], dpx = dd[2][0];
        double sr0 = -uu * drx - (dux) * r;
        double sp0 = -uu * dpx - (dux) * gamma * p;
        double su0 = -uu * dux - (dpx) / r;
        pp[0][0] = r - half * drx + sr0 * dtdx * half;
        pp[1][0] = uu - half * dux + su0 * dtdx * half;
        pp[2][0] = p - half * dpx + sp0 * dtdx * half;
        if (pp[0][0] < smallr) pp[0][0] = r;
        mm[0][0] = r + half * drx + sr0 * dtdx * half;
        mm[1][0] = uu + half * dux + su0 * dtdx * half;
        mm[2][0] = p + half * dpx + sp0 * dtdx * half;
        if (mm[0][0] < smallr) mm[0][0] = r;
      } else {
        double v = qq[2];
        double drx = dd[0][0], dux = dd[1][0], dvx = dd[2][0], dpx = dd[3][0];
        double dry = dd[0][1], duy = dd[1][1], dvy = dd[2][1], dpy = dd[3][1];
        double sr0 = -uu * drx - v * dry - (dux + dvy) * r;
        double sp0 = -uu * dpx - v * dpy - (dux + dvy) * gamma * p;
        double su0 = -uu * dux - v * duy - (dpx) / r;
        double sv0 = -uu * dvx - v * dvy - (dpy) / r;
        const double dtdy = dtdx;
        pp[0][0] = r - half * drx + sr0 * dtdx * half;
        pp[1][0] = uu - half * dux + su0 * dtdx * half;
        pp[2][0] = v - half * dvx + sv0 * dtdx * half;
        pp[3][0] = p - half * dpx + sp0 * dtdx * half;
        if (pp[0][0] < smallr) pp[0][0] = r;
        mm[0][0] = r + half * drx + sr0 * dtdx * half;
        mm[1][0] = uu + half * dux + su0 * dtdx * half;
        mm[2][0] = v + half * dvx + sv0 * dtdx * half;
        mm[3][0] = p + half * dpx + sp0 * dtdx * half;
        if (mm[0][0] < smallr) mm[0][0] = r;
        pp[0][1] = r - half * dry + sr0 * dtdy * half;
        pp[1][1] = uu - half * duy + su0 * dtdy * half;
        pp[2][1] = v - half * dvy + sv0 * dtdy * half;
        pp[3][1] = p - half * dpy + sp0 * dtdy * half;
        if (pp[0][1] < smallr) pp[0][1] = r;
        mm[0][1] = r + half * dry + sr0 * dtdy * half;
        mm[1][1] = uu + half * duy + su0 * dtdy * half;
        mm[2][1] = v + half * dvy + sv0 * dtdy * half;
        mm[3][1] = p + half * dpy + sp0 * dtdy * half;
        if (mm[0][1] < smallr) mm[0][1] = r;
      }
    }
  /* cmpflxm per direction: faces i = 1..3 (x) on rows j = 1..2 (2D) or 1;
   * faces j = 1..3 (y) on columns i = 1..2; left state qm of the cell
   * below, right state qp of the cell above */
  for (int d = 0; d < nd; d++) {
    const int ln = d + 1, lt1 = d == 0 ? 2 : 1;
    const int ilo = 1, ihi = d == 0 ? 3 : 2;
    const int jlo2 = 1, jhi2 = nd > 1 ? (d == 0 ? 2 : 3) : 1;
    for (int j = jlo2; j <= jhi2; j++)
      for (int i = ilo; i <= ihi; i++) {
        const int di = d == 0, dj = d == 1;
        double ql[5] = {0, 0, 0, 0, 0}, qr[5] = {0, 0, 0, 0, 0}, fg[6];
        ql[0] = qm[j + 1 - dj][i + 1 - di][0][d];
        qr[0] = qp[j + 1][i + 1][0][d];
        ql[1] = qm[j + 1 - dj][i + 1 - di][ln][d];
        qr[1] = qp[j + 1][i + 1][ln][d];
        ql[2] = qm[j + 1 - dj][i + 1 - di][ip][d];
        qr[2] = qp[j + 1][i + 1][ip][d];
        if (nd > 1) {
          ql[3] = qm[j + 1 - dj][i + 1 - di][lt1][d];
          qr[3] = qp[j + 1][i + 1][lt1][d];
        }
        if (orc_riemann_face(&T->hp, ql, qr, fg)) return -2;
        double *fx = flux[d][j][i];
        fx[0] = fg[0] * dt / dx;
        fx[ln] = fg[1] * dt / dx;
        fx[ip] = fg[2] * dt / dx;
        if (nd > 1) fx[lt1] = fg[3] * dt / dx;
      }
  }
  return 0;
}

/* godunov_fine / godfine1 (hydro/godunov_fine.f90:5-35, 486-908) */
static void godunov_fine(tamr *T, int ilevel) {
  const int nd = T->ndim, nv = T->nv;
  const double oneontwotondim = 1.0 / (double)T->twotondim;
  const int jmax1 = nd > 1 ? 2 : 0, jmax2 = nd > 1 ? 1 : 0;
  double dx = pow(0.5, ilevel) * scale_of(T), dt = T->dtnew[ilevel];
  int n = level_list(T, ilevel, T->lst);
  for (int i0 = 0; i0 < n; i0 += NVEC) {
    int ng = n - i0 < NVEC ? n - i0 : NVEC;
    /* gather + unsplit per grid: independent, run on the host's threads;
     * the update and the corrections below keep the reference's order */
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < ng; i++) {
      double uloc[6][6][NVMAX];
      int g = T->lst[i0 + i], nbf[9];
      get3cubefather(T, T->father[g], ilevel, nbf);
      int32_t (*ok)[6] = T->fok[i];
      for (int j1 = 0; j1 <= jmax1; j1++)
        for (int i1 = 0; i1 <= 2; i1++) {
          int fc = nbf[i1 + 3 * j1];
          int gn = fc > 0 ? T->son[fc] : 0;
          double u2[4][NVMAX];
          if (gn <= 0) {
            if (fc <= 0) { T->perr = 1; continue; }
            int f5[5];
            getnborfather(T, fc, ilevel, f5);
            double u1[5][NVMAX];
            for (int j = 0; j <= T->twondim; j++)
              for (int v = 1; v <= nv; v++) u1[j][v - 1] = UO(T, f5[j], v);
            if (interpol_hydro(T, u1, u2)) { T->perr = 2; continue; }
          }
          for (int j2 = 0; j2 <= jmax2; j2++)
            for (int i2 = 0; i2 <= 1; i2++) {
              int ind_son = 1 + i2 + 2 * j2;
              int i3 = 1 + 2 * (i1 - 1) + i2, j3 = nd > 1 ? 1 + 2 * (j1 - 1) + j2 : 1;
              if (gn > 0) {
                int c = CELL(T, gn, ind_son);
                for (int v = 1; v <= nv; v++) uloc[j3 + 1][i3 + 1][v - 1] = UO(T, c, v);
                ok[j3 + 1][i3 + 1] = T->son[c] > 0;
              } else {
                for (int v = 1; v <= nv; v++) uloc[j3 + 1][i3 + 1][v - 1] = u2[ind_son - 1][v - 1];
                ok[j3 + 1][i3 + 1] = 0;
              }
            }
        }
      if (unsplit(T, uloc, dx, dt, T->flux[i])) { T->perr = 3; continue; }
      for (int d = 0; d < nd; d++) { /* refined-face zeroing :720-747 */
        const int i0f = d == 0, j0f = d == 1;
        for (int j3 = 1; j3 <= (nd > 1 ? 2 : 1) + j0f * (nd > 1); j3++)
          for (int i3 = 1; i3 <= 2 + i0f; i3++)
            if (ok[j3 - j0f + 1][i3 - i0f + 1] || ok[j3 + 1][i3 + 1])
              for (int v = 0; v < nv; v++) T->flux[i][d][j3][i3][v] = 0.0;
      }
    }
    if (T->perr) {
      fail1(T, T->perr == 1 ? "godunov_fine: missing father neighbour"
                            : T->perr == 2 ? "interpol_hydro: unsupported options"
                                           : "unsplit: unsupported slope_type or Riemann solver");
      return;
    }
    for (int d = 0; d < nd; d++) { /* conservative update :751-792 */
      const int i0f = d == 0, j0f = d == 1;
      for (int j2 = 0; j2 <= jmax2; j2++)
        for (int i2 = 0; i2 <= 1; i2++) {
          int ind_son = 1 + i2 + 2 * j2, i3 = 1 + i2, j3 = 1 + j2;
          for (int v = 1; v <= nv; v++)
            for (int i = 0; i < ng; i++) {
              int c = CELL(T, T->lst[i0 + i], ind_son);
              UN(T, c, v) = UN(T, c, v) + (T->flux[i][d][j3][i3][v - 1] - T->flux[i][d][j3 + j0f][i3 + i0f][v - 1]);
            }
        }
    }
    /* fine -> coarse corrections :798-908 */
    static int nbi[NVEC], nbc[NVEC];
    for (int d = 0; d < nd; d++) {
      const int i0f = d == 0, j0f = d == 1;
      const int j3max = nd > 1 ? 2 : 1;
      for (int side = 0; side < 2; side++) {
        int nnb = 0;
        for (int i = 0; i < ng; i++) {
          int c = NB(T, T->lst[i0 + i], 2 * d + 1 + side);
          if (T->son[c] == 0) { nbc[nnb] = c; nbi[nnb] = i; nnb++; }
        }
        for (int v = 1; v <= nv; v++)
          if (side == 0) {
            for (int j3 = 1; j3 <= j3max - j0f; j3++)
              for (int i3 = 1; i3 <= 2 - i0f; i3++)
                for (int k = 0; k < nnb; k++)
                  UN(T, nbc[k], v) = UN(T, nbc[k], v) - T->flux[nbi[k]][d][j3][i3][v - 1] * oneontwotondim;
          } else {
            for (int j3 = 1 + j0f; j3 <= j3max; j3++)
              for (int i3 = 1 + i0f; i3 <= 2; i3++)
                for (int k = 0; k < nnb; k++)
                  UN(T, nbc[k], v) = UN(T, nbc[k], v) + T->flux[nbi[k]][d][j3 + j0f][i3 + i0f][v - 1] * oneontwotondim;
          }
      }
    }
  }
}

/* ---- drivers ---- */
static void flag_all(tamr *T) { /* flag (flag_utils.f90:5-17) */
  for (int l = T->nlevelmax - 1; l >= 1; l--) flag_fine(T, l, 2);
  flag_coarse(T);
}
static void refine_all(tamr *T) { /* refine (refine_utils.f90:1-20) */
  refine_coarse(T);
  for (int l = 1; l <= T->nlevelmax - 1; l++) refine_fine(T, l);
}
static void init_flow(tamr *T) { /* init_flow (hydro/init_flow_fine.f90:1-20) */
  for (int l = T->nlevelmax; l >= 1; l--) {
    if (l >= T->levelmin) init_flow_fine(T, l);
    upload_fine(T, l);
    make_boundary_hydro(T, l);
  }
}

/* update_time (amr/update_time.f90:191-380): the end test, then t += dt */
static int update_time(tamr *T, int ilevel) {
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
static int amr_step(tamr *T, int ilevel, int icount, orc_amr_result *res) {
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
  if (ilevel == T->levelmin && T->P->dt_force && T->nstep_coarse < T->P->dt_force_n)
    T->dtnew[ilevel] = T->P->dt_force[T->nstep_coarse];
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
  if (ilevel == T->levelmin && res->dt_log && T->nstep_coarse < res->dt_cap)
    res->dt_log[T->nstep_coarse] = T->dtnew[ilevel];
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

static void fill_result(tamr *T, orc_amr_result *res) {
  int nleaf = 0;
  for (int l = 1; l <= T->nlevelmax; l++) {
    int n = level_list(T, l, T->lst);
    res->noct[l] = n;
    for (int i = 0; i < n; i++)
      for (int ind = 1; ind <= T->twotondim; ind++) {
        int c = CELL(T, T->lst[i], ind);
        if (T->son[c] != 0) continue;
        if (nleaf < res->capacity) {
          double x[2];
          cell_pos(T, T->lst[i], ind, l, x);
          for (int d = 0; d < T->ndim; d++) res->pos[(size_t)nleaf * T->ndim + d] = x[d];
          res->level[nleaf] = l;
          for (int v = 1; v <= T->nv; v++) res->u[(size_t)nleaf * T->nv + v - 1] = UO(T, c, v);
        }
        nleaf++;
      }
  }
  res->ncell = nleaf;
  res->t = T->t;
  res->nstep = T->nstep;
  res->nstep_coarse = T->nstep_coarse;
}

/* coarse grid and boundary regions (hydro/read_hydro_params.f90:310-400) */
static int setup_boundaries(tamr *T, const orc_amr_params *P) {
  T->nx = 1; T->ny = 1;
  for (int i = 0; i < P->nboundary; i++) {
    if (P->ibound_min[i] * P->ibound_max[i] == 1 && P->bound_type[i] > 0) {
      T->nx += 1;
      if (P->ibound_min[i] == -1) { T->icoarse_min += 1; T->icoarse_max += 1; }
    }
  }
  for (int i = 0; i < P->nboundary; i++) {
    if (P->jbound_min[i] * P->jbound_max[i] == 1 && T->ndim > 1 && P->bound_type[i] > 0) {
      T->ny += 1;
      if (P->jbound_min[i] == -1) { T->jcoarse_min += 1; T->jcoarse_max += 1; }
    }
  }
  for (int i = 0; i < P->nboundary; i++) {
    int bt = P->bound_type[i];
    if (bt != 1 && bt != 2) return -1;
    if (P->ibound_min[i] * P->ibound_max[i] == 1) {
      if (P->ibound_min[i] == -1) {
        T->ibmin[i] = T->icoarse_min - 1; T->ibmax[i] = T->icoarse_min - 1;
        T->boundary_type[i] = bt == 1 ? 1 : 11;
      } else {
        T->ibmin[i] = T->icoarse_max + 1; T->ibmax[i] = T->icoarse_max + 1;
        T->boundary_type[i] = bt == 1 ? 2 : 12;
      }
      T->jbmin[i] = T->jcoarse_min + (T->ndim > 1 ? P->jbound_min[i] : 0);
      T->jbmax[i] = T->jcoarse_max + (T->ndim > 1 ? P->jbound_max[i] : 0);
    } else if (T->ndim > 1 && P->jbound_min[i] * P->jbound_max[i] == 1) {
      T->ibmin[i] = T->icoarse_min + P->ibound_min[i];
      T->ibmax[i] = T->icoarse_max + P->ibound_max[i];
      if (P->jbound_min[i] == -1) {
        T->jbmin[i] = T->jcoarse_min - 1; T->jbmax[i] = T->jcoarse_min - 1;
        T->boundary_type[i] = bt == 1 ? 3 : 13;
      } else {
        T->jbmin[i] = T->jcoarse_max + 1; T->jbmax[i] = T->jcoarse_max + 1;
        T->boundary_type[i] = bt == 1 ? 4 : 14;
      }
    } else {
      return -1;
    }
    if (T->ibmin[i] < 0 || T->ibmax[i] > T->nx - 1 || T->jbmin[i] < 0 || T->jbmax[i] > T->ny - 1) return -1;
  }
  T->nboundary = P->nboundary;
  return 0;
}

int orc_amr_run(const orc_amr_params *P, orc_amr_result *res) {
  if (P && P->dt_force && P->levelmin != P->nlevelmax) return -1;
  if (!P || !res || (P->ndim != 1 && P->ndim != 2) || P->nlevelmax < 1 || P->nlevelmax > ORC_MAXLEVEL ||
      P->levelmin < 1 || P->levelmin > P->nlevelmax || P->ngridmax < 4 || P->nboundary < 0 ||
      P->nboundary > NB_MAX || P->nregion < 0 || P->nregion > ORC_AMR_MAXREGION)
    return -1;
  tamr T;
  memset(&T, 0, sizeof T);
  T.P = P;
  T.hp = P->hydro;
  T.ndim = P->ndim;
  T.nv = P->ndim + 2;
  T.twotondim = 1 << P->ndim;
  T.twondim = 2 * P->ndim;
  T.threetondim = P->ndim == 1 ? 3 : 9;
  T.nlevelmax = P->nlevelmax;
  T.levelmin = P->levelmin;
  T.ngridmax = P->ngridmax;
  if (setup_boundaries(&T, P)) return -1;
  T.ncoarse = T.nx * T.ny;
  T.ncell = T.ncoarse + T.twotondim * T.ngridmax;
  T.son = calloc((size_t)T.ncell + 1, sizeof(int32_t));
  T.flag1 = calloc((size_t)T.ncell + 1, sizeof(int32_t));
  T.flag2 = calloc((size_t)T.ncell + 1, sizeof(int32_t));
  T.father = calloc((size_t)T.ngridmax + 1, sizeof(int32_t));
  T.next = calloc((size_t)T.ngridmax + 1, sizeof(int32_t));
  T.prev = calloc((size_t)T.ngridmax + 1, sizeof(int32_t));
  T.nbor = calloc(((size_t)T.ngridmax + 1) * 4, sizeof(int32_t));
  T.xg = calloc(((size_t)T.ngridmax + 1) * 2, sizeof(double));
  T.uold = calloc(((size_t)T.ncell + 1) * NVMAX, sizeof(double));
  T.unew = calloc(((size_t)T.ncell + 1) * NVMAX, sizeof(double));
  T.lst = calloc((size_t)T.ngridmax + 1, sizeof(int32_t));
  T.lst2 = calloc((size_t)T.ngridmax + 1, sizeof(int32_t));
  T.flux = calloc(NVEC, sizeof *T.flux);
  T.fok = calloc(NVEC, sizeof *T.fok);
  int rc = 0;
  if (!T.son || !T.flag1 || !T.flag2 || !T.father || !T.next || !T.prev || !T.nbor || !T.xg || !T.uold ||
      !T.unew || !T.lst || !T.lst2 || !T.flux || !T.fok) {
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
  free(T.flux); free(T.fok);
  return rc;
}
