/*
 * ramses_oracle.h -- CPU restatement of RAMSES's unsplit MUSCL-Hancock hydro
 * step (NDIM=3, NENER=0, nvar=5, real*8), used ONLY as test infrastructure:
 * the parity checker for the CUDA library and the timed CPU baseline.
 * Nothing in the product library links or calls this code.
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists in
 * the build image, so this restatement could not be compiled against the
 * reference binary. It is pinned (a) line by line to the cited Fortran,
 * (b) through its NDIM=1/2 companion (ramses_oracle_amr.c, which shares
 * the Riemann solvers) to the reference's own regression checksums of the
 * 1D AMR Sod run and the 2D AMR implosion (tests/hydro/sod-tube,
 * tests/hydro/implosion: same trees, sums within the checker's 3e-13), and (c)
 * physically to the reference's Sod known-answer file (sod-tube-ana.dat).
 * 3D bit-level parity with the Fortran binary is unpinned.
 *
 * Array conventions follow the Fortran ones exactly (column-major, 1-based
 * cell / grid indices stored as int32):
 *   uold/unew(1:ncell,1:nvar)      -> u[(ivar-1)*ncell + (icell-1)]
 *   son(1:ncell)                   -> son[icell-1]
 *   father(1:ngridmax)             -> father[igrid-1]
 *   nbor(1:ngridmax,1:6)           -> nbor[(j-1)*ngridmax + (igrid-1)]
 *   icell = ncoarse + (ind-1)*ngridmax + igrid   (ind = 1..8 child slot)
 */
#ifndef RAMSES_ORACLE_H
#define RAMSES_ORACLE_H
#include <stdint.h>

#define ORC_NVAR 5
#define ORC_MAXLEVEL 32

enum { ORC_RIEMANN_LLF = 1, ORC_RIEMANN_HLL = 2, ORC_RIEMANN_HLLC = 3, ORC_RIEMANN_ACOUSTIC = 4, ORC_RIEMANN_EXACT = 5 };

typedef struct orc_params {
  double gamma, smallr, smallc, courant_factor, slope_theta;
  int32_t riemann;       /* ORC_RIEMANN_* */
  int32_t slope_type;    /* 0,1,2,3,7,8 */
  int32_t interpol_var;  /* 0,1,2 */
  int32_t interpol_type; /* 0..4 */
  int32_t pressure_fix;  /* dual-energy fix: enew/divu tracked, set_uold repairs E */
  double beta_fix;       /* pressure-fix threshold (amr/amr_parameters.f90:167) */
  int32_t niter_riemann; /* Newton iterations of riemann_approx (hydro_parameters.f90:75) */
  double difmag;         /* artificial diffusion where the flow converges (0: off) */
  int32_t scheme;        /* 0: 'muscl' (trace3d), 1: 'plmde' (tracexyz) */
} orc_params;

/* &REFINE_PARAMS gradient criterion (hydro/hydro_parameters.f90:47-52) */
typedef struct orc_refine {
  double err_grad_d, err_grad_p, err_grad_u;
  double floor_d, floor_u, floor_p;
} orc_refine;

typedef struct orc_mesh {
  int32_t nx, ny, nz, ncoarse, ngridmax, nlevelmax, levelmin, nvector;
  double boxlen;
  int32_t *son, *father, *nbor;
  int32_t *active;      /* concatenated active(ilevel)%igrid lists        */
  int64_t *active_off;  /* [nlevelmax+2]; level l list = [off[l],off[l+1]) */
  double *uold, *unew;
  int32_t nsubcycle[ORC_MAXLEVEL + 1];
  double dtnew[ORC_MAXLEVEL + 1], dtold[ORC_MAXLEVEL + 1];
  double t;
  int64_t nstep;
  double mass_tot, ekin_tot, eint_tot;
  int64_t cell_updates; /* leaf-cell updates accumulated by orc_coarse_step */
  int32_t nthreads;     /* OpenMP threads for the flux phase (0 = default) */
  double *divu, *enew;  /* divu(1:ncell), enew(1:ncell); used when pressure_fix */
  /* physical boundaries (amr/amr_commons.f90 boundary(ibound,ilevel),
   * hydro/read_hydro_params.f90:310-420); nboundary = 0: periodic box */
  int32_t nx_loc;                /* icoarse_max-icoarse_min+1 (0: nx)         */
  int32_t nboundary;
  const int32_t *boundary_type;  /* [nboundary]: 1-6 wall, 11-16 free          */
  const int64_t *bound_off;      /* [nlevelmax*nboundary+1]: the grids of
                                    (ilevel, ibound) are bound_igrid[off[k]..off[k+1])
                                    with k = (ilevel-1)*nboundary + ibound-1   */
  const int32_t *bound_igrid;
} orc_mesh;

#ifdef __cplusplus
extern "C" {
#endif

/* umuscl.f90:22-171 with Fortran-layout arrays:
 * uin(nvector,-1:4,-1:4,-1:4,5), gravin(nvector,-1:4,-1:4,-1:4,3),
 * flux(nvector,1:3,1:3,1:3,5,3), tmp(nvector,1:3,1:3,1:3,2,3). */
int orc_unsplit(const orc_params *p, const double *uin, const double *gravin,
                double *flux, double *tmp, double dx, double dy, double dz,
                double dt, int ngrid, int nvector);

/* godunov_utils.f90:5-120 (cmpdt) for ncell cells, uu(nvector,5) layout. */
double orc_cmpdt(const orc_params *p, double *uu, const double *gg, double dx,
                 int ncell, int nvector);

/* Level operations on the mesh (godunov_fine.f90, courant_fine.f90,
 * interpol_hydro.f90). */
int orc_set_unew(const orc_params *p, orc_mesh *m, int ilevel);
int orc_set_uold(const orc_params *p, orc_mesh *m, int ilevel);
int orc_godunov_fine(const orc_params *p, orc_mesh *m, int ilevel, double dt);
int orc_courant_fine(const orc_params *p, orc_mesh *m, int ilevel,
                     double *dt_io, double *mass, double *ekin, double *eint);
int orc_upload_fine(const orc_params *p, orc_mesh *m, int ilevel);

/* amr_step.f90 hydro call sequence for one coarse step (levelmin .. finest),
 * followed by the restriction of levels levelmin-1..1 (adaptive_loop.f90). */
/* make_boundary_hydro(ilevel): hydro/hydro_boundary.f90:5-260 (wall and
 * free boundaries; imposed ones return -1). */
int orc_make_boundary_hydro(const orc_params *p, orc_mesh *m, int ilevel);
int orc_coarse_step(const orc_params *p, orc_mesh *m);

/* nbors_utils.f90:5-194 for one father cell: the 27 neighbouring father
 * cells (1-based cell indices) of cell ind_cell_father at level ilevel-1. */
int orc_get3cubefather(const orc_mesh *m, int ind_cell_father, int ilevel,
                       int32_t *nbors_father_cells27);

/* nbors_utils.f90:404-525: cell + 6 neighbour (or neighbour-father) cells. */
int orc_getnborfather(const orc_mesh *m, int ind_cell, int ilevel,
                      int32_t *ind_father7);

/* hydro_flag (hydro/hydro_flag.f90:1-180) with hydro_refine
 * (hydro/godunov_utils.f90:125-263) on level ilevel: flag1[icell] = 1 for the
 * cells meeting the gradient criterion (flag1 indexed 0..ncell, as flag1(0:ncell));
 * returns the number of cells newly flagged. */
int64_t orc_hydro_flag(const orc_params *p, const orc_refine *r, const orc_mesh *m, int ilevel, int32_t *flag1);

/* One coarse step of a complete level held as a dense grid u[v][z][y][x]:
 * courant_fine's dt, then godfine1 on every oct with a periodic or outflow
 * (zero-gradient) boundary per axis (bit d of bc_outflow set: axis d
 * outflow). u is advanced in place; dt_out receives the step's dt. */
int orc_dense_step(const orc_params *p, double *u, int nx, int ny, int nz, double dx, double dt_max,
                   int bc_outflow, int nvector, double *dt_out);

/* One Riemann problem of cmpflxm (umuscl.f90:791-803) in the face frame
 * (rho, u_n, p, u_t1, u_t2) with the solver p->riemann: fg[0..2] mass,
 * normal-momentum and energy fluxes (fg has room for 6). */
int orc_riemann_face(const orc_params *p, const double *ql, const double *qr, double *fg);

/* interpol_hydro.f90:268-444 for nn father stencils:
 * u1(nn,0:6,5) -> u2(nn,1:8,5), column-major with leading dim nn. */
int orc_interpol_hydro(const orc_params *p, double *u1, double *u2, int nn);

#ifdef __cplusplus
}
#endif
#endif
