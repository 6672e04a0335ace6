/* rb_types.h -- plain-C parameter structs shared by the C ABI, the host
 * runtime and the device kernels. The public header include/ramses_b200.h
 * includes this file. */
#ifndef RB_TYPES_H
#define RB_TYPES_H
#include <stdint.h>

#define RB_NVAR 5
#define RB_MAXLEVEL 32

enum { RB_RIEMANN_LLF = 1, RB_RIEMANN_HLL = 2, RB_RIEMANN_HLLC = 3, RB_RIEMANN_ACOUSTIC = 4, RB_RIEMANN_EXACT = 5 };
enum { RB_PREC_FP64 = 0, RB_PREC_MIXED = 1 };
enum { RB_SCHEME_MUSCL = 0, RB_SCHEME_PLMDE = 1 };

/* Status codes returned by every C-ABI entry point (0 = success). */
enum {
  RB_OK = 0,
  RB_ERR_INVALID = 1,     /* bad argument / unsupported namelist value     */
  RB_ERR_STATE = 2,       /* call out of order (no init, no tree, ...)     */
  RB_ERR_CUDA = 3,        /* CUDA runtime error                             */
  RB_ERR_NOMEM = 4,       /* device or host allocation failed               */
  RB_ERR_TREE = 5,        /* octree violates the nesting rule               */
  RB_ERR_NUMERIC = 6,     /* non-finite or non-positive state detected      */
  RB_ERR_NO_DEVICE = 7,   /* no CUDA device / kernel image for this GPU     */
  RB_ERR_CAPACITY = 8     /* request above a fixed capacity                 */
};

/* &HYDRO_PARAMS values consumed by the hydro step
 * (hydro/hydro_parameters.f90:74-89). Strings are passed as codes. */
typedef struct rb_hydro_params {
  double gamma;
  double smallr;
  double smallc;
  double courant_factor;
  double slope_theta;
  int32_t riemann;       /* RB_RIEMANN_*                                    */
  int32_t slope_type;    /* 0,1,2,3,7,8                                    */
  int32_t scheme;        /* RB_SCHEME_MUSCL ('muscl') or RB_SCHEME_PLMDE     */
  int32_t interpol_var;  /* 0,1,2                                          */
  int32_t interpol_type; /* 0..4                                           */
  int32_t pressure_fix;  /* 1: dual-energy fix (enew/divu tracked, set_uold  */
                         /*    repairs E where E - ekin is too small)       */
  double difmag;         /* artificial diffusion coefficient, >= 0 (0: off)  */
  double beta_fix;       /* pressure-fix threshold, >= 0 (default 0)       */
  int32_t niter_riemann; /* Newton iterations of the 'exact' solver (10)    */
  int32_t pad_;          /* zero                                            */
} rb_hydro_params;

/* Gradient refinement criterion of &REFINE_PARAMS
 * (hydro/read_hydro_params.f90:59-60; defaults hydro/hydro_parameters.f90:47-52:
 * err_grad_* = -1 (off), floor_* = 1e-10). A criterion is on when its
 * err_grad_* >= 0. */
typedef struct rb_refine_params {
  double err_grad_d;     /* relative density gradient threshold            */
  double err_grad_p;     /* relative pressure gradient threshold           */
  double err_grad_u;     /* relative velocity gradient threshold           */
  double floor_d, floor_u, floor_p;
} rb_refine_params;

/* &AMR_PARAMS / &RUN_PARAMS values and the tree dimensions
 * (amr/amr_parameters.f90, amr/amr_commons.f90). */
typedef struct rb_mesh_params {
  int32_t nx, ny, nz;          /* coarse grid                              */
  int32_t ncoarse;             /* nx*ny*nz                                 */
  int32_t ngridmax;            /* oct capacity                             */
  int32_t nlevelmax;
  int32_t levelmin;
  int32_t nvector;             /* host vector-sweep width (batch order)    */
  double boxlen;
  int32_t nsubcycle[RB_MAXLEVEL + 1]; /* index = level (1-based)          */
  int32_t nx_loc;              /* icoarse_max-icoarse_min+1: coarse cells   */
                               /* across the box without boundary layers   */
                               /* (dx = 0.5**l * boxlen/nx_loc); 0: nx     */
  int32_t pad_;                /* zero                                     */
} rb_mesh_params;

#endif
