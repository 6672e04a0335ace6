/*
 * ramses_oracle_1d.h -- TEST INFRASTRUCTURE ONLY: a whole RAMSES hydro run
 * restated for NDIM=1 (see ramses_oracle_1d.c), used to pin the oracle's
 * restatement against the reference's 1D regression checksums.
 */
#ifndef RAMSES_ORACLE_1D_H
#define RAMSES_ORACLE_1D_H
#include <stdint.h>

#include "ramses_oracle.h"

#define ORC1D_MAXREGION 8

/* &RUN_PARAMS, &AMR_PARAMS, &BOUNDARY_PARAMS, &INIT_PARAMS ('square'
 * regions), &OUTPUT_PARAMS (one output time), &HYDRO_PARAMS and
 * &REFINE_PARAMS of a 1D run */
typedef struct orc1d_params {
  orc_params hydro;
  orc_refine refine;
  int32_t levelmin, nlevelmax, ngridmax, nexpand;
  int32_t nsubcycle[ORC_MAXLEVEL + 1]; /* nsubcycle(ilevel) at [ilevel] */
  double boxlen, tout;
  int32_t nboundary;                   /* 0 (periodic) .. 2 */
  int32_t bound_side[2];               /* ibound_min = ibound_max: -1 (x min) or +1 (x max) */
  int32_t bound_type[2];               /* namelist bound_type: 1 reflexive, 2 outflow */
  int32_t nregion;
  double x_center[ORC1D_MAXREGION], length_x[ORC1D_MAXREGION], exp_region[ORC1D_MAXREGION];
  double d_region[ORC1D_MAXREGION], u_region[ORC1D_MAXREGION], p_region[ORC1D_MAXREGION];
  int64_t max_coarse_steps;
} orc1d_params;

typedef struct orc1d_result {
  int32_t capacity;  /* in: room for leaf cells in x, level, u */
  int32_t init_only; /* in: stop after the initial refinement */
  double *x;         /* out: leaf-cell centres */
  int32_t *level;    /* out: leaf-cell levels */
  double *u;         /* out: leaf-cell (rho, rho u, E), 3 per cell */
  int32_t ncell;     /* out: leaf cells (may exceed capacity) */
  int32_t taken;     /* out: the snapshot at t >= tout was reached */
  double t;
  int64_t nstep, nstep_coarse;
  int32_t noct[ORC_MAXLEVEL + 1]; /* out: active grids per level */
  char message[160];
} orc1d_result;

#ifdef __cplusplus
extern "C" {
#endif
/* Runs init_refine, init_refine_2 and adaptive_loop until the first coarse
 * step that starts at t >= tout (where the reference writes its snapshot
 * after that step's refinement); returns 0, or < 0 with res->message. */
int orc1d_run(const orc1d_params *p, orc1d_result *res);
#ifdef __cplusplus
}
#endif
#endif
