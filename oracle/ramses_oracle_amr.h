/*
 * ramses_oracle_amr.h -- TEST INFRASTRUCTURE ONLY: a whole RAMSES hydro run
 * restated for NDIM=1 and NDIM=2 (see ramses_oracle_amr.c), used to pin the
 * oracle's restatement against the reference's own regression checksums.
 */
#ifndef RAMSES_ORACLE_AMR_H
#define RAMSES_ORACLE_AMR_H
#include <stdint.h>

#include "ramses_oracle.h"

#define ORC_AMR_MAXREGION 8
#define ORC_AMR_MAXBOUND 4

/* &RUN_PARAMS, &AMR_PARAMS, &BOUNDARY_PARAMS, &INIT_PARAMS ('square'
 * regions), &OUTPUT_PARAMS (the last output time), &HYDRO_PARAMS and
 * &REFINE_PARAMS of a 1D or 2D run; level-dependent arrays are given per
 * level, as RAMSES holds them after read_params */
typedef struct orc_amr_params {
  orc_params hydro;
  orc_refine refine;
  int32_t ndim; /* 1 or 2 */
  int32_t levelmin, nlevelmax, ngridmax;
  int32_t nexpand[ORC_MAXLEVEL + 1];   /* nexpand(ilevel) at [ilevel] */
  int32_t nsubcycle[ORC_MAXLEVEL + 1]; /* nsubcycle(ilevel) at [ilevel] */
  double boxlen, tout;
  int32_t nboundary;                   /* 0 (periodic) .. 4 */
  /* namelist ibound_min/max, jbound_min/max (-1, 0, +1) and bound_type
   * (1 reflexive, 2 outflow) of each boundary region */
  int32_t ibound_min[ORC_AMR_MAXBOUND], ibound_max[ORC_AMR_MAXBOUND];
  int32_t jbound_min[ORC_AMR_MAXBOUND], jbound_max[ORC_AMR_MAXBOUND];
  int32_t bound_type[ORC_AMR_MAXBOUND];
  int32_t nregion;
  double x_center[ORC_AMR_MAXREGION], y_center[ORC_AMR_MAXREGION];
  double length_x[ORC_AMR_MAXREGION], length_y[ORC_AMR_MAXREGION], exp_region[ORC_AMR_MAXREGION];
  double d_region[ORC_AMR_MAXREGION], u_region[ORC_AMR_MAXREGION], v_region[ORC_AMR_MAXREGION];
  double p_region[ORC_AMR_MAXREGION];
  int64_t max_coarse_steps;
  /* optional, for one complete level (levelmin = nlevelmax): the time step
   * of coarse step k is dt_force[k] instead of courant_fine's, k < dt_force_n */
  const double *dt_force;
  int64_t dt_force_n;
} orc_amr_params;

typedef struct orc_amr_result {
  int32_t capacity;  /* in: room for leaf cells in pos, level, u */
  int32_t init_only; /* in: stop after the initial refinement */
  double *pos;       /* out: leaf-cell centres, ndim per cell */
  int32_t *level;    /* out: leaf-cell levels */
  double *u;         /* out: leaf-cell conservative state, ndim+2 per cell */
  int32_t ncell;     /* out: leaf cells (may exceed capacity) */
  int32_t taken;     /* out: the snapshot at t >= tout was reached */
  double t;
  int64_t nstep, nstep_coarse;
  int32_t noct[ORC_MAXLEVEL + 1]; /* out: active grids per level */
  char message[160];
  double *dt_log;    /* in (optional): the dt of each coarse step's levelmin
                        godunov_fine, dt_cap entries at most */
  int32_t dt_cap;
} orc_amr_result;

#ifdef __cplusplus
extern "C" {
#endif
/* Runs init_refine, init_refine_2 and adaptive_loop until the first coarse
 * step that starts at t >= tout (where the reference writes its snapshot
 * after that step's refinement); returns 0, or < 0 with res->message. */
int orc_amr_run(const orc_amr_params *p, orc_amr_result *res);
#ifdef __cplusplus
}
#endif
#endif
