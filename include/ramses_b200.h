/*
 * ramses_b200.h -- C ABI of the B200 hydro step (RAMSES unsplit MUSCL-Hancock,
 * NDIM=3, nvar=5). Plain pointers, sizes and status codes; no C++ or torch
 * types. Every entry point returns an int status (RB_OK = 0); the text of the
 * last error of the calling thread is available from rb_last_error().
 *
 * Array conventions at this boundary are RAMSES's own (Fortran column-major,
 * 1-based cell and grid indices stored as int32):
 *   uold(1:ncell,1:5)  : double[5*ncell], element (icell,ivar) at (ivar-1)*ncell+icell-1
 *   son(1:ncell)       : int32[ncell]
 *   father(1:ngridmax) : int32[ngridmax]
 *   nbor(1:ngridmax,6) : int32[6*ngridmax]
 *   icell = ncoarse + (ind-1)*ngridmax + igrid, ind = 1..8
 * The state lives on the GPU between calls (device-resident mirrors); the host
 * copy is only read or written by rb_upload_state / rb_download_state.
 *
 * Reference interfaces replaced (paths within ramses-organisation/ramses):
 *   godunov_fine(ilevel)               hydro/godunov_fine.f90:5-35   -> rb_godunov_fine
 *   unsplit(uin,gravin,pin,flux,tmp,dx,dy,dz,dt,ngrid)
 *                                      hydro/umuscl.f90:22-171        -> rb_unsplit
 *   courant_fine(ilevel)               hydro/courant_fine.f90:1-159   -> rb_courant_fine
 *   set_unew(ilevel)                   hydro/godunov_fine.f90:40-130  -> rb_set_unew
 *   set_uold(ilevel)                   hydro/godunov_fine.f90:135-232 -> rb_set_uold
 *   upload_fine(ilevel)                hydro/interpol_hydro.f90:5-68  -> rb_upload_fine
 *   amr_step hydro sequence            amr/amr_step.f90:320-445       -> rb_coarse_step
 *   make_boundary_hydro(ilevel)        hydro/hydro_boundary.f90:5-260 -> rb_make_boundary_hydro
 *   boundary(ibound,ilevel) lists      amr/amr_commons.f90, hydro/read_hydro_params.f90:310-420
 *                                                                     -> rb_set_boundary
 *   &HYDRO_PARAMS                      hydro/read_hydro_params.f90:43-54 -> rb_hydro_params
 */
#ifndef RAMSES_B200_H
#define RAMSES_B200_H

#include <stdint.h>

#include "../ramses_b200/csrc/rb_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rb_context rb_context;

/* Library version string. */
const char *rb_version(void);
/* Human-readable text for a status code. */
const char *rb_status_string(int status);
/* Text of the calling thread's last error (empty if none). */
const char *rb_last_error(void);
/* Number of visible CUDA devices (0 when none); never fails. */
int rb_device_count(void);
/* Make `device` the calling thread's current device for rb_create. */
int rb_select_device(int device);

/* Create a context on the current CUDA device. precision = RB_PREC_FP64
 * (drop-in) or RB_PREC_MIXED (FP32 slopes/trace/Riemann, FP64 state).
 * Replaces the namelist read (read_hydro_params.f90:43-54,138) + init_hydro
 * allocation (init_hydro.f90:31-32). Unsupported namelist values are rejected. */
int rb_create(const rb_hydro_params *hp, const rb_mesh_params *mp, int precision, rb_context **out);
int rb_destroy(rb_context *ctx);

/* Upload the octree (son, father, nbor as RAMSES stores them) and the active
 * grid lists: numbl[l-1] octs at level l, concatenated 1-based igrids in
 * active_igrid. Builds the device tile and interpolation tables. On a
 * re-sync with a state resident (and no newer host state noted), the octs
 * that are new since the previous tree (a level they did not have, or
 * another father cell) get make_grid_fine's state on the device: the
 * interpol_hydro prolongation of their father cell and its getnborfather
 * neighbours, level by level (amr/refine_utils.f90:590-948,
 * hydro/interpol_hydro.f90:268-444), so a remesh needs no state upload. */
int rb_sync_tree(rb_context *ctx, const int32_t *son, const int32_t *father, const int32_t *nbor,
                 const int32_t *numbl, const int32_t *active_igrid);

/* Physical boundaries (simple_boundary): the boundary regions' codes
 * boundary_type(1:nboundary) (1-6 walls, 11-16 free = zero-gradient, side
 * 1..6 = -x,+x,-y,+y,-z,+z; imposed 21-26 are rejected), the grid counts
 * numbb(1:nboundary,1:nlevelmax) (Fortran order) and the grids of
 * boundary(ibound,ilevel)%igrid concatenated level by level, boundary by
 * boundary within a level. The boundary octs are found by the stencil
 * gathers and never updated; mesh params nx_loc gives the coarse cells
 * across the box. Call it before rb_sync_tree, which takes the lists with
 * the tree; a tree synchronised earlier is dropped and must be synchronised
 * again. nboundary = 0 restores a periodic box. */
int rb_set_boundary(rb_context *ctx, int32_t nboundary, const int32_t *boundary_type, const int32_t *numbb,
                    const int32_t *boundary_igrid);
/* make_boundary_hydro(ilevel): fill the boundary octs of ilevel from their
 * reference octs (hydro/hydro_boundary.f90:5-260). rb_coarse_step, rb_run and
 * rb_uniform_run call it after each level step (amr/amr_step.f90:515); the
 * host calls it where the reference's init_flow_fine does. */
int rb_make_boundary_hydro(rb_context *ctx, int ilevel);

/* Fortran-layout uold(ncell,5) host <-> device mirror of uold. */
int rb_upload_state(rb_context *ctx, const double *uold);
int rb_download_state(rb_context *ctx, double *uold);
/* Only the rows of uold(ncell,5) that belong to the octs of level ilevel
 * (icell = ncoarse+(ind-1)*ngridmax+igrid, igrid in active(ilevel)%igrid:
 * the cells the level routines read and write, e.g. set_uold,
 * hydro/godunov_fine.f90:135-232), host <-> device; every other row keeps
 * its value on both sides. One copy per run of consecutive igrids, variable
 * and cell position. The tree and the whole state must have been uploaded
 * once (rb_sync_tree, rb_upload_state). */
int rb_upload_level_state(rb_context *ctx, int ilevel, const double *uold);
int rb_download_level_state(rb_context *ctx, int ilevel, double *uold);

/* Residency protocol of the drop-in boundary. The reference keeps uold and
 * the tree in host memory and every hydro routine reads them there
 * (amr/amr_step.f90:320-445); here the device copy stays authoritative across
 * hydro calls, and host code that reads or writes uold or changes the tree
 * says so:
 *   rb_note_tree_changed: the host changed son/father/nbor/active or the
 *     boundary lists (refine_fine, amr/refine_utils.f90:332-585; load_balance
 *     and defrag, amr/load_balance.f90); bumps a generation counter.
 *   rb_note_host_state_written: the host wrote uold (initial conditions,
 *     restart, load balancing); the host copy is the newer one.
 *   rb_ensure_device: before a device hydro call: re-synchronises the tree
 *     (rb_set_boundary + rb_sync_tree) when the generation changed, then
 *     uploads uold only when the host copy is newer (or none is resident).
 *     The tree and boundary arrays are read only when a re-sync is due, which
 *     rb_tree_needs_sync tells (a caller may pass placeholders otherwise).
 *   rb_ensure_host: before host code reads uold (output, flag criteria
 *     evaluated on the host): downloads only when the device copy is newer.
 * Every device call that writes uold (set_uold, upload_fine,
 * make_boundary_hydro, coarse steps, runs, new-oct prolongation) makes the
 * device copy the newer one; rb_upload_state / rb_download_state make them
 * equal. rb_transfer_stats reports the uold bytes moved each way, the tree
 * synchronisations and the octs prolonged on the device. */
int rb_note_tree_changed(rb_context *ctx);
int rb_note_host_state_written(rb_context *ctx);
int rb_tree_needs_sync(rb_context *ctx, int32_t *needed);
int rb_ensure_device(rb_context *ctx, const int32_t *son, const int32_t *father, const int32_t *nbor,
                     const int32_t *numbl, const int32_t *active_igrid, int32_t nboundary,
                     const int32_t *boundary_type, const int32_t *numbb, const int32_t *boundary_igrid,
                     const double *uold);
int rb_ensure_host(rb_context *ctx, double *uold);
int rb_transfer_stats(rb_context *ctx, int64_t *h2d_state_bytes, int64_t *d2h_state_bytes, int64_t *tree_syncs,
                      int64_t *octs_prolonged);
/* The last tree synchronisation (rb_sync_tree, or the one rb_ensure_device
 * ran): ms[5] host wall time of the whole sync, of the per-level position
 * indexes (with the son mirror), of the level tables, of the boundary pairs
 * and of the device prolongation of new octs; the levels whose tables were
 * rebuilt and those kept. A re-sync keeps a level's tables when their inputs
 * are unchanged: the level's active list and boundary octs, the positions and
 * nbor rows of the octs of that level and the next coarser one, and son of the
 * coarser level's cells (compared exactly). Replaces the per-remesh rebuild
 * that refine_fine's callers would otherwise pay (amr/refine_utils.f90:332-948
 * changes the tree; make_grid_fine's new octs are prolonged on the device). */
int rb_sync_stats(rb_context *ctx, double *ms, int32_t *levels_built, int32_t *levels_reused);
/* Same for unew (for callers that interleave host work with a level step). */
int rb_upload_unew(rb_context *ctx, const double *unew);
int rb_download_unew(rb_context *ctx, double *unew);
/* pressure_fix: Fortran-layout divu(ncell) and enew(ncell)
 * (hydro/hydro_commons.f90 divu, enew) as the last set_unew / godunov_fine /
 * set_uold left them. RB_ERR_STATE for a context without pressure_fix. */
int rb_download_pressure_fix(rb_context *ctx, double *divu, double *enew);

/* Level operations on the device mirrors (same semantics as the Fortran). */
int rb_set_unew(rb_context *ctx, int ilevel);
int rb_set_uold(rb_context *ctx, int ilevel);
int rb_godunov_fine(rb_context *ctx, int ilevel, double dt);
int rb_upload_fine(rb_context *ctx, int ilevel);
/* dt_io: in = current dtnew(ilevel); out = min(in, CFL dt of the level's leaf
 * cells). mass/ekin/eint: the level's totals (any may be NULL). */
int rb_courant_fine(rb_context *ctx, int ilevel, double *dt_io, double *mass, double *ekin, double *eint);
/* hydro_flag(ilevel) (hydro/hydro_flag.f90:1-180 with hydro_refine,
 * hydro/godunov_utils.f90:125-263) on the device state: every cell of level
 * ilevel's octs whose relative density, pressure or velocity jump to a face
 * neighbour exceeds the rb_refine_params thresholds gets flag1[icell] = 1.
 * flag1 is the host's flag1(0:ncell) (int32, indexed by the Fortran cell
 * index); other entries are left as they are, as in the reference. Only one
 * byte per cell of the level crosses PCIe, not uold. nflag_added (may be
 * NULL) receives the number of cells that went from 0 to 1. Does nothing on
 * the finest level, on an empty level or with every criterion off. */
int rb_hydro_flag(rb_context *ctx, int ilevel, const rb_refine_params *rp, int32_t *flag1, int64_t *nflag_added);

/* One coarse time step: the amr_step(levelmin) hydro call sequence with
 * subcycling, followed by the restriction of levels levelmin-1..1. t_io is
 * advanced by the step; dtnew_out (may be NULL) receives dtnew(1..nlevelmax). */
int rb_coarse_step(rb_context *ctx, double *t_io, double *dtnew_out);
/* Coarse steps until t >= t_end or max_steps steps have run, the loop of
 * adaptive_loop (amr/adaptive_loop.f90:118-205) over amr_step (same results
 * as repeated rb_coarse_step calls). The scheduler state (dtnew, dtold, t,
 * nstep, amr/amr_step.f90:320-331,571-576) stays on the device, so the steps
 * run without host round trips; with use_graph the steps run from a cached
 * CUDA graph of 8 coarse steps whose launches become no-ops past the stop
 * rule. steps_done (may be NULL) receives the coarse steps taken. */
int rb_run(rb_context *ctx, int max_steps, double t_end, int use_graph, double *t_io, int *steps_done);
/* Leaf-cell updates done by this context so far (one per leaf cell per step of its level). */
int rb_cell_updates(rb_context *ctx, int64_t *out);

/* Choose the tile shape of level ilevel's godunov kernel: shape >= 0 forces
 * one (see rb_tile_shape_info), shape < 0 times every shape on the current
 * state and keeps the fastest (the state is left unchanged). */
int rb_set_tile_shape(rb_context *ctx, int ilevel, int shape);
int rb_get_tile_shape(rb_context *ctx, int ilevel, int *shape);
int rb_tile_shape_info(int shape, int *tx, int *ty, int *tz, int *nthreads);
/* Launch order of every level's tiles (one CTA each): 0 (default) a 3D Morton
 * curve over the tile positions; 1 z slabs one tile thick, a 2D Morton curve
 * inside each, so that the CTAs resident at once cover neighbouring slabs and
 * the stencil halos a tile reads were read by a tile of the slab before it.
 * The results do not depend on the order. */
int rb_set_tile_order(rb_context *ctx, int order);

/* unsplit with the reference's argument list and Fortran layouts
 * (umuscl.f90:22-38): uin(nvector,-1:4,-1:4,-1:4,5),
 * gravin(nvector,-1:4,-1:4,-1:4,3) (may be NULL = zero gravity), pin unused,
 * flux(nvector,1:3,1:3,1:3,5,3), tmp(nvector,1:3,1:3,1:3,2,3). Host pointers;
 * FP64 only. */
int rb_unsplit(const rb_hydro_params *hp, const double *uin, const double *gravin, const double *pin,
               double *flux, double *tmp, double dx, double dy, double dz, double dt, int ngrid,
               int nvector);

/* Device-resident uniform-grid stepper (configs with one complete level):
 * state kept as uold/unew in the device layout, one fused kernel per step
 * (gather, fluxes, update, next-step CFL partials) and a single-thread dt
 * finalisation; nsteps steps are captured as one CUDA graph when
 * use_graph != 0. dt of each step is the CFL dt of the state it starts from,
 * as newdt_fine/courant_fine give it. t_io advanced; dt_last_out may be NULL. */
int rb_uniform_run(rb_context *ctx, int nsteps, int use_graph, double *t_io, double *dt_last_out);

/* Kernel used by rb_uniform_run: 0 = z-streaming stencil over a dense
 * Cartesian mirror of the level (default), 1 = the godunov_fine oct tiles.
 * Both give bit-identical results in FP64 (in FP32-mixed they differ by
 * FP32 rounding only). slope_type 3 always runs on the oct tiles. */
int rb_set_uniform_method(rb_context *ctx, int method);
/* Kernel configuration of the last rb_uniform_run: method, shape (z-streaming
 * column shape 0: 8x8, 1: 16x8, 2: 16x16 cells, or oct-tile shape), z extent
 * of a work item and number of work items (CTAs) per step. */
int rb_get_uniform_info(rb_context *ctx, int *method, int *shape, int *hz, int *items);
/* Autotune the z-streaming step on the live state: every column shape and
 * register budget (0: 8x8, 1: 16x8, 2: 16x16, 3: 16x8 at 2 CTAs/SM, 4: 8x8 at
 * 4 CTAs/SM) and z extent 4..64 is timed; the fastest is kept. The state, the time and the next dt are unchanged. Outputs may be
 * NULL. */
int rb_autotune_uniform(rb_context *ctx, int *shape, int *hz, float *ms);
/* Set the z-streaming configuration by hand (shape as above; hz even and
 * dividing the grid's nz), e.g. to replay an autotuned choice. */
int rb_set_stream_shape(rb_context *ctx, int shape, int hz);

/* CFL reduction over plain device arrays that allocates nothing.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc/cudaFree mid-run (those calls wait for the whole device to go
 * idle), e.g. a host loop keeping several problems in flight on one stream or
 * a host with its own fixed device-memory pool. Its scratch is a fixed
 * 2 MiB device array inside the library, shared by all calls.
 * d_u: device array of conservative variables, variable v of cell i at
 * d_u[v*stride + i], i < ncell, all treated as leaf cells of cell size dx.
 * d_out: 4 device doubles receiving (dt, mass, total energy, internal energy)
 * with dt = min(dt_in, courant_factor*dx/smallc, min over cells of the cmpdt
 * time step) as courant_fine gives it. Runs on `stream` (a cudaStream_t, NULL
 * for the default stream) without synchronising.
 * Limit: ncell <= RB_NOALLOC_MAX_CELLS, else RB_ERR_CAPACITY. Calls that
 * overlap on the GPU race on the shared scratch. The first call on each device
 * resolves the scratch address and should come before any stream capture. */
#define RB_NOALLOC_MAX_CELLS 16777216LL
int rb_courant_cells_noalloc(const rb_hydro_params *hp, const double *d_u, int64_t ncell, int64_t stride,
                             double dx, double dt_in, double *d_out, void *stream);

/* Wait for all work queued on the context's stream. */
int rb_synchronize(rb_context *ctx);
/* The context's CUDA stream (cudaStream_t) for callers that order their own work. */
int rb_get_stream(rb_context *ctx, void **stream);
/* Mean device milliseconds per godunov tile-kernel launch of the last
 * rb_godunov_fine call or un-graphed rb_uniform_run (CUDA events around the
 * kernel alone). */
int rb_last_kernel_ms(rb_context *ctx, float *ms);
/* Device milliseconds of the whole last rb_uniform_run or rb_run (all steps). */
int rb_last_run_ms(rb_context *ctx, float *ms);

/* ---- serving engine: many independent problems on one GPU ----------------
 * No counterpart in the reference (one RAMSES run is one problem). Problems
 * are admitted first-come first-served while their device memory fits in the
 * budget, stay resident until t >= t_end or max_steps steps, and their result
 * is then copied into the caller's `result` buffer. The caller keeps every
 * array it passes (input, tree, result) valid until the request completes or
 * is cancelled. A problem's result is bitwise the same whatever other
 * problems share the GPU with it: no reduction or atomic spans problems.
 * Single-threaded: one host thread drives a server. */
typedef struct rb_server rb_server;
#define RB_REQ_QUEUED 0
#define RB_REQ_ACTIVE 1
#define RB_REQ_DONE 2
#define RB_REQ_FAILED 3
#define RB_REQ_CANCELLED 4
/* hbm_budget_bytes <= 0: 85% of the free device memory. steps_per_round:
 * batched steps enqueued per rb_server_progress call (1..1024). */
int rb_server_create(const rb_hydro_params *hp, int precision, int64_t hbm_budget_bytes, int steps_per_round,
                     rb_server **out);
int rb_server_destroy(rb_server *srv);
/* A uniform problem as a dense grid: u[v][z][y][x] conservative
 * (rho, rho*u, rho*v, rho*w, E), nx = ny = nz, nx a multiple of 16. Every
 * step is a time step of the complete level (the z-streaming kernel, batched
 * with every other active dense problem); result has the layout of u.
 * outflow_mask bit d (x=0, y=1, z=2): outflow (zero-gradient, bound_type 2)
 * boundaries along axis d; clear bits are periodic. */
int rb_server_submit_dense(rb_server *srv, int32_t nx, int32_t ny, int32_t nz, double boxlen, int32_t outflow_mask,
                           const double *u, double t_end, int64_t max_steps, double *result, int64_t *id);
/* An AMR problem in the rb_sync_tree / rb_upload_state form; stepped by
 * coarse steps as rb_run does; result is uold(ncell,5). */
int rb_server_submit_octree(rb_server *srv, const rb_mesh_params *mp, const int32_t *son, const int32_t *father,
                            const int32_t *nbor, const int32_t *numbl, const int32_t *active_igrid,
                            const double *uold, double t_end, int64_t max_steps, double *result, int64_t *id);
/* The same with physical boundaries (rb_set_boundary's lists, kept by the
 * caller until the request completes); the boundary octs are filled once at
 * admission and after every level step. */
int rb_server_submit_octree_bounded(rb_server *srv, const rb_mesh_params *mp, const int32_t *son,
                                    const int32_t *father, const int32_t *nbor, const int32_t *numbl,
                                    const int32_t *active_igrid, int32_t nboundary, const int32_t *boundary_type,
                                    const int32_t *numbb, const int32_t *boundary_igrid, const double *uold,
                                    double t_end, int64_t max_steps, double *result, int64_t *id);
/* Admit, enqueue one round of steps, retire finished problems. Up to max_ids
 * completed request ids are written to done_ids (the rest on later calls). */
int rb_server_progress(rb_server *srv, int64_t *done_ids, int max_ids, int *ndone);
/* State (RB_REQ_*), time reached, steps, leaf-cell updates and seconds from
 * submission to completion (or to now). Returns the request's error status. */
int rb_server_request_info(rb_server *srv, int64_t id, int *state, double *t, int64_t *steps,
                           int64_t *cell_updates, double *seconds_in_system);
/* Cancel a queued or active request (it completes as RB_REQ_CANCELLED). */
int rb_server_cancel(rb_server *srv, int64_t id);
int rb_server_stats(rb_server *srv, int *queued, int *active, int64_t *bytes_in_use, int64_t *budget,
                    int64_t *cell_updates, int64_t *batch_launches);

#ifdef __cplusplus
}
#endif
#endif
