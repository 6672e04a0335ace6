// rb_context.h -- internal to the library: the per-problem context of the
// host runtime, its per-level tables, and the helpers shared by the runtime
// and the serving engine (error reporting, device allocation).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/ramses_b200.h"
#include "godunov_tile.cuh"
#include "rb_error.h"
#include "rb_aux.cuh"
#include "stream_kernel.cuh"
#include "tile_launch.h"

namespace rbi {

// host-side Fortran MIN with the same tie rule as the device and the oracle
inline double rb_min_host(double a, double b) { return a < b ? a : (b < a ? b : a); }

template <typename T>
int dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) return RB_OK;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(RB_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
  }
  return RB_OK;
}
template <typename T>
void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}
// Grow-only device buffer from a memory pool, ordered on `stream`: at least
// n elements (a quarter more when it has to grow); a smaller request keeps
// the allocation. The pool keeps freed memory (its release threshold is
// unbounded), so growing a table during a tree re-sync does not go through
// cudaMalloc/cudaFree, which cost up to hundreds of ms there.
template <typename T>
int dreserve(cudaMemPool_t pool, cudaStream_t stream, T** p, size_t* cap, size_t n) {
  if (n <= *cap && (*p || n == 0)) return RB_OK;
  if (*p) cudaFreeAsync((void*)*p, stream);
  *p = nullptr;
  *cap = 0;
  const size_t m = n + n / 4;
  cudaError_t e = cudaMallocFromPoolAsync((void**)p, m * sizeof(T), pool, stream);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(RB_ERR_NOMEM, "device table allocation of %zu bytes failed: %s", m * sizeof(T), cudaGetErrorString(e));
  }
  *cap = m;
  return RB_OK;
}
template <typename T>
void drelease(cudaStream_t stream, T*& p, size_t& cap) {
  if (p) cudaFreeAsync((void*)p, stream);
  p = nullptr;
  cap = 0;
}

inline int grid_for(int64_t n, int nt, int cap = 148 * 32) {
  int64_t g = (n + nt - 1) / nt;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

struct Level {
  int noct = 0;
  std::vector<int32_t> h_active;  // igrid (1-based), host order
  int32_t* d_active = nullptr;    // igrid-1
  int shape = -1;
  bool shape_user = false;        // shape set by rb_set_tile_shape (else re-chosen at every table build)
  int ntile = 0;
  int32_t* d_tile_blk = nullptr;
  int32_t* d_tile_corr_off = nullptr; // [ntile+1] first correction face entry of each tile (null: none)
  int32_t* d_tile_corr = nullptr;     // [entries][2] (oct in tile | face << 8, slot)
  int ninterp = 0;
  int32_t* d_interp7 = nullptr;
  double* d_interp_buf = nullptr;
  int has_refined = 0;
  int nslot = 0;
  double* d_corr_flux = nullptr;
  double* d_corr_tmp = nullptr;   // pressure_fix: [nslot][6][4][2] (divu, enew) fluxes of the correction faces
  int ntgt = 0;
  int32_t* d_tgt = nullptr;
  int32_t* d_tgt_off = nullptr;
  int32_t* d_contrib = nullptr;
  int32_t* d_nbor6 = nullptr;     // [noct][6] device cell of nbor(igrid,j) (hydro_flag)
  int64_t* d_nres6 = nullptr;     // [noct][6] nbor(igrid,j) resolved to the neighbouring oct (pressure_fix pdV)
  bool nbor6_ok = false, nres6_ok = false;  // d_nbor6 / d_nres6 hold this tree's values
  // capacities (elements) of the device buffers: they only grow, so a
  // re-sync reuses the allocations (no cudaFree/cudaMalloc per remesh)
  size_t cap_active = 0, cap_tile_blk = 0, cap_tile_corr = 0, cap_tile_corr_off = 0, cap_interp7 = 0,
         cap_interp_buf = 0, cap_corr_flux = 0, cap_corr_tmp = 0, cap_tgt = 0, cap_tgt_off = 0, cap_contrib = 0,
         cap_nbor6 = 0, cap_nres6 = 0, cap_bpair = 0;
  int64_t leaf_cells = 0;
  double dx = 0.0;
  bool complete = false;
  bool tables_built = false;
  // physical boundaries: per region (boundary order), the (boundary oct,
  // reference oct) pairs of this level, igrid-1 each, at [boff[r], boff[r+1])
  std::vector<int64_t> h_boff;
  int32_t* d_bpair = nullptr;
  // the level's boundary octs (all regions, in region order) of the last sync
  std::vector<int32_t> h_bnd;
  // runs of consecutive igrids of h_active as (first igrid, count) pairs,
  // for the level's uold transfers; valid for tree sync number runs_sync
  std::vector<int32_t> runs;
  int64_t runs_sync = -1;
};

// sorted (key, igrid) lookup of one level's octs
struct OctIndex {
  std::vector<std::pair<int64_t, int32_t>> v;
  int64_t nx = 1, ny = 1, nz = 1;  // octs per dimension at this level
  int64_t key(int64_t x, int64_t y, int64_t z) const {
    x = ((x % nx) + nx) % nx;
    y = ((y % ny) + ny) % ny;
    z = ((z % nz) + nz) % nz;
    return x + nx * (y + ny * z);
  }
  int32_t find(int64_t x, int64_t y, int64_t z) const {
    const int64_t k = key(x, y, z);
    auto it = std::lower_bound(v.begin(), v.end(), std::make_pair(k, (int32_t)INT32_MIN));
    if (it != v.end() && it->first == k) return it->second;
    return 0;
  }
};

}  // namespace rbi

struct rb_context {
  rb_hydro_params hp;
  rb_mesh_params mp;
  int precision = RB_PREC_FP64;
  int device = 0;
  int64_t ncell = 0;
  cudaStream_t stream = nullptr;
  cudaMemPool_t table_pool = nullptr;  // the level tables' device buffers (grow-only, kept across re-syncs)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  double* d_uold = nullptr;
  double* d_unew = nullptr;
  double* d_divu = nullptr;         // pressure_fix: velocity divergence x (-dt) per cell
  double* d_enew = nullptr;         // pressure_fix: internal energy per cell
  double dt_godunov[RB_MAXLEVEL + 2] = {0};  // dt of the last rb_godunov_fine per level (set_uold's dtnew)
  int32_t* d_son = nullptr;
  double* d_stage = nullptr;        // Fortran-layout staging [5*ncell]
  double* d_partial = nullptr;      // CFL partials
  int64_t partial_cap = 0;
  double* d_red = nullptr;          // [8] reduction output
  double* d_clock = nullptr;        // [8] device clock of the uniform stepper
  double* h_red = nullptr;          // pinned [8]
  double* d_sched = nullptr;        // [RB_S_SIZE] device-resident amr_step clock
  double* h_sched = nullptr;        // pinned [RB_S_SIZE]
  uint8_t* d_flag = nullptr;        // hydro_flag output, one byte per cell of a level
  int64_t flag_cap = 0;
  const double* gate = nullptr;     // level kernels return early when *gate != 0
  cudaGraphExec_t amr_graph = nullptr;  // cached graph of amr_chunk coarse steps
  int amr_chunk = 0;
  bool have_tree = false;
  bool have_state = false;
  bool clock_valid = false;
  // physical boundaries (make_boundary_hydro): region types and the
  // host's boundary(ibound,ilevel) lists, kept for tree re-syncs
  std::vector<int32_t> btype;
  std::vector<int64_t> boff;        // [nlevelmax*nb+1] as rb_set_boundary's numbb
  std::vector<int32_t> bgrid;
  std::vector<int8_t> is_bnd;       // [ngridmax] 1 for a boundary oct
  double* d_bbuf = nullptr;         // [largest region][8][5] staging of one fill
  int64_t bbuf_cap = 0;
  // host copies of the tree (Fortran layout)
  std::vector<int32_t> son, father, nbor;
  std::vector<int64_t> coords;      // [ngridmax*3] oct coordinates at its level
  std::vector<int8_t> level_of;     // [ngridmax] level of each oct (0 = unused)
  rbi::Level lv[RB_MAXLEVEL + 2];
  std::vector<rbi::OctIndex> idx;        // per-level position -> igrid lookup
  int finest = 0;                   // finest level holding octs
  std::vector<int32_t> h_corr_slot; // [ngridmax] correction slot of each oct or -1 (table building)
  std::vector<cudaEvent_t> evpool;  // per-step kernel timing events
  float kernel_ms_avg = 0.f;        // mean tile-kernel time of the last timed run
  cudaGraphExec_t graph = nullptr;  // cached uniform-run graph
  int graph_steps = 0;
  double* graph_cur = nullptr;
  // dense Cartesian mirror of the finest (complete) level for the z-streaming path
  int uniform_method = 0;           // 0: z-streaming over the dense mirror, 1: oct tiles
  double* d_dense[2] = {nullptr, nullptr};
  int dense_cur = 0;
  int64_t* d_cbase = nullptr;
  int32_t dnx = 0, dny = 0, dnz = 0;
  bool dense_valid = false;         // the dense mirror holds the newest state of `finest`
  bool oct_stale = false;           // the oct layout of `finest` lags the dense mirror
  int stream_shape = -1, stream_hz = 0, stream_items = 0;
  int tile_order = 0;               // launch order of a level's tiles: 0 3D Morton, 1 z slabs
  // residency protocol of the drop-in boundary: which copy of uold is newer
  // (0: host and device agree, 1: the device's, 2: the host's), the host's
  // tree generation and the one last synchronised, and the transfer counters
  int state_newer = 2;
  bool prev_tree_valid = false;     // level_of/father describe the last synchronised tree
  int64_t tree_gen = 0, synced_gen = -1;
  int64_t h2d_state_bytes = 0, d2h_state_bytes = 0, tree_syncs = 0, octs_prolonged = 0;
  // tree re-syncs: a level whose table inputs did not change keeps its
  // tables (tables_kept: the last tree's tables are still allocated, with
  // the boundary region types they were built for); wall time of the phases
  // of the last sync (ms: total, per-level index, level tables, boundary
  // pairs, new-oct prolongation) and its levels rebuilt / reused
  bool tables_kept = false;
  std::vector<int32_t> tables_btype;
  double sync_ms[5] = {0, 0, 0, 0, 0};
  int32_t levels_built = 0, levels_reused = 0;
  // scheduler state (amr_commons dtnew/dtold, t, nstep)
  double dtnew[RB_MAXLEVEL + 2] = {0}, dtold[RB_MAXLEVEL + 2] = {0};
  double t = 0.0;
  int64_t nstep = 0;
  int64_t cell_updates = 0;
  double mass_tot = 0, ekin_tot = 0, eint_tot = 0;
};

namespace rbi {
// parameter rules of rb_create (rb_runtime.cu)
int check_params(const rb_hydro_params* hp, const rb_mesh_params* mp);
// device-scheduled coarse steps without waiting (rb_runtime.cu)
int run_async_begin(rb_context* c, double t_end, int64_t max_coarse);
int run_async_chunk(rb_context* c, int chunk, bool use_graph);
int run_async_end(rb_context* c, int64_t* coarse_out);
// make_boundary_hydro of every level, queued on the context's stream (rb_runtime.cu)
int make_boundary_all(rb_context* c);
}  // namespace rbi
