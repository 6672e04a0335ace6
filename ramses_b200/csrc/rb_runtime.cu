// rb_runtime.cu -- host runtime and C ABI of the B200 hydro step.
//
// Owns one problem per rb_context: device mirrors of uold/unew/son in the
// device layout (variable-major, oct-major), per-level tables derived from the
// octree (active lists, godunov tiles, prolongation entries, fine-to-coarse
// correction lists), and the amr_step hydro scheduler
// (amr/amr_step.f90:320-445) that drives the level kernels on one stream.
// Compiled with --fmad=false (FP64 kernels bit-identical to the reference
// operation order).
#include <sched.h>

#include <atomic>
#include <chrono>
#include <mutex>
#include <thread>

#include "rb_context.h"

using namespace rbi;

namespace rbi {

// Host->device copy ordered on the context's stream. A plain cudaMemcpy from
// pageable memory may return before its DMA has landed and runs on the legacy
// default stream, which does not order with the context's non-blocking
// stream; kernels on the context's stream could then read stale device data.
int h2d(rb_context* c, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return RB_OK;
  RB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
  RB_CUDA(cudaStreamSynchronize(c->stream));  // the caller may free src next
  return RB_OK;
}

int check_params(const rb_hydro_params* hp, const rb_mesh_params* mp) {
  if (!hp || !mp) return fail(RB_ERR_INVALID, "null parameter struct");
  if (hp->riemann < RB_RIEMANN_LLF || hp->riemann > RB_RIEMANN_EXACT)
    return fail(RB_ERR_INVALID, "unknown Riemann solver code %d (llf=1, hll=2, hllc=3, acoustic=4, exact=5)",
                hp->riemann);
  if (hp->riemann == RB_RIEMANN_EXACT && hp->niter_riemann < 1)
    return fail(RB_ERR_INVALID, "niter_riemann=%d must be >= 1 for the exact Riemann solver", hp->niter_riemann);
  const int st = hp->slope_type;
  if (!(st == 0 || st == 1 || st == 2 || st == 3 || st == 7 || st == 8))
    return fail(RB_ERR_INVALID, "Unknown slope type %d", st);
  if (hp->scheme != RB_SCHEME_MUSCL && hp->scheme != RB_SCHEME_PLMDE)
    return fail(RB_ERR_INVALID, "scheme %d not supported (muscl=0, plmde=1)", hp->scheme);
  if (hp->pressure_fix != 0 && hp->pressure_fix != 1)
    return fail(RB_ERR_INVALID, "pressure_fix must be 0 or 1 (got %d)", hp->pressure_fix);
  if (!(hp->beta_fix >= 0.0) || !std::isfinite(hp->beta_fix))
    return fail(RB_ERR_INVALID, "beta_fix=%g must be finite and >= 0", hp->beta_fix);
  if (!(hp->difmag >= 0.0) || !std::isfinite(hp->difmag))
    return fail(RB_ERR_INVALID, "difmag=%g must be finite and >= 0", hp->difmag);
  if (hp->interpol_var < 0 || hp->interpol_var > 2 || hp->interpol_type < 0 || hp->interpol_type > 4)
    return fail(RB_ERR_INVALID, "bad interpol_var/interpol_type");
  if (hp->interpol_type == 4 && hp->interpol_var != 2)
    return fail(RB_ERR_INVALID, "interpol_type=4 is designed for interpol_var=2");
  if (!(hp->gamma > 1.0) || !(hp->smallr > 0.0) || !(hp->smallc > 0.0) || !(hp->courant_factor > 0.0))
    return fail(RB_ERR_INVALID, "gamma must exceed 1 and smallr, smallc, courant_factor be positive");
  if (mp->nx < 1 || mp->ny < 1 || mp->nz < 1 || mp->ncoarse != mp->nx * mp->ny * mp->nz)
    return fail(RB_ERR_INVALID, "bad coarse grid");
  if (mp->ngridmax < 1 || mp->nlevelmax < 1 || mp->nlevelmax > RB_MAXLEVEL || mp->levelmin < 1 ||
      mp->levelmin > mp->nlevelmax)
    return fail(RB_ERR_INVALID, "bad ngridmax/levelmin/nlevelmax");
  if (mp->nvector < 1) return fail(RB_ERR_INVALID, "nvector must be positive");
  // device cell indices are held in 32 bits in the level tables and kernels
  if ((int64_t)mp->ncoarse + 8 * (int64_t)mp->ngridmax >= (int64_t)INT32_MAX)
    return fail(RB_ERR_INVALID, "ncoarse + 8*ngridmax must stay below 2^31 cells");
  if (!(mp->boxlen > 0.0)) return fail(RB_ERR_INVALID, "boxlen must be positive");
  if (mp->nx_loc < 0 || mp->nx_loc > mp->nx)
    return fail(RB_ERR_INVALID, "nx_loc=%d must lie in 0..nx (0: nx)", mp->nx_loc);
  return RB_OK;
}

inline int64_t fcell(const rb_context* c, int ind /*1..8*/, int igrid /*1-based*/) {
  return (int64_t)c->mp.ncoarse + (int64_t)(ind - 1) * c->mp.ngridmax + igrid;
}
inline int64_t dev_of_fortran(const rb_context* c, int64_t icell) {
  if (icell <= c->mp.ncoarse) return icell - 1;
  const int64_t r = icell - 1 - c->mp.ncoarse;
  return c->mp.ncoarse + (r % c->mp.ngridmax) * 8 + r / c->mp.ngridmax;
}

inline uint64_t morton2(uint64_t x, uint64_t y) {
  auto spread = [](uint64_t a) {
    a &= 0x1fffff;
    a = (a | a << 16) & 0x0000ffff0000ffffULL;
    a = (a | a << 8) & 0x00ff00ff00ff00ffULL;
    a = (a | a << 4) & 0x0f0f0f0f0f0f0f0fULL;
    a = (a | a << 2) & 0x3333333333333333ULL;
    a = (a | a << 1) & 0x5555555555555555ULL;
    return a;
  };
  return spread(x) | spread(y) << 1;
}

inline uint64_t morton3(uint64_t x, uint64_t y, uint64_t z) {
  auto spread = [](uint64_t a) {
    a &= 0x1fffff;
    a = (a | a << 32) & 0x1f00000000ffffULL;
    a = (a | a << 16) & 0x1f0000ff0000ffULL;
    a = (a | a << 8) & 0x100f00f00f00f00fULL;
    a = (a | a << 4) & 0x10c30c30c30c30c3ULL;
    a = (a | a << 2) & 0x1249249249249249ULL;
    return a;
  };
  return spread(x) | spread(y) << 1 | spread(z) << 2;
}

// Invalidate a level's tables; with release the device buffers are freed
// too (else they are kept for the next build, which reuses them).
void free_level_tables(rb_context* c, Level& L, bool release = false) {
  if (release) {
    cudaStream_t st = c->stream;
    drelease(st, L.d_tile_blk, L.cap_tile_blk);
    drelease(st, L.d_tile_corr, L.cap_tile_corr);
    drelease(st, L.d_tile_corr_off, L.cap_tile_corr_off);
    drelease(st, L.d_interp7, L.cap_interp7);
    drelease(st, L.d_interp_buf, L.cap_interp_buf);
    drelease(st, L.d_corr_flux, L.cap_corr_flux);
    drelease(st, L.d_corr_tmp, L.cap_corr_tmp);
    drelease(st, L.d_tgt, L.cap_tgt);
    drelease(st, L.d_tgt_off, L.cap_tgt_off);
    drelease(st, L.d_contrib, L.cap_contrib);
    drelease(st, L.d_nbor6, L.cap_nbor6);
    drelease(st, L.d_nres6, L.cap_nres6);
  }
  L.nbor6_ok = L.nres6_ok = false;
  L.ntile = L.ninterp = L.nslot = L.ntgt = 0;
  L.tables_built = false;
}

void drop_graph(rb_context* c) {
  if (c->graph) cudaGraphExecDestroy(c->graph);
  c->graph = nullptr;
  c->graph_steps = 0;
  c->graph_cur = nullptr;
  if (c->amr_graph) cudaGraphExecDestroy(c->amr_graph);
  c->amr_graph = nullptr;
  c->amr_chunk = 0;
}

void free_dense(rb_context* c) {
  dfree(c->d_dense[0]);
  dfree(c->d_dense[1]);
  dfree(c->d_cbase);
  c->dense_valid = false;
  c->oct_stale = false;
  c->stream_shape = -1;
}

// Drop the synchronised tree. With keep_tables the per-level tables, active
// lists (host and device) and boundary lists stay allocated (tables_kept) for
// the next rb_sync_tree, which reuses the levels whose inputs did not change.
void free_tree(rb_context* c, bool keep_tables = false) {
  drop_graph(c);
  free_dense(c);
  const bool keep = keep_tables && (c->have_tree || c->tables_kept);
  for (int l = 0; l <= RB_MAXLEVEL + 1; l++) {
    Level& L = c->lv[l];
    L.h_boff.clear();
    if (keep) continue;
    drelease(c->stream, L.d_bpair, L.cap_bpair);
    drelease(c->stream, L.d_active, L.cap_active);
    free_level_tables(c, L, true);
    L.noct = 0;
    L.h_active.clear();
    L.h_bnd.clear();
  }
  c->tables_kept = keep;
  c->have_tree = false;
}

// Host threads for the table builds: the CPUs this process may run on
// (its affinity mask; a container's limit, not the machine's core count),
// at most 32.
int64_t host_threads() {
  static const int64_t n = [] {
    cpu_set_t set;
    int64_t k = 0;
    if (sched_getaffinity(0, sizeof set, &set) == 0) k = CPU_COUNT(&set);
    if (k < 1) k = std::max(1u, std::thread::hardware_concurrency());
    return std::min<int64_t>(k, 32);
  }();
  return n;
}

// Run f(begin, end) over [0, n) on up to host_threads() threads (one chunk
// each; small ranges run on the calling thread).
template <typename F>
void parallel_for(int64_t n, int64_t min_chunk, F&& f) {
  int64_t nt = host_threads();
  nt = std::min<int64_t>(nt, std::max<int64_t>(1, n / std::max<int64_t>(1, min_chunk)));
  if (nt <= 1) {
    f((int64_t)0, n);
    return;
  }
  std::vector<std::thread> th;
  th.reserve((size_t)nt);
  for (int64_t t = 0; t < nt; t++) th.emplace_back([&f, n, nt, t] { f(n * t / nt, n * (t + 1) / nt); });
  for (auto& x : th) x.join();
}

// std::sort on up to host_threads() threads: chunks sorted in
// parallel, then merged pairwise. The order is that of std::sort for a
// comparator with no ties (a strict total order), as every caller uses.
template <typename T, typename Cmp>
void parallel_sort(std::vector<T>& v, Cmp cmp) {
  const int64_t n = (int64_t)v.size();
  const int64_t nt = host_threads();
  if (n < (1 << 16) || nt < 2) {
    std::sort(v.begin(), v.end(), cmp);
    return;
  }
  int64_t p2 = 1;
  while (p2 * 2 <= nt) p2 *= 2;
  std::vector<int64_t> b((size_t)p2 + 1);
  for (int64_t i = 0; i <= p2; i++) b[i] = n * i / p2;
  parallel_for(p2, 1, [&](int64_t c0, int64_t c1) {
    for (int64_t i = c0; i < c1; i++) std::sort(v.begin() + b[i], v.begin() + b[i + 1], cmp);
  });
  for (int64_t w = 1; w < p2; w *= 2)
    parallel_for(p2 / (2 * w), 1, [&](int64_t m0, int64_t m1) {
      for (int64_t m = m0; m < m1; m++) {
        const int64_t i = m * 2 * w;
        std::inplace_merge(v.begin() + b[i], v.begin() + b[i + w], v.begin() + b[i + 2 * w], cmp);
      }
    });
}

// first error of a parallel region, reported through fail() on the calling
// thread afterwards (the last-error string is thread-local)
struct ParError {
  std::atomic<bool> set{false};
  std::mutex m;
  int code = RB_OK;
  std::string msg;
  void record(int code_, const char* fmt, ...) {
    if (set.load()) return;
    std::lock_guard<std::mutex> g(m);
    if (set.load()) return;
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    code = code_;
    msg = buf;
    set.store(true);
  }
  int report() const { return set.load() ? fail(code, "%s", msg.c_str()) : RB_OK; }
};

// With physical boundaries a tile must not hold both octs of the box and
// boundary octs: along a bounded axis the tile's octs must divide the
// 2^(l-1) octs of one coarse cell.
bool shape_fits(const rb_context* c, int l, int shape) {
  const rb::TileShape sh = rb::kTileShapes[shape];
  const int64_t h = (int64_t)1 << (l - 1);
  const int to[3] = {sh.tx / 2, sh.ty / 2, sh.tz / 2};
  for (int32_t bt : c->btype)
    if (h % to[(bt % 10 - 1) / 2] != 0) return false;
  return true;
}

int default_shape(const rb_context* c, int l, const Level& L) {
  int s = 0;                                            // single oct
  if (L.complete && L.noct >= 64 * 148) s = 4;          // 8x8x8 cells
  else if (L.noct >= 8 * 64) s = 1;                     // 4x4x4 cells
  return shape_fits(c, l, s) ? s : 0;
}

// Device cell of nbor(igrid,j), j = 1..6, for the level's octs in active
// order (hydro_flag and the pdV term of pressure_fix).
int ensure_nbor6(rb_context* c, Level& L) {
  if (L.nbor6_ok || !L.noct) return RB_OK;
  std::vector<int32_t> nb((size_t)L.noct * 6);
  for (int i = 0; i < L.noct; i++) {
    const int g = L.h_active[i];
    for (int j = 0; j < 6; j++)
      nb[(size_t)i * 6 + j] = (int32_t)dev_of_fortran(c, c->nbor[(size_t)j * c->mp.ngridmax + (g - 1)]);
  }
  RB_TRY(dreserve(c->table_pool, c->stream, &L.d_nbor6, &L.cap_nbor6, nb.size()));
  RB_TRY(h2d(c, L.d_nbor6, nb.data(), nb.size() * sizeof(int32_t)));
  L.nbor6_ok = true;
  return RB_OK;
}

// nbor(igrid,j) of the level's octs resolved for the pdV term: the device
// cell of child 0 of the neighbouring oct at this level where it exists,
// else -(device cell of the coarse neighbour) - 1.
int ensure_nres6(rb_context* c, Level& L) {
  if (L.nres6_ok || !L.noct) return RB_OK;
  std::vector<int64_t> nr((size_t)L.noct * 6);
  for (int i = 0; i < L.noct; i++) {
    const int g = L.h_active[i];
    for (int j = 0; j < 6; j++) {
      const int64_t fcell = c->nbor[(size_t)j * c->mp.ngridmax + (g - 1)];
      const int32_t gn = c->son[fcell - 1];
      nr[(size_t)i * 6 + j] = gn > 0 ? (int64_t)c->mp.ncoarse + 8 * (int64_t)(gn - 1) : -dev_of_fortran(c, fcell) - 1;
    }
  }
  RB_TRY(dreserve(c->table_pool, c->stream, &L.d_nres6, &L.cap_nres6, nr.size()));
  RB_TRY(h2d(c, L.d_nres6, nr.data(), nr.size() * sizeof(int64_t)));
  L.nres6_ok = true;
  return RB_OK;
}

// getnborfather (amr/nbors_utils.f90:404-525): the level-(l-1) cell f
// (Fortran index) and its 6 face neighbours (-x,+x,-y,+y,-z,+z) at level
// l-1, or the coarser cell nbor(...) where that neighbour oct does not exist.
// Needs c->idx[l-1] and c->idx[l] of the current tree.
void father_nbor_cells(const rb_context* c, int l, int64_t f, int64_t cells[7]) {
  cells[0] = f;
  if (l == 1) {
    const int64_t nx = c->mp.nx, ny = c->mp.ny, nz = c->mp.nz, nxny = nx * ny;
    const int64_t ib[3] = {nx - 1, ny - 1, nz - 1};
    const int64_t s1[3] = {1, nx, nxny};
    const int64_t s2[3] = {nx - 1, (ny - 1) * nx, (nz - 1) * nxny};
    int64_t ix[3];
    ix[2] = (f - 1) / nxny;
    ix[1] = (f - 1 - ix[2] * nxny) / nx;
    ix[0] = (f - 1 - ix[1] * nx - ix[2] * nxny);
    for (int d = 0; d < 3; d++) {
      cells[2 * d + 1] = ix[d] > 0 ? f - s1[d] : f + s2[d];
      cells[2 * d + 2] = ix[d] < ib[d] ? f + s1[d] : f - s2[d];
    }
    return;
  }
  const OctIndex& P = c->idx[l - 1];
  const int64_t cnx = c->idx[l].nx, cny = c->idx[l].ny, cnz = c->idx[l].nz;
  const int64_t r = f - 1 - c->mp.ncoarse;
  const int32_t pg = (int32_t)(r % c->mp.ngridmax) + 1;
  const int pos = (int)(r / c->mp.ngridmax);
  const int cc[3] = {pos & 1, (pos >> 1) & 1, (pos >> 2) & 1};
  const int64_t* pc = &c->coords[(size_t)(pg - 1) * 3];
  for (int j = 1; j <= 6; j++) {
    const int d = (j - 1) / 2, plus = (j - 1) & 1;
    int64_t q[3] = {2 * pc[0] + cc[0], 2 * pc[1] + cc[1], 2 * pc[2] + cc[2]};
    q[d] += plus ? 1 : -1;
    const int32_t g = P.find(q[0] >> 1, q[1] >> 1, q[2] >> 1);
    if (g > 0) {
      const int64_t cx = ((q[0] % cnx) + cnx) % cnx, cy = ((q[1] % cny) + cny) % cny, cz = ((q[2] % cnz) + cnz) % cnz;
      const int ind = 1 + (int)(cx & 1) + 2 * (int)(cy & 1) + 4 * (int)(cz & 1);
      cells[j] = fcell(c, ind, g);
    } else {
      cells[j] = c->nbor[(size_t)(j - 1) * c->mp.ngridmax + (pg - 1)];
    }
  }
}

// RB_SYNC_TRACE=1 in the environment: the host time of each part of a level
// table build goes to stderr (the tree re-sync's cost breakdown).
bool sync_trace() {
  static const bool on = [] {
    const char* v = std::getenv("RB_SYNC_TRACE");
    return v && v[0] && v[0] != '0';
  }();
  return on;
}
struct PhaseClock {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  std::string line;
  void mark(const char* what) {
    if (!sync_trace()) return;
    const auto t1 = std::chrono::steady_clock::now();
    char b[64];
    snprintf(b, sizeof b, " %s %.2f", what, std::chrono::duration<double, std::milli>(t1 - t0).count());
    line += b;
    t0 = t1;
  }
};

// Build the godunov tile / prolongation / correction tables of level l.
int build_level_tables(rb_context* c, int l, const std::vector<OctIndex>& idx) {
  Level& L = c->lv[l];
  PhaseClock pc;
  free_level_tables(c, L);
  pc.mark("free");
  if (L.noct == 0) return RB_OK;
  if (L.shape < 0 || !L.shape_user) L.shape = default_shape(c, l, L);
  if (!shape_fits(c, l, L.shape))
    return fail(RB_ERR_INVALID, "level %d: tile shape %d spans the box face and the boundary layer", l, L.shape);
  const rb::TileShape sh = rb::kTileShapes[L.shape];
  const int TOX = sh.tx / 2, TOY = sh.ty / 2, TOZ = sh.tz / 2;
  const int BX = TOX + 2, BY = TOY + 2, BZ = TOZ + 2, NBLK = BX * BY * BZ;
  const OctIndex& I = idx[l];
  // --- tiles: unique tile coordinates of the level's octs, Morton ordered
  std::vector<std::pair<uint64_t, std::array<int64_t, 3>>> tiles;
  {
    // the tile of every oct; runs of octs of one tile (siblings follow each
    // other in an active list) are cut to one entry per chunk before the sort
    const int nch = 64;
    std::vector<std::vector<std::pair<uint64_t, std::array<int64_t, 3>>>> part(nch);
    parallel_for(nch, 1, [&](int64_t c0, int64_t c1) {
      for (int64_t ch = c0; ch < c1; ch++)
        for (int64_t i = (int64_t)L.noct * ch / nch; i < (int64_t)L.noct * (ch + 1) / nch; i++) {
          const int64_t* x = &c->coords[(size_t)(L.h_active[i] - 1) * 3];
          const int64_t tx = x[0] / TOX, ty = x[1] / TOY, tz = x[2] / TOZ;
          // launch order of the tiles: a 3D Morton curve, or z slabs one tile
          // thick with a 2D Morton curve inside each (rb_set_tile_order)
          const uint64_t key = c->tile_order == 1 ? ((uint64_t)tz << 42 | morton2(tx, ty)) : morton3(tx, ty, tz);
          if (part[ch].empty() || part[ch].back().first != key) part[ch].push_back({key, {tx, ty, tz}});
        }
    });
    size_t tot = 0;
    for (auto& v : part) tot += v.size();
    tiles.reserve(tot);
    for (auto& v : part) tiles.insert(tiles.end(), v.begin(), v.end());
    // the order key is unique per tile position: octs of one tile tie on
    // the key and are equal entries, so a sort by key then a unique by key
    // gives the same list whatever the order of equal entries
    parallel_sort(tiles, [](const auto& a, const auto& b) { return a.first < b.first; });
    tiles.erase(std::unique(tiles.begin(), tiles.end(),
                            [](const auto& a, const auto& b) { return a.first == b.first; }),
                tiles.end());
  }
  L.ntile = (int)tiles.size();
  pc.mark("tiles");
  std::vector<int32_t> blk((size_t)L.ntile * NBLK, -1);
  const OctIndex* P = l >= 2 ? &idx[l - 1] : nullptr;
  // level l-1 cells per dimension
  const int64_t cnx = I.nx, cny = I.ny, cnz = I.nz;
  ParError perr;
  // level-(l-1) cell at coordinates (x,y,z) (a level-l oct position), 0 if absent
  auto father_cell_of_pos = [&](int64_t x, int64_t y, int64_t z) -> int64_t {
    x = ((x % cnx) + cnx) % cnx;
    y = ((y % cny) + cny) % cny;
    z = ((z % cnz) + cnz) % cnz;
    if (l == 1) return 1 + x + c->mp.nx * (y + (int64_t)c->mp.ny * z);
    const int32_t pg = P->find(x >> 1, y >> 1, z >> 1);
    if (pg <= 0) {
      perr.record(RB_ERR_TREE, "level %d: father cell (%lld,%lld,%lld) of a needed neighbour block does not exist "
                  "(refinement rule violated)", l, (long long)x, (long long)y, (long long)z);
      return 0;
    }
    const int ind = 1 + (int)(x & 1) + 2 * (int)(y & 1) + 4 * (int)(z & 1);
    return fcell(c, ind, pg);
  };
  // pass 1, tiles in parallel: the source of every block of each tile's
  // stencil box; an absent block that an oct of the tile needs is marked
  // with its father cell f as -1 - f (prolongation entries are numbered in
  // pass 2)
  parallel_for(L.ntile, 256, [&](int64_t t0, int64_t t1) {
    std::vector<char> inner((size_t)TOX * TOY * TOZ);
    for (int64_t t = t0; t < t1 && !perr.set.load(); t++) {
      const int64_t ox0 = tiles[t].second[0] * TOX, oy0 = tiles[t].second[1] * TOY, oz0 = tiles[t].second[2] * TOZ;
      int32_t* B = &blk[(size_t)t * NBLK];
      const bool x_inside = ox0 - 1 >= 0 && ox0 - 1 + BX <= I.nx;
      for (int bz = 0; bz < BZ; bz++)
        for (int by = 0; by < BY; by++) {
          int32_t* row = B + BX * (by + BY * bz);
          if (x_inside) {
            // one search per row of blocks: the row's positions are
            // consecutive keys, so its octs follow each other in I.v
            const int64_t k0 = I.key(ox0 - 1, oy0 - 1 + by, oz0 - 1 + bz);
            auto it = std::lower_bound(I.v.begin(), I.v.end(), std::make_pair(k0, (int32_t)INT32_MIN));
            for (int bx = 0; bx < BX; bx++) {
              while (it != I.v.end() && it->first < k0 + bx) ++it;
              row[bx] = (it != I.v.end() && it->first == k0 + bx) ? it->second - 1 : -1;
            }
          } else {
            for (int bx = 0; bx < BX; bx++) {
              const int32_t g = I.find(ox0 - 1 + bx, oy0 - 1 + by, oz0 - 1 + bz);
              row[bx] = g > 0 ? g - 1 : -1;
            }
          }
        }
      for (int z = 0; z < TOZ; z++)
        for (int y = 0; y < TOY; y++)
          for (int x = 0; x < TOX; x++) {
            const int32_t g = B[(x + 1) + BX * ((y + 1) + BY * (z + 1))];
            if (g >= 0 && c->is_bnd[g]) {
              perr.record(RB_ERR_TREE, "level %d: a tile holds a boundary oct", l);
              return;
            }
            inner[x + TOX * (y + TOY * z)] = g >= 0;
          }
      for (int bz = 0; bz < BZ; bz++)
        for (int by = 0; by < BY; by++)
          for (int bx = 0; bx < BX; bx++) {
            int32_t& code = B[bx + BX * (by + BY * bz)];
            if (code >= 0) continue;
            bool needed = false;
            for (int dz = -1; dz <= 1 && !needed; dz++)
              for (int dy = -1; dy <= 1 && !needed; dy++)
                for (int dx = -1; dx <= 1 && !needed; dx++) {
                  const int ix = bx - 1 + dx, iy = by - 1 + dy, iz = bz - 1 + dz;
                  if (ix < 0 || iy < 0 || iz < 0 || ix >= TOX || iy >= TOY || iz >= TOZ) continue;
                  needed = inner[ix + TOX * (iy + TOY * iz)];
                }
            if (!needed) continue;
            const int64_t f = father_cell_of_pos(ox0 - 1 + bx, oy0 - 1 + by, oz0 - 1 + bz);
            if (f <= 0) return;
            code = (int32_t)(-1 - f);
          }
    }
  });
  RB_TRY(perr.report());
  pc.mark("pass1");
  // pass 2: one prolongation entry per distinct father cell, numbered in the
  // order of first use (tile order, so that a tile's entries lie together in
  // the interpolation buffer), the blocks' codes -2 - entry
  std::vector<int32_t> fcells;   // entry -> father cell
  {
    const int64_t nb = (int64_t)blk.size();
    const int nch = 64;
    std::vector<std::vector<std::pair<int32_t, int64_t>>> part(nch);   // (father cell, first block)
    parallel_for(nch, 1, [&](int64_t c0, int64_t c1) {
      for (int64_t ch = c0; ch < c1; ch++)
        for (int64_t b = nb * ch / nch; b < nb * (ch + 1) / nch; b++)
          if (blk[b] <= -2) part[ch].push_back({-1 - blk[b], b});
    });
    std::vector<std::pair<int32_t, int64_t>> fb;
    size_t tot = 0;
    for (auto& v : part) tot += v.size();
    fb.reserve(tot);
    for (auto& v : part) fb.insert(fb.end(), v.begin(), v.end());
    parallel_sort(fb, [](const std::pair<int32_t, int64_t>& a, const std::pair<int32_t, int64_t>& b) { return a < b; });
    // first use of each father cell, then the cells in the order of first use
    std::vector<std::pair<int64_t, int32_t>> first;
    for (size_t i = 0; i < fb.size(); i++)
      if (i == 0 || fb[i].first != fb[i - 1].first) first.push_back({fb[i].second, fb[i].first});
    parallel_sort(first, [](const std::pair<int64_t, int32_t>& a, const std::pair<int64_t, int32_t>& b) { return a < b; });
    fcells.resize(first.size());
    std::vector<std::pair<int32_t, int32_t>> entry_of(first.size());   // (father cell, entry), by cell
    for (size_t e = 0; e < first.size(); e++) {
      fcells[e] = first[e].second;
      entry_of[e] = {first[e].second, (int32_t)e};
    }
    parallel_sort(entry_of, [](const std::pair<int32_t, int32_t>& a, const std::pair<int32_t, int32_t>& b) { return a < b; });
    parallel_for(nb, 1 << 16, [&](int64_t b0, int64_t b1) {
      for (int64_t b = b0; b < b1; b++) {
        const int32_t code = blk[b];
        if (code > -2) continue;
        const int32_t f = -1 - code;
        const auto it = std::lower_bound(entry_of.begin(), entry_of.end(), std::make_pair(f, (int32_t)INT32_MIN));
        blk[b] = -2 - it->second;
      }
    });
  }
  pc.mark("pass2");
  // pass 3, entries in parallel: the father cell and its getnborfather
  // neighbours of every entry
  std::vector<int32_t> interp7(fcells.size() * 7);
  parallel_for((int64_t)fcells.size(), 1024, [&](int64_t e0, int64_t e1) {
    for (int64_t e = e0; e < e1; e++) {
      int64_t cells[7];
      father_nbor_cells(c, l, fcells[e], cells);
      for (int j = 0; j < 7; j++) interp7[(size_t)e * 7 + j] = (int32_t)dev_of_fortran(c, cells[j]);
    }
  });
  pc.mark("pass3");
  L.ninterp = (int)fcells.size();
  RB_TRY(dreserve(c->table_pool, c->stream, &L.d_tile_blk, &L.cap_tile_blk, blk.size()));
  RB_TRY(h2d(c, L.d_tile_blk, blk.data(), blk.size() * 4));
  if (L.ninterp) {
    RB_TRY(dreserve(c->table_pool, c->stream, &L.d_interp7, &L.cap_interp7, interp7.size()));
    RB_TRY(h2d(c, L.d_interp7, interp7.data(), interp7.size() * 4));
    RB_TRY(dreserve(c->table_pool, c->stream, &L.d_interp_buf, &L.cap_interp_buf, (size_t)L.ninterp * 8 * 5));
  }
  pc.mark("upload");
  // --- fine-to-coarse corrections (godunov_fine.f90:798-908)
  struct Contrib { int64_t tgt; int64_t batch; int face; int slot; };
  // per oct (active order) the faces bordering an unrefined coarser cell;
  // slots are numbered in active order, contributions laid out in that
  // order too (prefix sums), so the tables do not depend on the threads
  std::vector<uint8_t> fmask((size_t)L.noct, 0);
  {
    ParError perr;
    parallel_for(L.noct, 1 << 14, [&](int64_t p0, int64_t p1) {
      for (int64_t p = p0; p < p1; p++) {
        const int32_t g = L.h_active[p];
        uint8_t m = 0;
        for (int j = 1; j <= 6; j++) {
          const int64_t nc = c->nbor[(size_t)(j - 1) * c->mp.ngridmax + (g - 1)];
          if (nc < 1 || nc > c->ncell) {
            perr.record(RB_ERR_TREE, "nbor(%d,%d)=%lld out of range", g, j, (long long)nc);
            return;
          }
          if (c->son[nc - 1] == 0) m |= (uint8_t)(1u << (j - 1));
        }
        fmask[p] = m;
      }
    });
    RB_TRY(perr.report());
  }
  std::vector<int32_t> slot_at((size_t)L.noct + 1, 0), con_at((size_t)L.noct + 1, 0);
  for (int p = 0; p < L.noct; p++) {
    slot_at[p + 1] = slot_at[p] + (fmask[p] != 0);
    con_at[p + 1] = con_at[p] + __builtin_popcount(fmask[p]);
  }
  const int nslot = slot_at[L.noct];
  std::vector<Contrib> cons((size_t)con_at[L.noct]);
  std::vector<uint8_t> slot_faces((size_t)nslot);  // faces of each slot that border an unrefined coarser cell
  parallel_for(L.noct, 1 << 14, [&](int64_t p0, int64_t p1) {
    for (int64_t p = p0; p < p1; p++) {
      const uint8_t m = fmask[p];
      if (!m) continue;
      const int32_t g = L.h_active[p];
      const int slot = slot_at[p];
      slot_faces[slot] = m;
      int k = con_at[p];
      for (int j = 1; j <= 6; j++)
        if (m >> (j - 1) & 1) {
          const int64_t nc = c->nbor[(size_t)(j - 1) * c->mp.ngridmax + (g - 1)];
          cons[k++] = {dev_of_fortran(c, nc), p / c->mp.nvector, j - 1, slot};
        }
    }
  });
  L.nslot = nslot;
  if (nslot) {
    // (target, face) is unique (a coarse cell has one contributing fine oct
    // per face direction); the slot, which follows the active order, breaks
    // any tie as the generation order would
    parallel_sort(cons, [](const Contrib& a, const Contrib& b) {
      if (a.tgt != b.tgt) return a.tgt < b.tgt;
      if (a.batch != b.batch) return a.batch < b.batch;
      if (a.face != b.face) return a.face < b.face;  // direction, then left (even) before right (odd)
      return a.slot < b.slot;
    });
    std::vector<int32_t> tgt, off, contrib(cons.size());
    for (size_t i = 0; i < cons.size(); i++) {
      if (i == 0 || cons[i].tgt != cons[i - 1].tgt) {
        tgt.push_back((int32_t)cons[i].tgt);
        off.push_back((int32_t)i);
      }
      contrib[i] = cons[i].slot * 6 + cons[i].face;
    }
    off.push_back((int32_t)cons.size());
    L.ntgt = (int)tgt.size();
    RB_TRY(dreserve(c->table_pool, c->stream, &L.d_tgt, &L.cap_tgt, tgt.size()));
    RB_TRY(dreserve(c->table_pool, c->stream, &L.d_tgt_off, &L.cap_tgt_off, off.size()));
    RB_TRY(dreserve(c->table_pool, c->stream, &L.d_contrib, &L.cap_contrib, contrib.size()));
    RB_TRY(dreserve(c->table_pool, c->stream, &L.d_corr_flux, &L.cap_corr_flux, (size_t)nslot * 120));
    if (c->hp.pressure_fix) RB_TRY(dreserve(c->table_pool, c->stream, &L.d_corr_tmp, &L.cap_corr_tmp, (size_t)nslot * 48));
    RB_TRY(h2d(c, L.d_tgt, tgt.data(), tgt.size() * 4));
    RB_TRY(h2d(c, L.d_tgt_off, off.data(), off.size() * 4));
    RB_TRY(h2d(c, L.d_contrib, contrib.data(), contrib.size() * 4));
  }
  // this level's entries of the per-oct correction slot table
  parallel_for(L.noct, 1 << 14, [&](int64_t p0, int64_t p1) {
    for (int64_t p = p0; p < p1; p++) c->h_corr_slot[L.h_active[p] - 1] = fmask[p] ? slot_at[p] : -1;
  });
  pc.mark("corr");
  // per tile, the faces whose fluxes the fine-to-coarse correction reads:
  // entries (oct position in the tile | face << 8, slot), tile t's in
  // [off[t], off[t+1]), so that the godunov kernel stores only those
  if (nslot) {
    const int NOCT = TOX * TOY * TOZ;
    std::vector<int32_t> off((size_t)L.ntile + 1, 0);
    auto tile_entries = [&](int t, int32_t* out) {  // entries of tile t (written when out != null)
      const int32_t* B = &blk[(size_t)t * NBLK];
      int k = 0;
      for (int o = 0; o < NOCT; o++) {
        const int ox = o % TOX, oy = (o / TOX) % TOY, oz = o / (TOX * TOY);
        const int32_t code = B[(ox + 1) + BX * ((oy + 1) + BY * (oz + 1))];
        if (code < 0 || c->h_corr_slot[code] < 0) continue;
        const int32_t slot = c->h_corr_slot[code];
        for (int f = 0; f < 6; f++)
          if (slot_faces[slot] >> f & 1) {
            if (out) { out[2 * k] = o | f << 8; out[2 * k + 1] = slot; }
            k++;
          }
      }
      return k;
    };
    parallel_for(L.ntile, 1024, [&](int64_t t0, int64_t t1) {
      for (int64_t t = t0; t < t1; t++) off[t + 1] = tile_entries((int)t, nullptr);
    });
    for (int t = 0; t < L.ntile; t++) off[t + 1] += off[t];
    std::vector<int32_t> ent((size_t)off[L.ntile] * 2);
    parallel_for(L.ntile, 1024, [&](int64_t t0, int64_t t1) {
      for (int64_t t = t0; t < t1; t++) tile_entries((int)t, ent.data() + 2 * (size_t)off[t]);
    });
    RB_TRY(dreserve(c->table_pool, c->stream, &L.d_tile_corr_off, &L.cap_tile_corr_off, off.size()));
    RB_TRY(h2d(c, L.d_tile_corr_off, off.data(), off.size() * 4));
    RB_TRY(dreserve(c->table_pool, c->stream, &L.d_tile_corr, &L.cap_tile_corr, ent.size()));
    RB_TRY(h2d(c, L.d_tile_corr, ent.data(), ent.size() * 4));
  }
  if (c->hp.pressure_fix) RB_TRY(ensure_nres6(c, L));
  pc.mark("tilecorr");
  if (sync_trace())
    fprintf(stderr, "[rb sync] level %d: %d octs, %d tiles, %d entries, %d slots; ms:%s\n", l, L.noct, L.ntile,
            L.ninterp, L.nslot, pc.line.c_str());
  L.tables_built = true;
  return RB_OK;
}

// make_boundary_hydro's pairs (hydro/hydro_boundary.f90:118-137): for each
// boundary oct of each region, the reference oct son(nbor(igrid,inbor)) across
// the region's face towards the box.
int build_boundary_pairs(rb_context* c) {
  const int nb = (int)c->btype.size();
  const int ngm = c->mp.ngridmax;
  int64_t cap = 0;
  for (int l = 1; l <= c->mp.nlevelmax; l++) {
    Level& L = c->lv[l];
    L.h_boff.assign((size_t)nb + 1, 0);
    if (nb == 0) continue;
    std::vector<int32_t> pairs;
    for (int ib = 0; ib < nb; ib++) {
      const int dir = c->btype[ib] % 10;
      const int inbor = (dir & 1) ? dir + 1 : dir - 1;  // the side towards the box
      const int64_t k = (int64_t)(l - 1) * nb + ib;
      for (int64_t i = c->boff[k]; i < c->boff[k + 1]; i++) {
        const int32_t g = c->bgrid[i];
        const int64_t nc = c->nbor[(size_t)(inbor - 1) * ngm + (g - 1)];
        if (nc < 1 || nc > c->ncell) return fail(RB_ERR_TREE, "boundary grid %d: nbor(%d) out of range", g, inbor);
        const int32_t ref = c->son[nc - 1];
        if (ref < 1 || ref > ngm || c->level_of[ref - 1] != l)
          return fail(RB_ERR_TREE, "boundary grid %d (level %d) has no reference grid towards the box", g, l);
        pairs.push_back(g - 1);
        pairs.push_back(ref - 1);
      }
      L.h_boff[ib + 1] = (int64_t)pairs.size() / 2;
      cap = std::max(cap, L.h_boff[ib + 1] - L.h_boff[ib]);
    }
    if (!pairs.empty()) {
      RB_TRY(dreserve(c->table_pool, c->stream, &L.d_bpair, &L.cap_bpair, pairs.size()));
      RB_TRY(h2d(c, L.d_bpair, pairs.data(), pairs.size() * 4));
    }
  }
  if (cap > c->bbuf_cap) {
    dfree(c->d_bbuf);
    RB_TRY(dalloc(&c->d_bbuf, (size_t)cap * 40));
    c->bbuf_cap = cap;
  }
  return RB_OK;
}

int sync_oct(rb_context* c);

// After a re-sync: the octs that are new since the previous tree (a level
// they did not have, or another father cell; born[l], igrids) get the state
// make_grid_fine gives them, prolonged on the device in level order, so that
// a remeshed tree needs no state upload.
int prolong_new_octs(rb_context* c, const std::vector<std::vector<int32_t>>& born) {
  for (int l = 2; l <= c->mp.nlevelmax; l++) {
    if (born[l].empty()) continue;
    std::vector<int32_t> octs, cells7;
    octs.reserve(born[l].size());
    cells7.reserve(born[l].size() * 7);
    for (int32_t g : born[l]) {
      int64_t cells[7];
      father_nbor_cells(c, l, c->father[g - 1], cells);
      for (int j = 0; j < 7; j++) {
        if (cells[j] < 1 || cells[j] > c->ncell) return fail(RB_ERR_TREE, "grid %d: prolongation cell out of range", g);
        cells7.push_back((int32_t)dev_of_fortran(c, cells[j]));
      }
      octs.push_back(g - 1);
    }
    // octs and cells in the staging buffer (8 ints per new oct, at most
    // ngridmax octs: within its 40 bytes per cell)
    int32_t* d_octs = reinterpret_cast<int32_t*>(c->d_stage);
    int32_t* d_cells = d_octs + octs.size();
    RB_TRY(h2d(c, d_octs, octs.data(), octs.size() * 4));
    RB_TRY(h2d(c, d_cells, cells7.data(), cells7.size() * 4));
    rb::prolong_new_octs_kernel<<<(int)((octs.size() + 127) / 128), 128, 0, c->stream>>>(
        c->d_uold, d_cells, d_octs, (int32_t)octs.size(), c->ncell, c->mp.ncoarse, c->hp);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(RB_ERR_CUDA, "prolongation of new octs failed: %s", cudaGetErrorString(e));
    RB_CUDA(cudaStreamSynchronize(c->stream));
    c->octs_prolonged += (int64_t)octs.size();
  }
  return RB_OK;
}

// A re-sync is incremental when the previous tree's host mirrors and level
// tables are still held (same boundary region types): the host mirrors are
// updated over the octs of the old and new trees only (not over ngridmax),
// the device son mirror receives the entries that changed, and a level keeps
// its tables (tiles, prolongation entries, corrections, nbor6/nres6), its
// position index and its device active list when their inputs are unchanged.
// Level l's tables are a function of: its active list (whose order fixes the
// nvector batches of the corrections) and boundary octs, the positions and
// nbor rows of the octs of levels l and l-1, and son of the level-(l-1) cells
// (of the coarse cells for l = 1); all compared exactly, not sampled.
int sync_tree_impl(rb_context* c, const int32_t* son, const int32_t* father, const int32_t* nbor,
                   const int32_t* numbl, const int32_t* active) {
  if (!son || !father || !nbor || !numbl || !active) return fail(RB_ERR_INVALID, "null tree array");
  using clk = std::chrono::steady_clock;
  auto ms_since = [](clk::time_point t0) { return std::chrono::duration<double, std::milli>(clk::now() - t0).count(); };
  const clk::time_point t_start = clk::now();
  // a state held in the dense mirror goes back to the oct layout first
  if (c->have_tree) RB_TRY(sync_oct(c));
  const int NL = c->mp.nlevelmax;
  const int64_t ncell = c->ncell;
  const int ngm = c->mp.ngridmax;
  // the previous tree (still in level_of/father after an rb_set_boundary
  // dropped it) decides which octs are new
  const bool prolong = c->prev_tree_valid && c->have_state && c->state_newer != 2;
  const bool incremental = c->prev_tree_valid && (c->have_tree || c->tables_kept) && c->tables_btype == c->btype &&
                           c->son.size() == (size_t)ncell && c->level_of.size() == (size_t)ngm;
  std::vector<std::vector<int32_t>> old_active(RB_MAXLEVEL + 2), old_bnd(RB_MAXLEVEL + 2);
  if (incremental)
    for (int l = 1; l <= NL; l++) {
      old_active[l].swap(c->lv[l].h_active);
      old_bnd[l].swap(c->lv[l].h_bnd);
    }
  c->prev_tree_valid = false;
  free_tree(c, incremental);
  // the new lists
  int64_t off = 0;
  c->finest = 0;
  const int nb = (int)c->btype.size();
  for (int l = 1; l <= NL; l++) {
    Level& L = c->lv[l];
    const int n = numbl[l - 1];
    if (n < 0 || n > ngm || off + n > (int64_t)ngm) return fail(RB_ERR_INVALID, "numbl(%d)=%d out of range", l, n);
    L.h_active.assign(active + off, active + off + n);
    off += n;
    L.noct = n;
    if (n) c->finest = l;
    L.dx = std::pow(0.5, l) * (c->mp.boxlen / (double)(c->mp.nx_loc > 0 ? c->mp.nx_loc : c->mp.nx));
    L.h_bnd.clear();
    for (int ib = 0; ib < nb; ib++) {
      const int64_t k = (int64_t)(l - 1) * nb + ib;
      L.h_bnd.insert(L.h_bnd.end(), c->bgrid.begin() + c->boff[k], c->bgrid.begin() + c->boff[k + 1]);
    }
    for (int32_t g : L.h_active)
      if (g < 1 || g > ngm) return fail(RB_ERR_INVALID, "active grid %d out of range", g);
    for (int32_t g : L.h_bnd)
      if (g < 1 || g > ngm) return fail(RB_ERR_INVALID, "boundary grid %d out of range", g);
  }
  // octs new since the previous tree, judged against it before any mirror
  // is overwritten
  std::vector<std::vector<int32_t>> born(RB_MAXLEVEL + 2);
  if (prolong)
    for (int l = 2; l <= NL; l++)
      for (int32_t g : c->lv[l].h_active)
        if (c->level_of[g - 1] != l || c->father[g - 1] != father[g - 1]) born[l].push_back(g);
  // per level: its octs changed (lists, positions, nbor rows) / son of its
  // cells changed; son of the coarse cells changed
  std::vector<char> oct_dirty(RB_MAXLEVEL + 2, incremental ? 0 : 1), cell_dirty(RB_MAXLEVEL + 2, incremental ? 0 : 1);
  bool coarse_dirty = !incremental;
  std::vector<int64_t> son_idx;   // device cells whose son changed, and the values
  std::vector<int32_t> son_val;
  if (incremental) {
    for (int l = 1; l <= NL; l++) {
      if (c->lv[l].h_active != old_active[l] || c->lv[l].h_bnd != old_bnd[l]) oct_dirty[l] = 1;
      for (int32_t g : old_active[l]) { c->level_of[g - 1] = 0; c->is_bnd[g - 1] = 0; }
      for (int32_t g : old_bnd[l]) { c->level_of[g - 1] = 0; c->is_bnd[g - 1] = 0; }
    }
    for (int64_t i = 0; i < c->mp.ncoarse; i++)
      if (c->son[i] != son[i]) {
        coarse_dirty = true;
        son_idx.push_back(i);
        son_val.push_back(son[i]);
        c->son[i] = son[i];
      }
  } else {
    c->son.assign(son, son + ncell);
    c->father.assign(father, father + ngm);
    c->nbor.assign(nbor, nbor + (size_t)6 * ngm);
    c->coords.assign((size_t)ngm * 3, 0);
    c->level_of.assign((size_t)ngm, 0);
    c->is_bnd.assign((size_t)ngm, 0);
    c->h_corr_slot.assign((size_t)ngm, -1);
  }
  // positions (from the father chain, level by level), level and boundary
  // marks; in the incremental case also the nbor rows, father and the son
  // entries of the octs' cells, compared with the previous tree's. Levels in
  // order (a level reads its parents' positions), the octs of a level on all
  // host threads (each oct writes only its own entries).
  {
    const int nch = 64;
    std::vector<std::vector<int64_t>> part_idx(nch);
    std::vector<std::vector<int32_t>> part_val(nch);
    for (int l = 1; l <= NL; l++) {
      Level& L = c->lv[l];
      const size_t n = L.h_active.size();
      const int64_t nall = (int64_t)(n + L.h_bnd.size());
      ParError perr;
      std::atomic<bool> odirty{false}, cdirty{false};
      parallel_for(nch, 1, [&](int64_t c0, int64_t c1) {
        for (int64_t ch = c0; ch < c1; ch++) {
          bool od = false, cd = false;
          for (int64_t o = nall * ch / nch; o < nall * (ch + 1) / nch; o++) {
            const int32_t g = (size_t)o < n ? L.h_active[o] : L.h_bnd[o - n];
            const size_t gi = (size_t)(g - 1);
            if (c->level_of[gi] != 0) { perr.record(RB_ERR_TREE, "grid %d listed twice", g); return; }
            const int64_t fc = father[gi];
            int64_t x[3];
            if (l == 1) {
              if (fc < 1 || fc > c->mp.ncoarse) {
                perr.record(RB_ERR_TREE, "level-1 grid %d father %lld is not coarse", g, (long long)fc);
                return;
              }
              x[0] = (fc - 1) % c->mp.nx;
              x[1] = ((fc - 1) / c->mp.nx) % c->mp.ny;
              x[2] = (fc - 1) / ((int64_t)c->mp.nx * c->mp.ny);
            } else {
              const int64_t r = fc - 1 - c->mp.ncoarse;
              if (r < 0 || r >= (int64_t)8 * ngm) {
                perr.record(RB_ERR_TREE, "grid %d father %lld out of range", g, (long long)fc);
                return;
              }
              const int32_t pg = (int32_t)(r % ngm) + 1;
              const int pos = (int)(r / ngm);
              if (c->level_of[pg - 1] != l - 1) {
                perr.record(RB_ERR_TREE, "grid %d: father grid %d is not at level %d", g, pg, l - 1);
                return;
              }
              const int64_t* px = &c->coords[(size_t)(pg - 1) * 3];
              x[0] = 2 * px[0] + (pos & 1);
              x[1] = 2 * px[1] + ((pos >> 1) & 1);
              x[2] = 2 * px[2] + ((pos >> 2) & 1);
            }
            int64_t* xc = &c->coords[gi * 3];
            if (incremental) {
              if (xc[0] != x[0] || xc[1] != x[1] || xc[2] != x[2]) od = true;
              for (int j = 0; j < 6; j++) {
                const size_t k = (size_t)j * ngm + gi;
                if (c->nbor[k] != nbor[k]) { od = true; c->nbor[k] = nbor[k]; }
              }
              c->father[gi] = father[gi];
              for (int ind = 1; ind <= 8; ind++) {
                const int64_t cf = fcell(c, ind, g) - 1;
                if (c->son[cf] != son[cf]) {
                  cd = true;
                  part_idx[ch].push_back(dev_of_fortran(c, cf + 1));
                  part_val[ch].push_back(son[cf]);
                  c->son[cf] = son[cf];
                }
              }
            }
            xc[0] = x[0]; xc[1] = x[1]; xc[2] = x[2];
            c->level_of[gi] = (int8_t)l;
            if ((size_t)o >= n) c->is_bnd[gi] = 1;
          }
          if (od) odirty.store(true);
          if (cd) cdirty.store(true);
        }
      });
      RB_TRY(perr.report());
      if (odirty.load()) oct_dirty[l] = 1;
      if (cdirty.load()) cell_dirty[l] = 1;
    }
    for (int ch = 0; ch < nch; ch++) {
      son_idx.insert(son_idx.end(), part_idx[ch].begin(), part_idx[ch].end());
      son_val.insert(son_val.end(), part_val[ch].begin(), part_val[ch].end());
    }
  }
  // the position indexes of the changed levels (sorted on all host threads)
  c->idx.resize(RB_MAXLEVEL + 2);
  for (int l = 1; l <= NL; l++) {
    if (!oct_dirty[l]) continue;
    const Level& L = c->lv[l];
    OctIndex& I = c->idx[l];
    I.nx = (int64_t)c->mp.nx << (l - 1);
    I.ny = (int64_t)c->mp.ny << (l - 1);
    I.nz = (int64_t)c->mp.nz << (l - 1);
    const size_t n = L.h_active.size(), nall = n + L.h_bnd.size();
    I.v.resize(nall);
    parallel_for((int64_t)nall, 1 << 14, [&](int64_t o0, int64_t o1) {
      for (int64_t o = o0; o < o1; o++) {
        const int32_t g = (size_t)o < n ? L.h_active[o] : L.h_bnd[o - n];
        const int64_t* x = &c->coords[(size_t)(g - 1) * 3];
        I.v[o] = {I.key(x[0], x[1], x[2]), g};
      }
    });
    parallel_sort(I.v, [](const std::pair<int64_t, int32_t>& a, const std::pair<int64_t, int32_t>& b) { return a < b; });
    for (size_t i = 1; i < I.v.size(); i++)
      if (I.v[i].first == I.v[i - 1].first) return fail(RB_ERR_TREE, "level %d: two octs at one position", l);
  }
  // per level: completeness, leaf cells, device active list (re-uploaded
  // only when the list changed)
  for (int l = 1; l <= NL; l++) {
    Level& L = c->lv[l];
    const int n = L.noct;
    L.complete = (int64_t)n == c->idx[l].nx * c->idx[l].ny * c->idx[l].nz;
    std::atomic<int64_t> leaf{0};
    std::atomic<int> refined{0};
    parallel_for(n, 1 << 15, [&](int64_t i0, int64_t i1) {
      int64_t lf = 0;
      int rf = 0;
      for (int64_t i = i0; i < i1; i++)
        for (int ind = 1; ind <= 8; ind++) {
          const int32_t sv = son[fcell(c, ind, L.h_active[i]) - 1];
          lf += (sv == 0);
          rf |= (sv > 0);
        }
      leaf += lf;
      if (rf) refined.store(1);
    });
    L.leaf_cells = leaf.load();
    L.has_refined = refined.load();
    const bool same_list = incremental && L.h_active == old_active[l] && (L.d_active || n == 0);
    if (!same_list && n) {
      std::vector<int32_t> a0(n);
      for (int i = 0; i < n; i++) a0[i] = L.h_active[i] - 1;
      RB_TRY(dreserve(c->table_pool, c->stream, &L.d_active, &L.cap_active, (size_t)n));
      RB_TRY(h2d(c, L.d_active, a0.data(), (size_t)n * 4));
    }
  }
  // son mirror (device layout): the whole array, or the entries that changed
  if (!incremental) {
    RB_TRY(h2d(c, c->d_stage, son, ncell * 4));
    rb::permute_son_kernel<<<grid_for(ncell, 256), 256, 0, c->stream>>>((const int32_t*)c->d_stage, c->d_son, ncell,
                                                                        c->mp.ncoarse, ngm);
    RB_CUDA(cudaGetLastError());
    RB_CUDA(cudaStreamSynchronize(c->stream));
  } else if (!son_idx.empty()) {
    const int64_t m = (int64_t)son_idx.size();
    // staging: indexes then values in the (5 * ncell doubles) stage buffer
    if ((size_t)m * 12 > (size_t)ncell * 40) return fail(RB_ERR_TREE, "son diff larger than the staging buffer");
    int64_t* d_idx = reinterpret_cast<int64_t*>(c->d_stage);
    int32_t* d_val = reinterpret_cast<int32_t*>(d_idx + m);
    RB_TRY(h2d(c, d_idx, son_idx.data(), (size_t)m * 8));
    RB_TRY(h2d(c, d_val, son_val.data(), (size_t)m * 4));
    rb::scatter_son_kernel<<<grid_for(m, 256), 256, 0, c->stream>>>(c->d_son, d_idx, d_val, m);
    RB_CUDA(cudaGetLastError());
    RB_CUDA(cudaStreamSynchronize(c->stream));
  }
  c->sync_ms[1] = ms_since(t_start);
  const clk::time_point t_tables = clk::now();
  c->levels_built = c->levels_reused = 0;
  for (int l = 1; l <= NL; l++) {
    Level& L = c->lv[l];
    const bool keep = incremental && L.tables_built && L.noct > 0 && !oct_dirty[l] &&
                      (l == 1 ? !coarse_dirty : (!oct_dirty[l - 1] && !cell_dirty[l - 1]));
    if (keep) {
      c->levels_reused++;
      continue;
    }
    RB_TRY(build_level_tables(c, l, c->idx));
    if (L.noct) c->levels_built++;
  }
  c->sync_ms[2] = ms_since(t_tables);
  const clk::time_point t_bnd = clk::now();
  RB_TRY(build_boundary_pairs(c));
  c->sync_ms[3] = ms_since(t_bnd);
  c->have_tree = true;
  c->tables_kept = false;
  c->tables_btype = c->btype;
  c->prev_tree_valid = true;
  c->clock_valid = false;
  c->tree_syncs++;
  const clk::time_point t_pro = clk::now();
  if (prolong) {
    RB_TRY(prolong_new_octs(c, born));
    if (c->state_newer == 0) c->state_newer = 1;
  }
  c->sync_ms[4] = ms_since(t_pro);
  c->sync_ms[0] = ms_since(t_start);
  if (sync_trace())
    fprintf(stderr, "[rb sync] %s: total %.2f ms (index %.2f, tables %.2f, boundary pairs %.2f, prolongation %.2f), "
            "%d levels built, %d kept, %zu son entries changed\n", incremental ? "incremental" : "full",
            c->sync_ms[0], c->sync_ms[1], c->sync_ms[2], c->sync_ms[3], c->sync_ms[4], c->levels_built,
            c->levels_reused, son_idx.size());
  return RB_OK;
}

int ensure_partial(rb_context* c, int64_t n) {
  if (n <= c->partial_cap) return RB_OK;
  drop_graph(c);
  dfree(c->d_partial);
  RB_TRY(dalloc(&c->d_partial, (size_t)n * 4));
  c->partial_cap = n;
  return RB_OK;
}

int check_level(rb_context* c, int l) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (!c->have_tree) return fail(RB_ERR_STATE, "rb_sync_tree has not been called");
  if (l < 1 || l > c->mp.nlevelmax) return fail(RB_ERR_INVALID, "level %d out of range", l);
  return RB_OK;
}

int set_unew_impl(rb_context* c, int l) {
  Level& L = c->lv[l];
  if (!L.noct) return RB_OK;
  rb::copy_octs_kernel<<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
      c->d_uold, c->d_unew, L.d_active, L.noct, c->ncell, c->mp.ncoarse, c->gate);
  RB_CUDA(cudaGetLastError());
  if (c->hp.pressure_fix) {
    rb::pf_set_unew_kernel<<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
        c->d_uold, c->d_divu, c->d_enew, L.d_active, L.noct, c->ncell, c->mp.ncoarse, c->hp.smallr, c->gate);
    RB_CUDA(cudaGetLastError());
  }
  return RB_OK;
}

// pressure_fix: the pdV term of set_uold on the old state (before the copy)
int pdv_impl(rb_context* c, int l, const double* dt_dev, double dt) {
  Level& L = c->lv[l];
  RB_TRY(ensure_nres6(c, L));
  int e2;
  const int dx_pow2 = std::frexp(L.dx, &e2) == 0.5;
  rb::pdv_kernel<<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
      c->d_uold, L.d_active, L.d_nres6, L.noct, c->ncell, c->mp.ncoarse, L.dx, dx_pow2, dt_dev, dt, c->hp,
      c->d_enew, c->gate);
  RB_CUDA(cudaGetLastError());
  return RB_OK;
}

// pressure_fix: the energy fix of set_uold on the new state (after the copy)
int pf_fix_impl(rb_context* c, int l, const double* dt_dev, double dt, int skip_split) {
  Level& L = c->lv[l];
  rb::pf_fix_kernel<<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
      c->d_uold, c->d_divu, c->d_enew, c->d_son, L.d_active, L.noct, c->ncell, c->mp.ncoarse, L.dx, dt_dev, dt,
      c->hp.smallr, c->hp.beta_fix, skip_split, c->gate);
  RB_CUDA(cudaGetLastError());
  return RB_OK;
}

// set_uold (per call): with pressure_fix, dtnew(ilevel) is the dt of the
// level's last rb_godunov_fine
int set_uold_impl(rb_context* c, int l) {
  Level& L = c->lv[l];
  if (!L.noct) return RB_OK;
  if (c->hp.pressure_fix) RB_TRY(pdv_impl(c, l, nullptr, c->dt_godunov[l]));
  rb::copy_octs_kernel<<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
      c->d_unew, c->d_uold, L.d_active, L.noct, c->ncell, c->mp.ncoarse, c->gate);
  RB_CUDA(cudaGetLastError());
  if (c->hp.pressure_fix) RB_TRY(pf_fix_impl(c, l, nullptr, c->dt_godunov[l], 0));
  return RB_OK;
}

// set_uold + upload_fine of level l in one pass (set_uold_upload_kernel);
// with pressure_fix, the pdV term before, and the energy fix in the same
// pass. dt: *dt_dev if non-null.
int set_uold_upload_impl(rb_context* c, int l, const double* dt_dev, double dt) {
  Level& L = c->lv[l];
  if (!L.noct) return RB_OK;
  const int do_upload = (l < c->mp.nlevelmax && L.has_refined) ? 1 : 0;
  if (c->hp.pressure_fix) RB_TRY(pdv_impl(c, l, dt_dev, dt));
  rb::set_uold_upload_kernel<<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
      c->d_uold, c->d_unew, c->d_son, L.d_active, L.noct, c->ncell, c->mp.ncoarse, c->hp, do_upload, c->gate,
      c->d_divu, c->d_enew, L.dx, dt_dev, dt);
  RB_CUDA(cudaGetLastError());
  return RB_OK;
}

int upload_fine_impl(rb_context* c, int l) {
  if (l == c->mp.nlevelmax) return RB_OK;  // interpol_hydro.f90:16
  Level& L = c->lv[l];
  if (!L.noct || !L.has_refined) return RB_OK;
  rb::upload_fine_kernel<<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
      c->d_uold, c->d_son, L.d_active, L.noct, c->ncell, c->mp.ncoarse, c->hp, c->gate);
  RB_CUDA(cudaGetLastError());
  return RB_OK;
}

// make_boundary_hydro(l) (hydro/hydro_boundary.f90:5-260): the boundary
// regions in order, each in two launches (stage, write).
int boundary_impl(rb_context* c, int l) {
  const Level& L = c->lv[l];
  if (c->btype.empty() || L.h_boff.empty()) return RB_OK;
  for (size_t ib = 0; ib < c->btype.size(); ib++) {
    const int64_t n = L.h_boff[ib + 1] - L.h_boff[ib];
    if (n == 0) continue;
    for (int phase = 0; phase < 2; phase++) {
      rb::boundary_fill_kernel<<<grid_for(n * 8, 256), 256, 0, c->stream>>>(
          c->d_uold, L.d_bpair + 2 * L.h_boff[ib], n, c->ncell, c->mp.ncoarse, c->btype[ib], c->hp.smallr,
          c->d_bbuf, phase, c->gate);
      RB_CUDA(cudaGetLastError());
    }
  }
  return RB_OK;
}

int make_boundary_all(rb_context* c) {
  for (int l = 1; l <= c->mp.nlevelmax; l++) RB_TRY(boundary_impl(c, l));
  return RB_OK;
}

// Write the dense mirror of the finest level back into the oct layout and
// restrict it to the coarser levels (amr_step.f90:442, adaptive_loop.f90),
// when the dense mirror is ahead.
int sync_oct(rb_context* c) {
  if (!c->oct_stale) return RB_OK;
  Level& L = c->lv[c->finest];
  const int64_t vstr = (int64_t)c->dnx * c->dny * c->dnz;
  rb::dense_to_oct_kernel<<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
      c->d_dense[c->dense_cur], c->d_uold, L.d_active, c->d_cbase, L.noct, c->ncell, c->mp.ncoarse, c->dnx,
      c->dny, vstr);
  RB_CUDA(cudaGetLastError());
  for (int l = c->finest - 1; l >= 1; l--) RB_TRY(upload_fine_impl(c, l));
  c->oct_stale = false;
  return RB_OK;
}

// Any change of the oct-layout state makes the dense mirror stale.
inline void oct_changed(rb_context* c) {
  c->dense_valid = false;
  c->clock_valid = false;
}

// A device call wrote uold: the device copy is now the newer one.
inline void dev_wrote(rb_context* c) {
  if (c->have_state) c->state_newer = 1;
}

bool stream_shape_fits(const rb_context* c, int s) {
  const int tx = rb::kStreamShapes[s][0], ty = rb::kStreamShapes[s][1];
  if (rb::kStreamShapeV2[s] && (c->precision != RB_PREC_MIXED || !rb::stream2_supports(c->hp))) return false;
  return c->dnx % tx == 0 && c->dny % ty == 0 && c->dnx >= tx && c->dny >= ty;
}
int stream_items_of(const rb_context* c, int s, int hz) {
  return (c->dnx / rb::kStreamShapes[s][0]) * (c->dny / rb::kStreamShapes[s][1]) * (c->dnz / hz);
}
// z extent of a work item: the longest power of two <= 64 dividing nz that
// still gives >= 4 work items per SM
int default_stream_hz(const rb_context* c, int s) {
  int hz = 64;
  while (hz > 2 && (c->dnz % hz != 0 || stream_items_of(c, s, hz) < 4 * 148)) hz >>= 1;
  if (c->dnz % hz != 0) hz = 2;
  return hz;
}

// Allocate the dense mirror of the finest level (complete by construction of
// the callers) and the per-oct dense base offsets; pick the column shape.
int dense_prepare(rb_context* c) {
  const int lf = c->finest;
  Level& L = c->lv[lf];
  const int32_t nx = c->mp.nx << lf, ny = c->mp.ny << lf, nz = c->mp.nz << lf;
  if (c->d_dense[0] && c->dnx == nx && c->dny == ny && c->dnz == nz) return RB_OK;
  free_dense(c);
  c->dnx = nx; c->dny = ny; c->dnz = nz;
  const int64_t ncells = (int64_t)nx * ny * nz;
  RB_TRY(dalloc(&c->d_dense[0], (size_t)ncells * 5));
  RB_TRY(dalloc(&c->d_dense[1], (size_t)ncells * 5));
  std::vector<int64_t> cb(L.noct);
  for (int i = 0; i < L.noct; i++) {
    const int64_t* x = &c->coords[(size_t)(L.h_active[i] - 1) * 3];
    cb[i] = 2 * x[0] + (int64_t)nx * (2 * x[1] + (int64_t)ny * 2 * x[2]);
  }
  RB_TRY(dalloc(&c->d_cbase, cb.size()));
  RB_TRY(h2d(c, c->d_cbase, cb.data(), cb.size() * 8));
  // default column shape: the FP32-mixed kernel of stream2_kernel.cuh where
  // it applies, else the widest of 16x16, 16x8, 8x8 that divides the grid
  int shape = -1;
  for (int s : {6, 2, 1, 0})
    if (stream_shape_fits(c, s)) { shape = s; break; }
  c->stream_shape = shape;
  if (shape >= 0) {
    c->stream_hz = default_stream_hz(c, shape);
    c->stream_items = stream_items_of(c, shape, c->stream_hz);
  }
  c->dense_valid = false;
  return RB_OK;
}

rb::TileArgs tile_args(rb_context* c, Level& L, double dt) {
  rb::TileArgs a;
  memset(&a, 0, sizeof a);
  a.uold = c->d_uold;
  a.unew = c->d_unew;
  a.son = c->d_son;
  a.interp = L.d_interp_buf;
  a.tile_blk = L.d_tile_blk;
  a.tile_corr = L.nslot ? L.d_tile_corr : nullptr;
  a.tile_corr_off = L.nslot ? L.d_tile_corr_off : nullptr;
  a.corr_flux = L.d_corr_flux;
  a.divu = c->d_divu;    // null unless pressure_fix
  a.enew = c->d_enew;
  a.corr_tmp = L.d_corr_tmp;
  a.ncell = c->ncell;
  a.ninterp8 = (int64_t)L.ninterp * 8;
  a.ncoarse = c->mp.ncoarse;
  a.ntile = L.ntile;
  a.has_refined = L.has_refined;
  int e2;
  const double m = std::frexp(L.dx, &e2);
  a.dx_pow2 = (m == 0.5);
  a.fused = 0;
  a.dt = dt;
  a.dx = L.dx;
  a.inv_dx = 1.0 / L.dx;
  a.dt_dev = nullptr;
  a.partial = nullptr;
  a.gate = c->gate;
  a.hp = c->hp;
  return a;
}

int launch_tile(rb_context* c, int shape, const rb::TileArgs& a, int grid) {
  cudaError_t e = c->precision == RB_PREC_MIXED ? rb::launch_tile_mixed(shape, a, grid, c->stream)
                                                : rb::launch_tile_f64(shape, a, grid, c->stream);
  if (e != cudaSuccess) return fail(RB_ERR_CUDA, "godunov tile kernel launch failed: %s", cudaGetErrorString(e));
  return RB_OK;
}

// fuse_unew: the level has no finer octs, so at godunov time its unew is
// set_unew's copy of uold (no fine-to-coarse correction went into it); the
// kernel then starts the update from uold and writes unew without reading it
// (the caller skips set_unew's copy for the level). Same values bit for bit.
int godunov_impl(rb_context* c, int l, double dt, bool timed, const double* dt_dev = nullptr,
                 bool fuse_unew = false) {
  Level& L = c->lv[l];
  if (!L.noct) return RB_OK;
  if (!dt_dev && (!(dt > 0.0) || !std::isfinite(dt)))
    return fail(RB_ERR_INVALID, "dt=%g must be positive and finite", dt);
  if (L.ninterp) {
    rb::interp_blocks_kernel<<<(L.ninterp + 127) / 128, 128, 0, c->stream>>>(c->d_uold, L.d_interp7, L.ninterp,
                                                                             c->ncell, L.d_interp_buf, c->hp,
                                                                             c->gate);
    RB_CUDA(cudaGetLastError());
  }
  rb::TileArgs a = tile_args(c, L, dt);
  a.dt_dev = dt_dev;
  if (fuse_unew) a.fused = 2;
  if (!dt_dev) c->dt_godunov[l] = dt;
  if (timed) RB_CUDA(cudaEventRecord(c->ev0, c->stream));
  RB_TRY(launch_tile(c, L.shape, a, L.ntile));
  if (timed) RB_CUDA(cudaEventRecord(c->ev1, c->stream));
  if (L.ntgt) {
    rb::apply_corrections_kernel<<<(L.ntgt + 127) / 128, 128, 0, c->stream>>>(
        c->d_unew, L.d_tgt, L.d_tgt_off, L.d_contrib, L.ntgt, L.d_corr_flux, c->ncell, c->gate, c->d_divu, c->d_enew,
        L.d_corr_tmp);
    RB_CUDA(cudaGetLastError());
  }
  return RB_OK;
}

int courant_impl(rb_context* c, int l, double* dt_io, double* mass, double* ekin, double* eint,
                 bool with_set_unew = false) {
  Level& L = c->lv[l];
  if (!L.noct) return RB_OK;
  const int nt = 256;
  const int nblk = grid_for((int64_t)L.noct * 8, nt, 148 * 8);
  RB_TRY(ensure_partial(c, nblk));
  auto k = c->precision == RB_PREC_MIXED ? rb::courant_partial_kernel<256, true> : rb::courant_partial_kernel<256, false>;
  k<<<nblk, nt, 0, c->stream>>>(c->d_uold, c->d_son, L.d_active, L.noct, c->ncell, c->mp.ncoarse, L.dx, c->hp,
                                c->d_partial, c->gate, with_set_unew ? c->d_unew : nullptr,
                                with_set_unew ? c->d_divu : nullptr, with_set_unew ? c->d_enew : nullptr);
  RB_CUDA(cudaGetLastError());
  const double dt0 = c->hp.courant_factor * L.dx / c->hp.smallc;
  rb::reduce_partials_kernel<<<1, RB_RED_NT, 0, c->stream>>>(c->d_partial, nblk, *dt_io, dt0,
                                                            L.leaf_cells > 0 ? 1 : 0, c->d_red, 0);
  RB_CUDA(cudaGetLastError());
  RB_CUDA(cudaMemcpyAsync(c->h_red, c->d_red, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  RB_CUDA(cudaStreamSynchronize(c->stream));
  *dt_io = c->h_red[0];
  if (mass) *mass = c->h_red[1];
  if (ekin) *ekin = c->h_red[2];
  if (eint) *eint = c->h_red[3];
  return RB_OK;
}

// amr_step hydro call sequence (amr/amr_step.f90:320-445, 571-576;
// pm/newdt_fine.f90:47-51,177; amr/update_time.f90:330-331).
int amr_step_impl(rb_context* c, int l, int icount) {
  if (c->lv[l].noct == 0) return RB_OK;
  c->dtold[l] = c->dtnew[l];
  c->dtnew[l] = c->mp.boxlen / c->hp.smallc;
  double dt_all = c->dtnew[l], ma = 0, ek = 0, ei = 0;
  // a level without finer octs gets set_unew inside its godunov kernel
  const bool fuse = !c->lv[l].has_refined;
  RB_TRY(courant_impl(c, l, &dt_all, &ma, &ek, &ei, /*with_set_unew=*/!fuse));
  c->mass_tot += ma; c->ekin_tot += ek; c->eint_tot += ei;
  c->dtnew[l] = rb_min_host(c->dtnew[l], dt_all);
  if (l > c->mp.levelmin)
    c->dtnew[l] = rb_min_host(c->dtnew[l - 1] / (double)(float)c->mp.nsubcycle[l - 1], c->dtnew[l]);
  if (l < c->mp.nlevelmax) {
    if (c->lv[l + 1].noct > 0) {
      if (c->mp.nsubcycle[l] == 2) {
        RB_TRY(amr_step_impl(c, l + 1, 1));
        RB_TRY(amr_step_impl(c, l + 1, 2));
      } else {
        RB_TRY(amr_step_impl(c, l + 1, 1));
      }
    } else {
      c->dtold[l + 1] = c->dtnew[l] / (double)c->mp.nsubcycle[l];
      c->dtnew[l + 1] = c->dtnew[l] / (double)c->mp.nsubcycle[l];
      c->t += c->dtnew[l];
      c->nstep++;
    }
  } else {
    c->t += c->dtnew[l];
    c->nstep++;
  }
  RB_TRY(godunov_impl(c, l, c->dtnew[l], false, nullptr, fuse));
  c->cell_updates += c->lv[l].leaf_cells;
  RB_TRY(set_uold_upload_impl(c, l, nullptr, c->dtnew[l]));
  RB_TRY(boundary_impl(c, l));  // amr_step.f90:515
  if (l > c->mp.levelmin) {
    if (c->mp.nsubcycle[l - 1] == 1) c->dtnew[l - 1] = c->dtnew[l];
    if (icount == 2) c->dtnew[l - 1] = c->dtold[l] + c->dtnew[l];
  }
  return RB_OK;
}

// ---- device-scheduled coarse steps ----------------------------------------
// Twin of amr_step_impl with the same launches, in the same order, on the same
// stream; the scalar scheduler state lives in c->d_sched (sched_* kernels)
// and every level kernel is gated on c->d_sched[RB_S_DONE].
int courant_blocks(const rb_context* c, int l) { return grid_for((int64_t)c->lv[l].noct * 8, 256, 148 * 8); }

int amr_step_dev(rb_context* c, int l, int icount) {
  Level& L = c->lv[l];
  if (L.noct == 0) return RB_OK;
  double* s = c->d_sched;
  const int nblk = courant_blocks(c, l);
  auto k = c->precision == RB_PREC_MIXED ? rb::courant_partial_kernel<256, true> : rb::courant_partial_kernel<256, false>;
  // + set_unew, which a level without finer octs gets in its godunov kernel
  const bool fuse = !L.has_refined;
  k<<<nblk, 256, 0, c->stream>>>(c->d_uold, c->d_son, L.d_active, L.noct, c->ncell, c->mp.ncoarse, L.dx, c->hp,
                                 c->d_partial, c->gate, fuse ? nullptr : c->d_unew, fuse ? nullptr : c->d_divu,
                                 fuse ? nullptr : c->d_enew);
  RB_CUDA(cudaGetLastError());
  const double nsub_prev = l > c->mp.levelmin ? (double)(float)c->mp.nsubcycle[l - 1] : 1.0;
  rb::sched_courant_kernel<<<1, RB_RED_NT, 0, c->stream>>>(
      c->d_partial, nblk, l, c->mp.levelmin, c->hp.courant_factor * L.dx / c->hp.smallc, L.leaf_cells > 0 ? 1 : 0,
      c->mp.boxlen / c->hp.smallc, nsub_prev, s);
  RB_CUDA(cudaGetLastError());
  if (l < c->mp.nlevelmax) {
    if (c->lv[l + 1].noct > 0) {
      RB_TRY(amr_step_dev(c, l + 1, 1));
      if (c->mp.nsubcycle[l] == 2) RB_TRY(amr_step_dev(c, l + 1, 2));
    } else {
      rb::sched_advance_kernel<<<1, 1, 0, c->stream>>>(s, l, 1, (double)c->mp.nsubcycle[l]);
    }
  } else {
    rb::sched_advance_kernel<<<1, 1, 0, c->stream>>>(s, l, 2, 1.0);
  }
  RB_CUDA(cudaGetLastError());
  RB_TRY(godunov_impl(c, l, 0.0, false, s + RB_S_DTNEW + l, fuse));
  RB_TRY(set_uold_upload_impl(c, l, s + RB_S_DTNEW + l, 0.0));
  RB_TRY(boundary_impl(c, l));
  if (l > c->mp.levelmin && (c->mp.nsubcycle[l - 1] == 1 || icount == 2)) {
    rb::sched_end_kernel<<<1, 1, 0, c->stream>>>(s, l, c->mp.nsubcycle[l - 1] == 1 ? 1 : 0, icount);
    RB_CUDA(cudaGetLastError());
  }
  return RB_OK;
}

int coarse_step_dev(rb_context* c) {
  rb::sched_gate_kernel<<<1, 1, 0, c->stream>>>(c->d_sched);
  RB_CUDA(cudaGetLastError());
  RB_TRY(amr_step_dev(c, c->mp.levelmin, 1));
  for (int l = c->mp.levelmin - 1; l >= 1; l--) RB_TRY(upload_fine_impl(c, l));
  rb::sched_finish_kernel<<<1, 1, 0, c->stream>>>(c->d_sched);
  RB_CUDA(cudaGetLastError());
  return RB_OK;
}

// leaf-cell updates of one coarse step: every amr_step(l) call adds the
// level's leaf cells (adaptive_loop.f90:204-207 counts the same cell-steps)
int64_t updates_per_coarse(const rb_context* c, int l) {
  if (l > c->mp.nlevelmax || c->lv[l].noct == 0) return 0;
  int64_t n = c->lv[l].leaf_cells;
  if (l < c->mp.nlevelmax && c->lv[l + 1].noct > 0) n += c->mp.nsubcycle[l] * updates_per_coarse(c, l + 1);
  return n;
}

// Enqueue `chunk` gated coarse steps, from a cached CUDA graph if asked.
int enqueue_chunk(rb_context* c, int chunk, bool use_graph) {
  if (!use_graph) {
    for (int k = 0; k < chunk; k++) RB_TRY(coarse_step_dev(c));
    return RB_OK;
  }
  if (!c->amr_graph || c->amr_chunk != chunk) {
    if (c->amr_graph) cudaGraphExecDestroy(c->amr_graph);
    c->amr_graph = nullptr;
    cudaGraph_t g;
    RB_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = RB_OK;
    for (int k = 0; k < chunk && rc == RB_OK; k++) rc = coarse_step_dev(c);
    cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
    if (rc) return rc;
    if (ce != cudaSuccess) return fail(RB_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&c->amr_graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
      c->amr_graph = nullptr;
      return fail(RB_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ce));
    }
    c->amr_chunk = chunk;
  }
  RB_CUDA(cudaGraphLaunch(c->amr_graph, c->stream));
  return RB_OK;
}

// Load the host scheduler state into the device clock; set the stop rule.
int sched_upload(rb_context* c, int64_t max_coarse, double t_end) {
  double* h = c->h_sched;
  for (int i = 0; i < RB_S_SIZE; i++) h[i] = 0.0;
  for (int l = 0; l < RB_NLV; l++) {
    h[RB_S_DTNEW + l] = c->dtnew[l];
    h[RB_S_DTOLD + l] = c->dtold[l];
  }
  h[RB_S_T] = c->t;
  h[RB_S_NSTEP] = (double)c->nstep;
  h[RB_S_TEND] = t_end;
  h[RB_S_MAXC] = (double)max_coarse;
  RB_CUDA(cudaMemcpyAsync(c->d_sched, h, RB_S_SIZE * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return RB_OK;
}

// Read the device clock back into the host scheduler state.
int sched_download(rb_context* c, int64_t* coarse_out) {
  RB_CUDA(cudaMemcpyAsync(c->h_sched, c->d_sched, RB_S_SIZE * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  RB_CUDA(cudaStreamSynchronize(c->stream));
  const double* h = c->h_sched;
  for (int l = 0; l < RB_NLV; l++) {
    c->dtnew[l] = h[RB_S_DTNEW + l];
    c->dtold[l] = h[RB_S_DTOLD + l];
  }
  c->t = h[RB_S_T];
  c->nstep = (int64_t)h[RB_S_NSTEP];
  c->mass_tot = h[RB_S_MASS];
  c->ekin_tot = h[RB_S_EKIN];
  c->eint_tot = h[RB_S_EINT];
  if (coarse_out) *coarse_out = (int64_t)h[RB_S_COARSE];
  return RB_OK;
}

// Asynchronous device-scheduled run (rb_run and the serving engine): begin
// loads the stop rule and the scheduler state, each chunk enqueues up to
// `chunk` coarse steps without waiting, end brings the state back.
int run_async_begin(rb_context* c, double t_end, int64_t max_coarse) {
  RB_TRY(sync_oct(c));
  oct_changed(c);
  int nblk = 1;
  for (int l = 1; l <= c->mp.nlevelmax; l++)
    if (c->lv[l].noct) nblk = std::max(nblk, courant_blocks(c, l));
  RB_TRY(ensure_partial(c, nblk));
  RB_TRY(sched_upload(c, max_coarse, t_end));
  c->gate = c->d_sched + RB_S_DONE;
  return RB_OK;
}

int run_async_chunk(rb_context* c, int chunk, bool use_graph) { return enqueue_chunk(c, chunk, use_graph); }

int run_async_end(rb_context* c, int64_t* coarse_out) {
  c->gate = nullptr;
  int64_t coarse = 0;
  RB_TRY(sched_download(c, &coarse));
  c->cell_updates += coarse * updates_per_coarse(c, c->mp.levelmin);
  c->clock_valid = false;
  if (coarse_out) *coarse_out = coarse;
  return RB_OK;
}

}  // namespace rbi

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* rb_version(void) { return "ramses_b200 0.1 (sm_100a)"; }

const char* rb_status_string(int s) {
  switch (s) {
    case RB_OK: return "ok";
    case RB_ERR_INVALID: return "invalid argument or unsupported parameter";
    case RB_ERR_STATE: return "call out of order";
    case RB_ERR_CUDA: return "CUDA error";
    case RB_ERR_NOMEM: return "out of memory";
    case RB_ERR_TREE: return "octree violates the refinement rules";
    case RB_ERR_NUMERIC: return "non-physical state";
    case RB_ERR_NO_DEVICE: return "no usable CUDA device";
    case RB_ERR_CAPACITY: return "request above a fixed capacity";
  }
  return "unknown status";
}

const char* rb_last_error(void) { return g_last_error.c_str(); }

int rb_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int rb_select_device(int device) {
  const int n = rb_device_count();
  if (device < 0 || device >= n) return fail(RB_ERR_NO_DEVICE, "device %d not visible (%d devices)", device, n);
  RB_CUDA(cudaSetDevice(device));
  return RB_OK;
}

int rb_create(const rb_hydro_params* hp, const rb_mesh_params* mp, int precision, rb_context** out) {
  if (!out) return fail(RB_ERR_INVALID, "null output pointer");
  *out = nullptr;
  RB_TRY(check_params(hp, mp));
  if (precision != RB_PREC_FP64 && precision != RB_PREC_MIXED)
    return fail(RB_ERR_INVALID, "precision must be RB_PREC_FP64 or RB_PREC_MIXED");
  if (rb_device_count() == 0) return fail(RB_ERR_NO_DEVICE, "no CUDA device visible");
  rb_context* c = new rb_context();
  c->hp = *hp;
  c->mp = *mp;
  c->precision = precision;
  c->ncell = (int64_t)mp->ncoarse + 8 * (int64_t)mp->ngridmax;
  auto bail = [&](int rc) { rb_destroy(c); return rc; };
  if (cudaGetDevice(&c->device) != cudaSuccess) return bail(fail(RB_ERR_NO_DEVICE, "cudaGetDevice failed"));
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess)
    return bail(fail(RB_ERR_CUDA, "stream/event creation failed"));
  {
    // the level tables' pool: freed blocks stay in it for the next re-sync
    cudaMemPoolProps props;
    memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = c->device;
    uint64_t keep_all = UINT64_MAX;
    if (cudaMemPoolCreate(&c->table_pool, &props) != cudaSuccess) {
      c->table_pool = nullptr;
      return bail(fail(RB_ERR_CUDA, "memory pool creation failed"));
    }
    if (cudaMemPoolSetAttribute(c->table_pool, cudaMemPoolAttrReleaseThreshold, &keep_all) != cudaSuccess)
      return bail(fail(RB_ERR_CUDA, "memory pool set-up failed"));
  }
  int rc;
  if ((rc = dalloc(&c->d_uold, (size_t)c->ncell * 5)) || (rc = dalloc(&c->d_unew, (size_t)c->ncell * 5)) ||
      (rc = dalloc(&c->d_son, (size_t)c->ncell)) ||
      (rc = dalloc(&c->d_stage, (size_t)c->ncell * 5)) || (rc = dalloc(&c->d_red, 8)) ||
      (rc = dalloc(&c->d_clock, 8)) || (rc = dalloc(&c->d_sched, RB_S_SIZE)))
    return bail(rc);
  if (c->hp.pressure_fix) {
    if ((rc = dalloc(&c->d_divu, (size_t)c->ncell)) || (rc = dalloc(&c->d_enew, (size_t)c->ncell))) return bail(rc);
    if (cudaMemsetAsync(c->d_divu, 0, (size_t)c->ncell * sizeof(double), c->stream) != cudaSuccess ||
        cudaMemsetAsync(c->d_enew, 0, (size_t)c->ncell * sizeof(double), c->stream) != cudaSuccess)
      return bail(fail(RB_ERR_CUDA, "initialising device buffers failed"));
  }
  if (cudaMallocHost((void**)&c->h_red, 8 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost((void**)&c->h_sched, RB_S_SIZE * sizeof(double)) != cudaSuccess)
    return bail(fail(RB_ERR_NOMEM, "pinned allocation failed"));
  if (cudaMemsetAsync(c->d_uold, 0, (size_t)c->ncell * 5 * sizeof(double), c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_unew, 0, (size_t)c->ncell * 5 * sizeof(double), c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_clock, 0, 8 * sizeof(double), c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return bail(fail(RB_ERR_CUDA, "initialising device buffers failed"));
  // make sure the kernel image for this GPU is present
  cudaError_t e = rb::launch_tile_f64(0, rb::TileArgs{}, 0, c->stream);
  if (e != cudaSuccess) return bail(fail(RB_ERR_NO_DEVICE, "tile kernel unavailable on this device: %s", cudaGetErrorString(e)));
  *out = c;
  return RB_OK;
}

int rb_destroy(rb_context* c) {
  if (!c) return RB_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_tree(c);
  if (c->stream) cudaStreamSynchronize(c->stream);  // the tables' pool frees are stream-ordered
  if (c->table_pool) cudaMemPoolDestroy(c->table_pool);
  c->table_pool = nullptr;
  dfree(c->d_uold); dfree(c->d_unew); dfree(c->d_son);
  dfree(c->d_divu); dfree(c->d_enew); dfree(c->d_bbuf);
  dfree(c->d_stage); dfree(c->d_partial); dfree(c->d_red); dfree(c->d_clock); dfree(c->d_sched);
  dfree(c->d_flag);
  if (c->h_red) cudaFreeHost(c->h_red);
  if (c->h_sched) cudaFreeHost(c->h_sched);
  for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
  c->evpool.clear();
  drop_graph(c);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return RB_OK;
}

int rb_sync_tree(rb_context* c, const int32_t* son, const int32_t* father, const int32_t* nbor,
                 const int32_t* numbl, const int32_t* active_igrid) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  int rc = sync_tree_impl(c, son, father, nbor, numbl, active_igrid);
  if (rc) free_tree(c);
  else c->synced_gen = c->tree_gen;  // the device now holds the host's current tree
  return rc;
}

int rb_set_boundary(rb_context* c, int32_t nboundary, const int32_t* boundary_type, const int32_t* numbb,
                    const int32_t* boundary_igrid) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (nboundary < 0 || nboundary > 6) return fail(RB_ERR_INVALID, "nboundary=%d must be 0..6", nboundary);
  if (nboundary > 0 && (!boundary_type || !numbb || !boundary_igrid))
    return fail(RB_ERR_INVALID, "null boundary array");
  std::vector<int32_t> bt(boundary_type, boundary_type + nboundary);
  for (int32_t t : bt)
    if (!((t >= 1 && t <= 6) || (t >= 11 && t <= 16)))
      return fail(RB_ERR_INVALID, "boundary_type %d not supported (walls 1-6, free 11-16; imposed 21-26 are not)", t);
  const int nl = c->mp.nlevelmax;
  std::vector<int64_t> off((size_t)nl * nboundary + 1, 0);
  for (int l = 1; l <= nl; l++)
    for (int ib = 0; ib < nboundary; ib++) {
      const int64_t k = (int64_t)(l - 1) * nboundary + ib;
      const int32_t n = numbb[ib + (int64_t)nboundary * (l - 1)];
      if (n < 0 || n > c->mp.ngridmax) return fail(RB_ERR_INVALID, "numbb(%d,%d)=%d out of range", ib + 1, l, n);
      off[k + 1] = off[k] + n;
    }
  c->btype = bt;
  c->boff = off;
  c->bgrid.assign(boundary_igrid, boundary_igrid + off.back());
  // the lists belong to the next rb_sync_tree: a synchronised tree is
  // dropped (the state it held in a dense mirror goes back to the octs), and
  // the tree it leaves behind is what that sync compares against
  if (c->have_tree) {
    RB_TRY(sync_oct(c));
    free_tree(c, true);  // the level tables stay for the comparison in the sync
  }
  return RB_OK;
}

int rb_make_boundary_hydro(rb_context* c, int l) {
  RB_TRY(check_level(c, l));
  RB_TRY(sync_oct(c));
  dev_wrote(c);
  RB_TRY(boundary_impl(c, l));
  RB_CUDA(cudaStreamSynchronize(c->stream));
  return RB_OK;
}

static int upload_impl(rb_context* c, const double* h, double* d) {
  if (!c || !h) return fail(RB_ERR_INVALID, "null argument");
  RB_CUDA(cudaMemcpyAsync(c->d_stage, h, (size_t)c->ncell * 5 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  rb::permute_f2d_kernel<<<grid_for(c->ncell, 256), 256, 0, c->stream>>>(c->d_stage, d, c->ncell, c->mp.ncoarse,
                                                                            c->mp.ngridmax, 5);
  RB_CUDA(cudaGetLastError());
  RB_CUDA(cudaStreamSynchronize(c->stream));
  return RB_OK;
}
static int download_impl(rb_context* c, const double* d, double* h) {
  if (!c || !h) return fail(RB_ERR_INVALID, "null argument");
  rb::permute_d2f_kernel<<<grid_for(c->ncell * 5, 256), 256, 0, c->stream>>>(d, c->d_stage, c->ncell, c->mp.ncoarse,
                                                                            c->mp.ngridmax, 5);
  RB_CUDA(cudaGetLastError());
  RB_CUDA(cudaMemcpyAsync(h, c->d_stage, (size_t)c->ncell * 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  RB_CUDA(cudaStreamSynchronize(c->stream));
  return RB_OK;
}

int rb_upload_state(rb_context* c, const double* uold) {
  RB_TRY(upload_impl(c, uold, c ? c->d_uold : nullptr));
  c->have_state = true;
  c->oct_stale = false;  // overwritten entirely
  oct_changed(c);
  c->state_newer = 0;
  c->h2d_state_bytes += c->ncell * 5 * (int64_t)sizeof(double);
  return RB_OK;
}
int rb_download_state(rb_context* c, double* uold) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  RB_TRY(sync_oct(c));
  RB_TRY(download_impl(c, c->d_uold, uold));
  if (c->have_state) c->state_newer = 0;
  c->d2h_state_bytes += c->ncell * 5 * (int64_t)sizeof(double);
  return RB_OK;
}

// ---- one level's rows of uold ----
// Runs of consecutive igrids of a level's active list, (first, count)
// pairs, cached until the next tree sync.
static const std::vector<int32_t>& level_runs(rb_context* c, int l) {
  Level& L = c->lv[l];
  if (L.runs_sync != c->tree_syncs) {
    L.runs.clear();
    const std::vector<int32_t>& a = L.h_active;
    for (size_t i = 0; i < a.size();) {
      size_t j = i + 1;
      while (j < a.size() && a[j] == a[j - 1] + 1) j++;
      L.runs.push_back(a[i]);
      L.runs.push_back((int32_t)(j - i));
      i = j;
    }
    L.runs_sync = c->tree_syncs;
  }
  return L.runs;
}
// The level's rows between the host array and the staging buffer, one copy
// per run, variable and cell position (same offsets on both sides).
static int level_rows_copy(rb_context* c, int l, double* h, bool to_device) {
  const std::vector<int32_t>& runs = level_runs(c, l);
  const size_t nc = (size_t)c->ncell;
  for (size_t r = 0; r < runs.size(); r += 2) {
    const size_t g0 = (size_t)runs[r] - 1, n = (size_t)runs[r + 1];
    for (int v = 0; v < 5; v++)
      for (int ind = 0; ind < 8; ind++) {
        const size_t off = v * nc + (size_t)c->mp.ncoarse + (size_t)ind * c->mp.ngridmax + g0;
        if (to_device)
          RB_CUDA(cudaMemcpyAsync(c->d_stage + off, h + off, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        else
          RB_CUDA(cudaMemcpyAsync(h + off, c->d_stage + off, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      }
  }
  return RB_OK;
}
static int check_level_transfer(rb_context* c, int ilevel, const void* uold) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (!uold) return fail(RB_ERR_INVALID, "null uold");
  if (!c->have_tree || !c->have_state) return fail(RB_ERR_STATE, "tree and state must be uploaded first");
  if (ilevel < 1 || ilevel > c->mp.nlevelmax) return fail(RB_ERR_INVALID, "ilevel=%d out of 1..%d", ilevel, c->mp.nlevelmax);
  return RB_OK;
}
int rb_upload_level_state(rb_context* c, int ilevel, const double* uold) {
  RB_TRY(check_level_transfer(c, ilevel, uold));
  RB_TRY(sync_oct(c));  // the device's own newer cells first, so the rows not sent stay current
  Level& L = c->lv[ilevel];
  if (L.noct == 0) return RB_OK;
  RB_TRY(level_rows_copy(c, ilevel, const_cast<double*>(uold), true));
  rb::permute_level_kernel<true><<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
      c->d_stage, c->d_uold, L.d_active, L.noct, c->ncell, c->mp.ncoarse, c->mp.ngridmax);
  RB_CUDA(cudaGetLastError());
  RB_CUDA(cudaStreamSynchronize(c->stream));
  oct_changed(c);
  c->h2d_state_bytes += (int64_t)L.noct * 8 * 5 * (int64_t)sizeof(double);
  return RB_OK;
}
int rb_download_level_state(rb_context* c, int ilevel, double* uold) {
  RB_TRY(check_level_transfer(c, ilevel, uold));
  RB_TRY(sync_oct(c));
  Level& L = c->lv[ilevel];
  if (L.noct == 0) return RB_OK;
  rb::permute_level_kernel<false><<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
      c->d_stage, c->d_uold, L.d_active, L.noct, c->ncell, c->mp.ncoarse, c->mp.ngridmax);
  RB_CUDA(cudaGetLastError());
  RB_TRY(level_rows_copy(c, ilevel, uold, false));
  RB_CUDA(cudaStreamSynchronize(c->stream));
  c->d2h_state_bytes += (int64_t)L.noct * 8 * 5 * (int64_t)sizeof(double);
  return RB_OK;
}

// ---- residency protocol of the drop-in boundary ----
int rb_note_tree_changed(rb_context* c) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  c->tree_gen++;
  return RB_OK;
}
int rb_note_host_state_written(rb_context* c) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  c->state_newer = 2;
  return RB_OK;
}
int rb_tree_needs_sync(rb_context* c, int32_t* needed) {
  if (!c || !needed) return fail(RB_ERR_INVALID, "null argument");
  *needed = (!c->have_tree || c->synced_gen != c->tree_gen) ? 1 : 0;
  return RB_OK;
}
int rb_ensure_device(rb_context* c, const int32_t* son, const int32_t* father, const int32_t* nbor,
                     const int32_t* numbl, const int32_t* active_igrid, int32_t nboundary,
                     const int32_t* boundary_type, const int32_t* numbb, const int32_t* boundary_igrid,
                     const double* uold) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (!c->have_tree || c->synced_gen != c->tree_gen) {
    RB_TRY(rb_set_boundary(c, nboundary, boundary_type, numbb, boundary_igrid));
    RB_TRY(rb_sync_tree(c, son, father, nbor, numbl, active_igrid));
    c->synced_gen = c->tree_gen;
  }
  if (!c->have_state || c->state_newer == 2) RB_TRY(rb_upload_state(c, uold));
  return RB_OK;
}
int rb_ensure_host(rb_context* c, double* uold) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (!uold) return fail(RB_ERR_INVALID, "null uold");
  if (c->have_state && c->state_newer == 1) RB_TRY(rb_download_state(c, uold));
  return RB_OK;
}
int rb_transfer_stats(rb_context* c, int64_t* h2d_state_bytes, int64_t* d2h_state_bytes, int64_t* tree_syncs,
                      int64_t* octs_prolonged) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (h2d_state_bytes) *h2d_state_bytes = c->h2d_state_bytes;
  if (d2h_state_bytes) *d2h_state_bytes = c->d2h_state_bytes;
  if (tree_syncs) *tree_syncs = c->tree_syncs;
  if (octs_prolonged) *octs_prolonged = c->octs_prolonged;
  return RB_OK;
}
int rb_sync_stats(rb_context* c, double* ms, int32_t* levels_built, int32_t* levels_reused) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (ms)
    for (int i = 0; i < 5; i++) ms[i] = c->sync_ms[i];
  if (levels_built) *levels_built = c->levels_built;
  if (levels_reused) *levels_reused = c->levels_reused;
  return RB_OK;
}
int rb_upload_unew(rb_context* c, const double* unew) { return upload_impl(c, unew, c ? c->d_unew : nullptr); }
int rb_download_pressure_fix(rb_context* c, double* divu, double* enew) {
  if (!c || !divu || !enew) return fail(RB_ERR_INVALID, "null argument");
  if (!c->hp.pressure_fix) return fail(RB_ERR_STATE, "the context was created without pressure_fix");
  for (int k = 0; k < 2; k++) {
    rb::permute_d2f_kernel<<<grid_for(c->ncell, 256), 256, 0, c->stream>>>(
        k == 0 ? c->d_divu : c->d_enew, c->d_stage, c->ncell, c->mp.ncoarse, c->mp.ngridmax, 1);
    RB_CUDA(cudaGetLastError());
    RB_CUDA(cudaMemcpyAsync(k == 0 ? divu : enew, c->d_stage, (size_t)c->ncell * sizeof(double),
                            cudaMemcpyDeviceToHost, c->stream));
    RB_CUDA(cudaStreamSynchronize(c->stream));
  }
  return RB_OK;
}
int rb_download_unew(rb_context* c, double* unew) { return download_impl(c, c ? c->d_unew : nullptr, unew); }

int rb_set_unew(rb_context* c, int l) {
  RB_TRY(check_level(c, l));
  RB_TRY(sync_oct(c));
  return set_unew_impl(c, l);
}
int rb_set_uold(rb_context* c, int l) {
  RB_TRY(check_level(c, l));
  RB_TRY(sync_oct(c));
  oct_changed(c);
  dev_wrote(c);
  return set_uold_impl(c, l);
}
int rb_upload_fine(rb_context* c, int l) {
  RB_TRY(check_level(c, l));
  RB_TRY(sync_oct(c));
  oct_changed(c);
  dev_wrote(c);
  return upload_fine_impl(c, l);
}

int rb_godunov_fine(rb_context* c, int l, double dt) {
  RB_TRY(check_level(c, l));
  RB_TRY(sync_oct(c));
  RB_TRY(godunov_impl(c, l, dt, true));
  RB_CUDA(cudaStreamSynchronize(c->stream));
  RB_CUDA(cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1));
  c->kernel_ms_avg = c->last_ms;
  return RB_OK;
}

int rb_courant_fine(rb_context* c, int l, double* dt_io, double* mass, double* ekin, double* eint) {
  RB_TRY(check_level(c, l));
  if (!dt_io) return fail(RB_ERR_INVALID, "null dt");
  RB_TRY(sync_oct(c));
  return courant_impl(c, l, dt_io, mass, ekin, eint);
}

int rb_coarse_step(rb_context* c, double* t_io, double* dtnew_out) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (!c->have_tree || !c->have_state) return fail(RB_ERR_STATE, "tree and state must be uploaded first");
  RB_TRY(sync_oct(c));
  oct_changed(c);
  dev_wrote(c);
  if (t_io) c->t = *t_io;
  c->mass_tot = c->ekin_tot = c->eint_tot = 0.0;
  RB_TRY(amr_step_impl(c, c->mp.levelmin, 1));
  for (int l = c->mp.levelmin - 1; l >= 1; l--) RB_TRY(upload_fine_impl(c, l));
  RB_CUDA(cudaStreamSynchronize(c->stream));
  if (t_io) *t_io = c->t;
  if (dtnew_out)
    for (int l = 1; l <= c->mp.nlevelmax; l++) dtnew_out[l - 1] = c->dtnew[l];
  c->clock_valid = false;
  return RB_OK;
}

int rb_run(rb_context* c, int max_steps, double t_end, int use_graph, double* t_io, int* steps_done) {
  if (steps_done) *steps_done = 0;
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (!c->have_tree || !c->have_state) return fail(RB_ERR_STATE, "tree and state must be uploaded first");
  if (max_steps < 0) return fail(RB_ERR_INVALID, "max_steps=%d must be non-negative", max_steps);
  if (std::isnan(t_end)) return fail(RB_ERR_INVALID, "t_end is NaN");
  if (t_io) c->t = *t_io;
  dev_wrote(c);
  struct GateScope {
    rb_context* c;
    ~GateScope() { c->gate = nullptr; }
  } scope{c};
  RB_TRY(run_async_begin(c, t_end, max_steps));
  const int chunk = std::max(1, std::min(max_steps, 8));
  RB_CUDA(cudaEventRecord(c->ev0, c->stream));
  RB_CUDA(cudaEventRecord(c->ev1, c->stream));
  for (int64_t launched = 0; launched < max_steps;) {
    RB_TRY(run_async_chunk(c, chunk, use_graph != 0));
    RB_CUDA(cudaEventRecord(c->ev1, c->stream));
    launched += chunk;
    RB_CUDA(cudaMemcpyAsync(c->h_sched, c->d_sched, RB_S_SIZE * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    RB_CUDA(cudaStreamSynchronize(c->stream));
    const double* h = c->h_sched;
    if (!(h[RB_S_T] < h[RB_S_TEND]) || !(h[RB_S_COARSE] < h[RB_S_MAXC])) break;
  }
  int64_t coarse = 0;
  RB_TRY(run_async_end(c, &coarse));
  RB_CUDA(cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1));  // device time of all chunks
  if (t_io) *t_io = c->t;
  if (steps_done) *steps_done = (int)coarse;
  return RB_OK;
}

int rb_hydro_flag(rb_context* c, int l, const rb_refine_params* rp, int32_t* flag1, int64_t* nflag_added) {
  if (nflag_added) *nflag_added = 0;
  RB_TRY(check_level(c, l));
  if (!rp || !flag1) return fail(RB_ERR_INVALID, "null argument");
  if (!c->have_state) return fail(RB_ERR_STATE, "the state must be uploaded first");
  // hydro_flag.f90:43-44 and 60-70: nothing to do on the finest level, on an
  // empty level, or with every criterion switched off
  if (l == c->mp.nlevelmax) return RB_OK;
  Level& L = c->lv[l];
  if (!L.noct) return RB_OK;
  if (rp->err_grad_d == -1.0 && rp->err_grad_p == -1.0 && rp->err_grad_u == -1.0) return RB_OK;
  RB_TRY(sync_oct(c));
  RB_TRY(ensure_nbor6(c, L));
  const int64_t n = (int64_t)L.noct * 8;
  if (n > c->flag_cap) {
    dfree(c->d_flag);
    RB_TRY(dalloc(&c->d_flag, (size_t)n));
    c->flag_cap = n;
  }
  rb::hydro_flag_kernel<<<grid_for(n, 256), 256, 0, c->stream>>>(c->d_uold, c->d_son, L.d_active, L.d_nbor6, L.noct,
                                                                 c->ncell, c->mp.ncoarse, c->hp, *rp, c->d_flag);
  RB_CUDA(cudaGetLastError());
  std::vector<uint8_t> f((size_t)n);
  RB_CUDA(cudaMemcpyAsync(f.data(), c->d_flag, (size_t)n, cudaMemcpyDeviceToHost, c->stream));
  RB_CUDA(cudaStreamSynchronize(c->stream));
  int64_t added = 0;
  for (int i = 0; i < L.noct; i++)
    for (int ind = 0; ind < 8; ind++) {
      if (!f[(size_t)i * 8 + ind]) continue;
      const int64_t icell = fcell(c, ind + 1, L.h_active[i]);
      if (flag1[icell] == 0) added++;
      flag1[icell] = 1;
    }
  if (nflag_added) *nflag_added = added;
  return RB_OK;
}

int rb_cell_updates(rb_context* c, int64_t* out) {
  if (!c || !out) return fail(RB_ERR_INVALID, "null argument");
  *out = c->cell_updates;
  return RB_OK;
}

int rb_tile_shape_info(int shape, int* tx, int* ty, int* tz, int* nthreads) {
  if (shape < 0 || shape >= rb::kNumTileShapes) return fail(RB_ERR_INVALID, "tile shape %d out of range", shape);
  if (tx) *tx = rb::kTileShapes[shape].tx;
  if (ty) *ty = rb::kTileShapes[shape].ty;
  if (tz) *tz = rb::kTileShapes[shape].tz;
  if (nthreads) *nthreads = rb::kTileShapes[shape].nthreads;
  return RB_OK;
}

int rb_get_tile_shape(rb_context* c, int l, int* shape) {
  RB_TRY(check_level(c, l));
  if (!shape) return fail(RB_ERR_INVALID, "null argument");
  *shape = c->lv[l].shape;
  return RB_OK;
}

int rb_synchronize(rb_context* c) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  RB_CUDA(cudaStreamSynchronize(c->stream));
  return RB_OK;
}

int rb_get_stream(rb_context* c, void** s) {
  if (!c || !s) return fail(RB_ERR_INVALID, "null argument");
  *s = (void*)c->stream;
  return RB_OK;
}

int rb_last_kernel_ms(rb_context* c, float* ms) {
  if (!c || !ms) return fail(RB_ERR_INVALID, "null argument");
  *ms = c->kernel_ms_avg;
  return RB_OK;
}

int rb_last_run_ms(rb_context* c, float* ms) {
  if (!c || !ms) return fail(RB_ERR_INVALID, "null argument");
  *ms = c->last_ms;
  return RB_OK;
}

int rb_unsplit(const rb_hydro_params* hp, const double* uin, const double* gravin, const double* pin, double* flux,
               double* tmp, double dx, double dy, double dz, double dt, int ngrid, int nvector) {
  (void)pin;
  rb_mesh_params mp;
  memset(&mp, 0, sizeof mp);
  mp.nx = mp.ny = mp.nz = mp.ncoarse = 1;
  mp.ngridmax = 1; mp.nlevelmax = 1; mp.levelmin = 1; mp.nvector = 1; mp.boxlen = 1.0;
  RB_TRY(check_params(hp, &mp));
  if (!uin || !flux || !tmp) return fail(RB_ERR_INVALID, "null array");
  if (nvector < 1 || ngrid < 0 || ngrid > nvector) return fail(RB_ERR_INVALID, "bad ngrid/nvector");
  if (ngrid == 0) return RB_OK;
  if (rb_device_count() == 0) return fail(RB_ERR_NO_DEVICE, "no CUDA device visible");
  const size_t nin = (size_t)nvector * 216, nfl = (size_t)nvector * 27;
  double *d_uin = nullptr, *d_g = nullptr, *d_flux = nullptr, *d_tmp = nullptr;
  int rc = RB_OK;
  if ((rc = dalloc(&d_uin, nin * 5)) || (rc = dalloc(&d_g, nin * 3)) || (rc = dalloc(&d_flux, nfl * 15)) ||
      (rc = dalloc(&d_tmp, nfl * 6))) {
    dfree(d_uin); dfree(d_g); dfree(d_flux); dfree(d_tmp);
    return rc;
  }
  cudaError_t e = cudaMemcpy(d_uin, uin, nin * 5 * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = gravin ? cudaMemcpy(d_g, gravin, nin * 3 * sizeof(double), cudaMemcpyHostToDevice)
               : cudaMemset(d_g, 0, nin * 3 * sizeof(double));
  // outputs keep the caller's values outside the computed ranges
  if (e == cudaSuccess) e = cudaMemcpy(d_flux, flux, nfl * 15 * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_tmp, tmp, nfl * 6 * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rb::unsplit_fortran_kernel<<<ngrid, 64>>>(d_uin, d_g, d_flux, d_tmp, dx, dy, dz, dt, ngrid, nvector, *hp);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(flux, d_flux, nfl * 15 * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(tmp, d_tmp, nfl * 6 * sizeof(double), cudaMemcpyDeviceToHost);
  dfree(d_uin); dfree(d_g); dfree(d_flux); dfree(d_tmp);
  if (e != cudaSuccess) return fail(RB_ERR_CUDA, "rb_unsplit: %s", cudaGetErrorString(e));
  return RB_OK;
}

int rb_set_tile_order(rb_context* c, int order) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (order != 0 && order != 1) return fail(RB_ERR_INVALID, "tile order %d must be 0 (Morton) or 1 (z slabs)", order);
  if (order == c->tile_order) return RB_OK;
  c->tile_order = order;
  if (!c->have_tree) return RB_OK;
  drop_graph(c);
  RB_TRY(sync_oct(c));
  for (int l = 1; l <= c->mp.nlevelmax; l++)
    if (c->lv[l].noct) RB_TRY(build_level_tables(c, l, c->idx));
  return RB_OK;
}

int rb_set_tile_shape(rb_context* c, int l, int shape) {
  RB_TRY(check_level(c, l));
  Level& L = c->lv[l];
  if (shape >= rb::kNumTileShapes) return fail(RB_ERR_INVALID, "tile shape %d out of range", shape);
  drop_graph(c);
  RB_TRY(sync_oct(c));
  L.shape_user = true;
  if (shape >= 0 || L.noct == 0) {
    L.shape = shape >= 0 ? shape : L.shape;
    return build_level_tables(c, l, c->idx);
  }
  // time every shape on the current state against a scratch copy of unew
  int best = -1;
  float best_ms = 1e30f;
  double* keep_unew = c->d_unew;
  for (int s = 0; s < rb::kNumTileShapes; s++) {
    const size_t smem = c->precision == RB_PREC_MIXED ? rb::tile_smem_mixed(s) : rb::tile_smem_f64(s);
    if (smem > 227 * 1024 || !shape_fits(c, l, s)) continue;
    L.shape = s;
    RB_TRY(build_level_tables(c, l, c->idx));
    if (L.ninterp) {
      rb::interp_blocks_kernel<<<(L.ninterp + 127) / 128, 128, 0, c->stream>>>(c->d_uold, L.d_interp7, L.ninterp,
                                                                               c->ncell, L.d_interp_buf, c->hp,
                                                                               nullptr);
      RB_CUDA(cudaGetLastError());
    }
    RB_CUDA(cudaMemcpyAsync(c->d_stage, keep_unew, (size_t)c->ncell * 5 * sizeof(double), cudaMemcpyDeviceToDevice,
                            c->stream));
    c->d_unew = c->d_stage;
    rb::TileArgs a = tile_args(c, L, 1e-30);
    c->d_unew = keep_unew;
    // the trial launches leave divu/enew alone (shapes are timed on the
    // variant without the pressure fix)
    a.divu = a.enew = a.corr_tmp = nullptr;
    float ms = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
      RB_CUDA(cudaEventRecord(c->ev0, c->stream));
      int rc = launch_tile(c, s, a, L.ntile);
      if (rc) return rc;
      RB_CUDA(cudaEventRecord(c->ev1, c->stream));
      RB_CUDA(cudaEventSynchronize(c->ev1));
      float t = 0.f;
      RB_CUDA(cudaEventElapsedTime(&t, c->ev0, c->ev1));
      if (rep > 0) ms = std::min(ms, t);
    }
    if (ms < best_ms) { best_ms = ms; best = s; }
  }
  if (best < 0) return fail(RB_ERR_INVALID, "no tile shape fits on this device");
  L.shape = best;
  return build_level_tables(c, l, c->idx);
}

// Device-resident uniform-grid stepper: one complete finest level, every
// coarser level fully refined (no leaf cell). Per step: the fused tile kernel
// (unew = uold + fluxes, CFL partials of the new state) and the device clock
// update; the two state buffers alternate; optionally captured as one graph.
static int uniform_run_tiles(rb_context* c, int nsteps, int use_graph, double* t_io, double* dt_last_out) {
  RB_TRY(sync_oct(c));
  c->dense_valid = false;
  const int lf = c->finest;
  Level& L = c->lv[lf];
  // (with physical boundaries the level covers the box, not the extended
  // coarse grid, and the run takes the amr_step sequence below)
  if (lf < 1 || (!L.complete && c->btype.empty()) || L.leaf_cells != (int64_t)L.noct * 8)
    return fail(RB_ERR_STATE, "rb_uniform_run needs a complete, unrefined finest level");
  for (int l = 1; l < lf; l++)
    if (c->lv[l].leaf_cells != 0) return fail(RB_ERR_STATE, "level %d has leaf cells: not a uniform grid", l);
  if (L.ninterp || L.nslot) return fail(RB_ERR_STATE, "uniform level unexpectedly needs prolongation/corrections");
  RB_TRY(ensure_partial(c, std::max<int64_t>(L.ntile, 1)));
  const double dt_max = c->mp.boxlen / c->hp.smallc;
  const double dt0 = c->hp.courant_factor * L.dx / c->hp.smallc;
  if (t_io) c->t = *t_io;
  if (!c->clock_valid) {
    // newdt_fine + courant_fine on the starting state
    const int nblk = grid_for((int64_t)L.noct * 8, 256, 148 * 8);
    RB_TRY(ensure_partial(c, nblk));
    rb::courant_partial_kernel<256><<<nblk, 256, 0, c->stream>>>(c->d_uold, c->d_son, L.d_active, L.noct, c->ncell,
                                                                c->mp.ncoarse, L.dx, c->hp, c->d_partial, nullptr);
    RB_CUDA(cudaGetLastError());
    rb::reduce_partials_kernel<<<1, RB_RED_NT, 0, c->stream>>>(c->d_partial, nblk, dt_max, dt0, 1, c->d_red, 0);
    RB_CUDA(cudaGetLastError());
    c->h_red[0] = c->t;
    RB_CUDA(cudaMemcpyAsync(c->d_clock, c->d_red, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    RB_CUDA(cudaMemcpyAsync(c->d_clock + 1, c->h_red, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    RB_CUDA(cudaStreamSynchronize(c->stream));
    c->clock_valid = true;
  } else if (t_io) {
    c->h_red[0] = c->t;
    RB_CUDA(cudaMemcpyAsync(c->d_clock + 1, c->h_red, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  auto enqueue = [&](double* cur, double* nxt) -> int {
    rb::TileArgs a = tile_args(c, L, 0.0);
    a.uold = cur;
    a.unew = nxt;
    a.fused = 1;
    a.dt_dev = c->d_clock;
    a.partial = c->d_partial;
    RB_TRY(launch_tile(c, L.shape, a, L.ntile));
    rb::reduce_partials_kernel<<<1, RB_RED_NT, 0, c->stream>>>(c->d_partial, L.ntile, dt_max, dt0, 1, c->d_clock, 1);
    RB_CUDA(cudaGetLastError());
    return RB_OK;
  };
  if (nsteps > 0) {
    if (use_graph) {
      if (!(c->graph && c->graph_steps == nsteps && c->graph_cur == c->d_uold)) {
        drop_graph(c);
        cudaGraph_t g;
        RB_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        double *cur = c->d_uold, *nxt = c->d_unew;
        int rc = RB_OK;
        for (int s = 0; s < nsteps && rc == RB_OK; s++) {
          rc = enqueue(cur, nxt);
          std::swap(cur, nxt);
        }
        cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
        if (rc) return rc;
        if (ce != cudaSuccess) return fail(RB_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&c->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) { c->graph = nullptr; return fail(RB_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ce)); }
        c->graph_steps = nsteps;
        c->graph_cur = c->d_uold;
      }
      RB_CUDA(cudaEventRecord(c->ev0, c->stream));
      RB_CUDA(cudaGraphLaunch(c->graph, c->stream));
      RB_CUDA(cudaEventRecord(c->ev1, c->stream));
    } else {
      // per-step events around the tile kernel only (kernel-time roofline)
      const int ntimed = std::min(nsteps, 4096);
      while ((int)c->evpool.size() < 2 * ntimed) {
        cudaEvent_t e;
        RB_CUDA(cudaEventCreate(&e));
        c->evpool.push_back(e);
      }
      RB_CUDA(cudaEventRecord(c->ev0, c->stream));
      double *cur = c->d_uold, *nxt = c->d_unew;
      for (int s = 0; s < nsteps; s++) {
        if (s < ntimed) RB_CUDA(cudaEventRecord(c->evpool[2 * s], c->stream));
        rb::TileArgs a = tile_args(c, L, 0.0);
        a.uold = cur;
        a.unew = nxt;
        a.fused = 1;
        a.dt_dev = c->d_clock;
        a.partial = c->d_partial;
        RB_TRY(launch_tile(c, L.shape, a, L.ntile));
        if (s < ntimed) RB_CUDA(cudaEventRecord(c->evpool[2 * s + 1], c->stream));
        rb::reduce_partials_kernel<<<1, RB_RED_NT, 0, c->stream>>>(c->d_partial, L.ntile, dt_max, dt0, 1,
                                                                  c->d_clock, 1);
        RB_CUDA(cudaGetLastError());
        std::swap(cur, nxt);
      }
      RB_CUDA(cudaEventRecord(c->ev1, c->stream));
      RB_CUDA(cudaEventSynchronize(c->ev1));
      double tot = 0.0;
      for (int s = 0; s < ntimed; s++) {
        float ms = 0.f;
        RB_CUDA(cudaEventElapsedTime(&ms, c->evpool[2 * s], c->evpool[2 * s + 1]));
        tot += ms;
      }
      c->kernel_ms_avg = ntimed ? (float)(tot / ntimed) : 0.f;
    }
    if (nsteps & 1) {
      std::swap(c->d_uold, c->d_unew);  // a cached odd-length graph is recaptured on the next call
    }
  }
  // coarser levels: restriction of the final state (adaptive_loop.f90 + amr_step.f90:442)
  for (int l = lf - 1; l >= 1; l--) RB_TRY(upload_fine_impl(c, l));
  RB_CUDA(cudaMemcpyAsync(c->h_red, c->d_clock, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  RB_CUDA(cudaStreamSynchronize(c->stream));
  if (nsteps > 0) RB_CUDA(cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1));
  c->t = c->h_red[1];
  c->nstep += nsteps;
  c->cell_updates += (int64_t)nsteps * L.leaf_cells;
  c->dtnew[lf] = c->h_red[0];
  c->mass_tot = c->h_red[2];
  c->ekin_tot = c->h_red[3];
  c->eint_tot = c->h_red[4];
  if (t_io) *t_io = c->t;
  if (dt_last_out) *dt_last_out = c->h_red[0];
  return RB_OK;
}

// z-streaming stepper over the dense mirror of the finest level.
static int uniform_run_dense(rb_context* c, int nsteps, int use_graph, double* t_io, double* dt_last_out) {
  const int lf = c->finest;
  Level& L = c->lv[lf];
  RB_TRY(dense_prepare(c));
  if (c->stream_shape < 0) return uniform_run_tiles(c, nsteps, use_graph, t_io, dt_last_out);
  const double dt_max = c->mp.boxlen / c->hp.smallc;
  const double dt0 = c->hp.courant_factor * L.dx / c->hp.smallc;
  const int64_t vstr = (int64_t)c->dnx * c->dny * c->dnz;
  if (t_io) c->t = *t_io;
  if (!c->dense_valid) {
    RB_TRY(sync_oct(c));
    rb::oct_to_dense_kernel<<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
        c->d_uold, c->d_dense[c->dense_cur], L.d_active, c->d_cbase, L.noct, c->ncell, c->mp.ncoarse, c->dnx,
        c->dny, vstr);
    RB_CUDA(cudaGetLastError());
    c->dense_valid = true;
    drop_graph(c);
  }
  RB_TRY(ensure_partial(c, std::max<int64_t>(c->stream_items, grid_for((int64_t)L.noct * 8, 256, 148 * 8))));
  if (!c->clock_valid) {
    const int nblk = grid_for((int64_t)L.noct * 8, 256, 148 * 8);
    rb::courant_partial_kernel<256><<<nblk, 256, 0, c->stream>>>(c->d_uold, c->d_son, L.d_active, L.noct, c->ncell,
                                                                c->mp.ncoarse, L.dx, c->hp, c->d_partial, nullptr);
    RB_CUDA(cudaGetLastError());
    rb::reduce_partials_kernel<<<1, RB_RED_NT, 0, c->stream>>>(c->d_partial, nblk, dt_max, dt0, 1, c->d_red, 0);
    RB_CUDA(cudaGetLastError());
    c->h_red[0] = c->t;
    RB_CUDA(cudaMemcpyAsync(c->d_clock, c->d_red, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    RB_CUDA(cudaMemcpyAsync(c->d_clock + 1, c->h_red, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    RB_CUDA(cudaStreamSynchronize(c->stream));
    c->clock_valid = true;
  } else if (t_io) {
    c->h_red[0] = c->t;
    RB_CUDA(cudaMemcpyAsync(c->d_clock + 1, c->h_red, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  rb::StreamArgs sa;
  memset(&sa, 0, sizeof sa);
  sa.partial = c->d_partial;
  sa.dt_dev = c->d_clock;
  sa.nx = c->dnx; sa.ny = c->dny; sa.nz = c->dnz;
  sa.hz = c->stream_hz;
  int e2;
  sa.dx_pow2 = std::frexp(L.dx, &e2) == 0.5;
  sa.dx = L.dx;
  sa.inv_dx = 1.0 / L.dx;
  sa.hp = c->hp;
  auto step = [&](int s_idx, bool timed) -> int {
    sa.uin = c->d_dense[(c->dense_cur + s_idx) & 1];
    sa.uout = c->d_dense[(c->dense_cur + s_idx + 1) & 1];
    if (timed) RB_CUDA(cudaEventRecord(c->evpool[2 * s_idx], c->stream));
    cudaError_t e = c->precision == RB_PREC_MIXED
                        ? rb::launch_stream_mixed(c->stream_shape, sa, c->stream_items, c->stream)
                        : rb::launch_stream_f64(c->stream_shape, sa, c->stream_items, c->stream);
    if (e != cudaSuccess) return fail(RB_ERR_CUDA, "stream kernel launch failed: %s", cudaGetErrorString(e));
    if (timed) RB_CUDA(cudaEventRecord(c->evpool[2 * s_idx + 1], c->stream));
    rb::reduce_partials_kernel<<<1, RB_RED_NT, 0, c->stream>>>(c->d_partial, c->stream_items, dt_max, dt0, 1,
                                                              c->d_clock, 1);
    RB_CUDA(cudaGetLastError());
    return RB_OK;
  };
  if (nsteps > 0) {
    if (use_graph) {
      if (!(c->graph && c->graph_steps == nsteps && c->graph_cur == c->d_dense[c->dense_cur])) {
        drop_graph(c);
        cudaGraph_t g;
        RB_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int rc = RB_OK;
        for (int s = 0; s < nsteps && rc == RB_OK; s++) rc = step(s, false);
        cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
        if (rc) return rc;
        if (ce != cudaSuccess) return fail(RB_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&c->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) { c->graph = nullptr; return fail(RB_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ce)); }
        c->graph_steps = nsteps;
        c->graph_cur = c->d_dense[c->dense_cur];
      }
      RB_CUDA(cudaEventRecord(c->ev0, c->stream));
      RB_CUDA(cudaGraphLaunch(c->graph, c->stream));
      RB_CUDA(cudaEventRecord(c->ev1, c->stream));
    } else {
      const int ntimed = std::min(nsteps, 4096);
      while ((int)c->evpool.size() < 2 * ntimed) {
        cudaEvent_t e;
        RB_CUDA(cudaEventCreate(&e));
        c->evpool.push_back(e);
      }
      RB_CUDA(cudaEventRecord(c->ev0, c->stream));
      for (int s = 0; s < nsteps; s++) RB_TRY(step(s, s < ntimed));
      RB_CUDA(cudaEventRecord(c->ev1, c->stream));
      RB_CUDA(cudaEventSynchronize(c->ev1));
      double tot = 0.0;
      for (int s = 0; s < ntimed; s++) {
        float ms = 0.f;
        RB_CUDA(cudaEventElapsedTime(&ms, c->evpool[2 * s], c->evpool[2 * s + 1]));
        tot += ms;
      }
      c->kernel_ms_avg = ntimed ? (float)(tot / ntimed) : 0.f;
    }
    c->dense_cur = (c->dense_cur + nsteps) & 1;
    c->oct_stale = true;
  }
  RB_CUDA(cudaMemcpyAsync(c->h_red, c->d_clock, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  RB_CUDA(cudaStreamSynchronize(c->stream));
  if (nsteps > 0) RB_CUDA(cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1));
  c->t = c->h_red[1];
  c->nstep += nsteps;
  c->cell_updates += (int64_t)nsteps * L.leaf_cells;
  c->dtnew[lf] = c->h_red[0];
  c->mass_tot = c->h_red[2];
  c->ekin_tot = c->h_red[3];
  c->eint_tot = c->h_red[4];
  if (t_io) *t_io = c->t;
  if (dt_last_out) *dt_last_out = c->h_red[0];
  return RB_OK;
}

// Autotuner of the z-streaming step: times every column shape / register
// budget (kStreamShapes) and z extent (4..64) on the live state, reading the
// current dense buffer and writing the other one (the state, the clock and t
// are left unchanged), and keeps the fastest.
int rb_autotune_uniform(rb_context* c, int* shape_out, int* hz_out, float* ms_out) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  const int lf = c->finest;
  if (!c->have_tree || !c->have_state || lf < 1 || !c->lv[lf].complete)
    return fail(RB_ERR_STATE, "autotuning needs a uniform grid with its state uploaded");
  if (c->hp.slope_type == 3) return fail(RB_ERR_STATE, "slope_type 3 runs on the oct tiles only");
  Level& L = c->lv[lf];
  RB_TRY(dense_prepare(c));
  if (c->stream_shape < 0) return fail(RB_ERR_STATE, "grid too small for the z-streaming kernel");
  if (!c->dense_valid) {
    RB_TRY(sync_oct(c));
    const int64_t vstr = (int64_t)c->dnx * c->dny * c->dnz;
    rb::oct_to_dense_kernel<<<grid_for((int64_t)L.noct * 8, 256), 256, 0, c->stream>>>(
        c->d_uold, c->d_dense[c->dense_cur], L.d_active, c->d_cbase, L.noct, c->ncell, c->mp.ncoarse, c->dnx,
        c->dny, vstr);
    RB_CUDA(cudaGetLastError());
    c->dense_valid = true;
  }
  // a representative dt in a scratch slot of the reduction buffer (the
  // trial launches read it there)
  {
    double d = c->mp.boxlen / c->hp.smallc;
    const int nblk = grid_for((int64_t)L.noct * 8, 256, 148 * 8);
    RB_TRY(ensure_partial(c, nblk));
    rb::courant_partial_kernel<256><<<nblk, 256, 0, c->stream>>>(c->d_uold, c->d_son, L.d_active, L.noct, c->ncell,
                                                                c->mp.ncoarse, L.dx, c->hp, c->d_partial, nullptr);
    RB_CUDA(cudaGetLastError());
    rb::reduce_partials_kernel<<<1, RB_RED_NT, 0, c->stream>>>(c->d_partial, nblk, d, c->hp.courant_factor * L.dx / c->hp.smallc, 1, c->d_red + 4, 0);
    RB_CUDA(cudaGetLastError());
  }
  int best_s = -1, best_hz = 0;
  float best_ms = 1e30f;
  for (int s = 0; s < rb::kNumStreamShapes; s++) {
    if (!stream_shape_fits(c, s)) continue;
    const size_t smem = c->precision == RB_PREC_MIXED ? rb::stream_smem_mixed(s) : rb::stream_smem_f64(s);
    if (smem > 227 * 1024) continue;
    for (int hz = 4; hz <= 64; hz *= 2) {
      if (c->dnz % hz != 0) continue;
      const int items = stream_items_of(c, s, hz);
      if (items < 148 && hz != 4) continue;
      RB_TRY(ensure_partial(c, items));
      rb::StreamArgs sa;
      memset(&sa, 0, sizeof sa);
      sa.uin = c->d_dense[c->dense_cur];
      sa.uout = c->d_dense[c->dense_cur ^ 1];
      sa.partial = c->d_partial;
      sa.dt_dev = c->d_red + 4;
      sa.nx = c->dnx; sa.ny = c->dny; sa.nz = c->dnz;
      sa.hz = hz;
      int e2;
      sa.dx_pow2 = std::frexp(L.dx, &e2) == 0.5;
      sa.dx = L.dx;
      sa.inv_dx = 1.0 / L.dx;
      sa.hp = c->hp;
      float ms = 1e30f;
      for (int rep = 0; rep < 4; rep++) {
        RB_CUDA(cudaEventRecord(c->ev0, c->stream));
        cudaError_t e = c->precision == RB_PREC_MIXED ? rb::launch_stream_mixed(s, sa, items, c->stream)
                                                      : rb::launch_stream_f64(s, sa, items, c->stream);
        if (e != cudaSuccess) return fail(RB_ERR_CUDA, "stream kernel launch failed: %s", cudaGetErrorString(e));
        RB_CUDA(cudaEventRecord(c->ev1, c->stream));
        RB_CUDA(cudaEventSynchronize(c->ev1));
        float t = 0.f;
        RB_CUDA(cudaEventElapsedTime(&t, c->ev0, c->ev1));
        if (rep > 0) ms = std::min(ms, t);
      }
      if (ms < best_ms) { best_ms = ms; best_s = s; best_hz = hz; }
    }
  }
  if (best_s < 0) return fail(RB_ERR_STATE, "no z-streaming configuration fits this grid");
  c->stream_shape = best_s;
  c->stream_hz = best_hz;
  c->stream_items = stream_items_of(c, best_s, best_hz);
  drop_graph(c);
  if (shape_out) *shape_out = best_s;
  if (hz_out) *hz_out = best_hz;
  if (ms_out) *ms_out = best_ms;
  return RB_OK;
}

int rb_set_stream_shape(rb_context* c, int shape, int hz) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  const int lf = c->finest;
  if (!c->have_tree || lf < 1 || !c->lv[lf].complete)
    return fail(RB_ERR_STATE, "the z-streaming kernel needs a uniform grid");
  if (c->hp.slope_type == 3) return fail(RB_ERR_STATE, "slope_type 3 runs on the oct tiles only");
  if (shape < 0 || shape >= rb::kNumStreamShapes) return fail(RB_ERR_INVALID, "stream shape %d out of range", shape);
  RB_TRY(dense_prepare(c));
  if (!stream_shape_fits(c, shape)) return fail(RB_ERR_INVALID, "stream shape %d does not tile the grid", shape);
  if (hz < 2 || hz % 2 != 0 || c->dnz % hz != 0)
    return fail(RB_ERR_INVALID, "hz=%d must be even and divide nz=%d", hz, c->dnz);
  c->stream_shape = shape;
  c->stream_hz = hz;
  c->stream_items = stream_items_of(c, shape, hz);
  drop_graph(c);
  return RB_OK;
}

int rb_uniform_run(rb_context* c, int nsteps, int use_graph, double* t_io, double* dt_last_out) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (!c->have_tree || !c->have_state) return fail(RB_ERR_STATE, "tree and state must be uploaded first");
  if (nsteps < 0) return fail(RB_ERR_INVALID, "nsteps must be >= 0");
  if (nsteps > 0) dev_wrote(c);
  const int lf = c->finest;
  Level& L = c->lv[lf];
  // (with physical boundaries the level covers the box, not the extended
  // coarse grid, and the run takes the amr_step sequence below)
  if (lf < 1 || (!L.complete && c->btype.empty()) || L.leaf_cells != (int64_t)L.noct * 8)
    return fail(RB_ERR_STATE, "rb_uniform_run needs a complete, unrefined finest level");
  for (int l = 1; l < lf; l++)
    if (c->lv[l].leaf_cells != 0) return fail(RB_ERR_STATE, "level %d has leaf cells: not a uniform grid", l);
  // with pressure_fix the pdV term and the energy fix come between the update
  // and the next CFL condition, and physical boundaries refill their ghost
  // octs after each step: the amr_step sequence, step by step
  if (c->hp.pressure_fix || !c->btype.empty()) {
    if (t_io) c->t = *t_io;
    for (int s = 0; s < nsteps; s++) RB_TRY(rb_coarse_step(c, nullptr, nullptr));
    if (t_io) *t_io = c->t;
    if (dt_last_out) *dt_last_out = c->dtnew[lf];
    return RB_OK;
  }
  // the multi-dimensional limiter (slope_type 3) reads the 26 neighbours of
  // every cell, and the artificial diffusion (difmag) the cell corners, which
  // the z-streaming kernel does not hold: oct tiles only
  if (c->uniform_method == 0 && c->hp.slope_type != 3 && c->hp.difmag == 0.0)
    return uniform_run_dense(c, nsteps, use_graph, t_io, dt_last_out);
  return uniform_run_tiles(c, nsteps, use_graph, t_io, dt_last_out);
}

int rb_get_uniform_info(rb_context* c, int* method, int* shape, int* hz, int* items) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  const int m =
      (c->uniform_method == 0 && c->hp.slope_type != 3 && c->hp.difmag == 0.0 && c->btype.empty()) ? 0 : 1;
  if (method) *method = m;
  if (shape) *shape = m == 0 ? c->stream_shape : (c->finest ? c->lv[c->finest].shape : -1);
  if (hz) *hz = m == 0 ? c->stream_hz : 0;
  if (items) *items = m == 0 ? c->stream_items : (c->finest ? c->lv[c->finest].ntile : 0);
  return RB_OK;
}

int rb_set_uniform_method(rb_context* c, int method) {
  if (!c) return fail(RB_ERR_INVALID, "null context");
  if (method != 0 && method != 1) return fail(RB_ERR_INVALID, "method must be 0 (z-streaming) or 1 (oct tiles)");
  if (method != c->uniform_method) {
    RB_TRY(sync_oct(c));
    c->dense_valid = false;
    drop_graph(c);
  }
  c->uniform_method = method;
  return RB_OK;
}

}  // extern "C"
