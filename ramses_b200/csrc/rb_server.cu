// rb_server.cu -- serving engine: many independent hydro problems on one GPU.
//
// Problems ("requests") are admitted first-come first-served while their
// device memory fits in the server's HBM budget and stay resident until they
// reach their end time. Two kinds:
//  * dense: one complete level as a periodic Cartesian grid (the layout of the
//    z-streaming kernel). All active dense problems advance together: every
//    step is ONE launch of stream_batch_kernel over the work items of all of
//    them, then one batch_clock_kernel launch that advances each problem's own
//    clock. Problems never share a reduction or an atomic, so a problem's
//    result does not depend on which others share its launches.
//  * octree: an AMR problem with its own rb_context, stepped by device-
//    scheduled coarse steps (CUDA graphs of 8 steps) on its own stream, so
//    several run concurrently with the dense batch.
// The host drives the engine by calling rb_server_progress in a loop; each
// call enqueues one round (steps_per_round batched steps and one graph chunk
// per octree problem) before it waits for the previous round, so the GPU
// always has queued work while the host harvests results and admits requests.
// Compiled with --fmad=false.
#include <chrono>
#include <deque>

#include "rb_context.h"
#include "serve_kernels.cuh"

using namespace rbi;

namespace {

enum ReqState { RQ_QUEUED = 0, RQ_ACTIVE = 1, RQ_DONE = 2, RQ_FAILED = 3, RQ_CANCELLED = 4 };

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
  int64_t id = 0;
  int kind = 0;  // 0 dense, 1 octree
  int state = RQ_QUEUED;
  bool cancel = false;
  double t_end = 0.0;
  int64_t max_steps = 0;
  const double* h_in = nullptr;
  double* h_out = nullptr;
  int64_t bytes = 0;  // device bytes charged against the budget
  // dense
  int32_t nx = 0, ny = 0, nz = 0;
  int hz = 0, items = 0;
  int outflow = 0;  // bit d: outflow boundaries along axis d
  double dx = 0.0;
  double* d_buf = nullptr;  // [2][5][n]
  int slot = -1;            // clock slot
  // octree
  rb_mesh_params mp{};
  const int32_t *son = nullptr, *father = nullptr, *nbor = nullptr, *numbl = nullptr, *active = nullptr;
  int32_t nboundary = 0;  // physical boundaries of an octree problem (rb_set_boundary's lists)
  const int32_t *btype = nullptr, *numbb = nullptr, *bgrid = nullptr;
  rb_context* ctx = nullptr;
  cudaEvent_t ev = nullptr;
  bool chunk_in_flight = false;
  // results
  double t = 0.0;
  int64_t steps = 0, cell_updates = 0;
  double t_submit = 0.0, t_admit = 0.0, t_done = 0.0;
  int error = RB_OK;
};

constexpr int kMaxSlots = 1 << 16;  // dense problems resident at once

}  // namespace

struct rb_server {
  rb_hydro_params hp;
  int precision = RB_PREC_FP64;
  int device = 0;
  int64_t budget = 0, in_use = 0;
  int steps_per_round = 8;
  int shape = 1;  // column shape of the batched kernel (16x8; 6: stream2_batch_kernel)
  cudaStream_t stream = nullptr;  // dense batch stream
  cudaStream_t copy = nullptr;    // result downloads
  int64_t next_id = 1;
  std::deque<Request*> queue;
  std::vector<Request*> dense, tree;  // active
  std::unordered_map<int64_t, Request*> all;
  // device clocks of the dense problems: [kMaxSlots][8], read back whole
  double* d_clocks = nullptr;
  double* h_clocks[2] = {nullptr, nullptr};
  unsigned long long* d_smax = nullptr;  // [kMaxSlots] scratch of the first dt
  std::vector<int> free_slots;
  // round buffers
  rb::BatchDesc* d_desc = nullptr;
  int32_t* d_off = nullptr;
  double* d_partial = nullptr;
  int desc_cap = 0, item_cap = 0;
  rb::BatchDesc* h_desc[2] = {nullptr, nullptr};
  int32_t* h_off[2] = {nullptr, nullptr};
  int hcap[2] = {0, 0};
  cudaEvent_t round_ev[2] = {nullptr, nullptr};
  bool round_live[2] = {false, false};
  std::vector<Request*> round_members[2];
  int64_t round = 0;
  std::deque<int64_t> done_pending;  // completed ids not yet returned
  int64_t total_updates = 0;
  int64_t rounds_launched = 0, batch_launches = 0;
};

namespace {

int64_t dense_bytes(int64_t n) { return 2 * 5 * n * (int64_t)sizeof(double); }

// device memory of an octree problem: uold, unew and the staging copy
// (5 variables each), son, the per-oct tables and the CFL partials
int64_t tree_bytes(const rb_mesh_params& mp) {
  const int64_t ncell = (int64_t)mp.ncoarse + 8 * (int64_t)mp.ngridmax;
  return ncell * (3 * 5 * 8 + 4) + (int64_t)mp.ngridmax * 96 + (4 << 20);
}

// the longest z extent (power of two <= 64 dividing nz) that still gives the
// problem at least 16 work items
int pick_hz(int nx, int ny, int nz, int tx, int ty) {
  const int cols = (nx / tx) * (ny / ty);
  int hz = 64;
  while (hz > 8 && (nz % hz != 0 || cols * (nz / hz) < 16)) hz >>= 1;
  while (hz > 2 && nz % hz != 0) hz >>= 1;
  return hz;
}

int grow_round_buffers(rb_server* s, int nprob, int nitems) {
  if (nprob + 1 > s->desc_cap) {
    int cap = std::max(nprob + 1, 2 * s->desc_cap);
    if (s->d_desc) cudaFreeAsync(s->d_desc, s->stream);
    if (s->d_off) cudaFreeAsync(s->d_off, s->stream);
    RB_CUDA(cudaMallocAsync((void**)&s->d_desc, cap * sizeof(rb::BatchDesc), s->stream));
    RB_CUDA(cudaMallocAsync((void**)&s->d_off, (cap + 1) * sizeof(int32_t), s->stream));
    s->desc_cap = cap;
  }
  if (nitems > s->item_cap) {
    int cap = std::max(nitems, 2 * s->item_cap);
    if (s->d_partial) cudaFreeAsync(s->d_partial, s->stream);
    RB_CUDA(cudaMallocAsync((void**)&s->d_partial, (size_t)cap * 4 * sizeof(double), s->stream));
    s->item_cap = cap;
  }
  const int k = s->round & 1;
  if (nprob + 1 > s->hcap[k]) {
    // this pinned buffer was last used by round-2, which has completed
    if (s->h_desc[k]) cudaFreeHost(s->h_desc[k]);
    if (s->h_off[k]) cudaFreeHost(s->h_off[k]);
    s->h_desc[k] = nullptr;
    s->h_off[k] = nullptr;
    int cap = std::max(nprob + 1, 2 * s->hcap[k]);
    if (cudaMallocHost((void**)&s->h_desc[k], cap * sizeof(rb::BatchDesc)) != cudaSuccess ||
        cudaMallocHost((void**)&s->h_off[k], (cap + 1) * sizeof(int32_t)) != cudaSuccess) {
      s->hcap[k] = 0;
      return fail(RB_ERR_NOMEM, "pinned allocation of round descriptors failed");
    }
    s->hcap[k] = cap;
  }
  return RB_OK;
}

void release_dense(rb_server* s, Request* r) {
  if (r->d_buf) cudaFreeAsync(r->d_buf, s->stream);  // after every launch already enqueued
  r->d_buf = nullptr;
  if (r->slot >= 0) s->free_slots.push_back(r->slot);
  r->slot = -1;
  s->in_use -= r->bytes;
}

void release_tree(rb_server* s, Request* r) {
  if (r->ev) cudaEventDestroy(r->ev);
  r->ev = nullptr;
  if (r->ctx) rb_destroy(r->ctx);
  r->ctx = nullptr;
  s->in_use -= r->bytes;
}

void finish(Request* r, int state, int err) {
  r->state = state;
  r->error = err;
  r->t_done = now_s();
}

// Admit one queued request: allocate, upload, first time step.
int admit_dense(rb_server* s, Request* r) {
  const int64_t n = (int64_t)r->nx * r->ny * r->nz;
  if (s->free_slots.empty()) return fail(RB_ERR_CAPACITY, "all %d dense slots in use", kMaxSlots);
  cudaError_t e = cudaMallocAsync((void**)&r->d_buf, (size_t)dense_bytes(n), s->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    r->d_buf = nullptr;
    return fail(RB_ERR_NOMEM, "device allocation of %lld bytes failed", (long long)dense_bytes(n));
  }
  r->slot = s->free_slots.back();
  s->free_slots.pop_back();
  s->in_use += r->bytes;
  RB_CUDA(cudaMemcpyAsync(r->d_buf, r->h_in, (size_t)n * 5 * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  RB_CUDA(cudaMemsetAsync(s->d_smax + r->slot, 0, sizeof(unsigned long long), s->stream));
  rb::dense_cfl_kernel<<<grid_for(n, 256, 148 * 4), 256, 0, s->stream>>>(r->d_buf, n, s->hp, s->d_smax + r->slot);
  RB_CUDA(cudaGetLastError());
  const double boxlen = r->dx * r->nx;
  rb::dense_clock_init_kernel<<<1, 1, 0, s->stream>>>(
      s->d_clocks + (int64_t)r->slot * 8, s->d_smax + r->slot, 0.0, r->t_end, (double)r->max_steps,
      boxlen / s->hp.smallc, s->hp.courant_factor * r->dx / s->hp.smallc, r->dx, s->hp.courant_factor);
  RB_CUDA(cudaGetLastError());
  // the caller keeps h_in valid until the request completes, so the copy
  // needs no wait here
  r->state = RQ_ACTIVE;
  r->t_admit = now_s();
  s->dense.push_back(r);
  return RB_OK;
}

int admit_tree(rb_server* s, Request* r) {
  rb_context* c = nullptr;
  RB_TRY(rb_create(&s->hp, &r->mp, s->precision, &c));
  r->ctx = c;
  s->in_use += r->bytes;
  int rc;
  if ((r->nboundary && (rc = rb_set_boundary(c, r->nboundary, r->btype, r->numbb, r->bgrid))) ||
      (rc = rb_sync_tree(c, r->son, r->father, r->nbor, r->numbl, r->active)) ||
      (rc = rb_upload_state(c, r->h_in)) || (r->nboundary && (rc = make_boundary_all(c))) ||
      (rc = run_async_begin(c, r->t_end, r->max_steps))) {
    release_tree(s, r);
    return rc;
  }
  RB_CUDA(cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming));
  r->state = RQ_ACTIVE;
  r->t_admit = now_s();
  s->tree.push_back(r);
  return RB_OK;
}

// FIFO admission while the head of the queue fits in the budget. A request
// that fails for lack of memory stays queued; other failures end it.
void admit(rb_server* s) {
  while (!s->queue.empty()) {
    Request* r = s->queue.front();
    if (r->cancel) {
      s->queue.pop_front();
      finish(r, RQ_CANCELLED, RB_OK);
      continue;
    }
    if (s->in_use + r->bytes > s->budget) break;
    const int rc = r->kind == 0 ? admit_dense(s, r) : admit_tree(s, r);
    if (rc == RB_ERR_NOMEM || rc == RB_ERR_CAPACITY) break;
    s->queue.pop_front();
    if (rc) finish(r, RQ_FAILED, rc);
  }
}

// Enqueue one round: steps_per_round batched steps of the dense problems and
// one graph chunk for every octree problem without one in flight.
int launch_round(rb_server* s) {
  const int k = s->round & 1;
  s->round_members[k].clear();
  int nitems = 0;
  for (Request* r : s->dense) nitems += r->items;
  const int nprob = (int)s->dense.size();
  if (nprob) {
    RB_TRY(grow_round_buffers(s, nprob, nitems));
    rb::BatchDesc* hd = s->h_desc[k];
    int32_t* ho = s->h_off[k];
    int off = 0;
    for (int p = 0; p < nprob; p++) {
      Request* r = s->dense[p];
      rb::BatchDesc& d = hd[p];
      memset(&d, 0, sizeof d);
      d.a.partial = s->d_partial + (int64_t)off * 4;
      d.a.nx = r->nx; d.a.ny = r->ny; d.a.nz = r->nz;
      d.a.hz = r->hz;
      d.a.outflow = r->outflow;
      int e2;
      d.a.dx_pow2 = std::frexp(r->dx, &e2) == 0.5;
      d.a.dx = r->dx;
      d.a.inv_dx = 1.0 / r->dx;
      d.a.hp = s->hp;
      const int64_t n = (int64_t)r->nx * r->ny * r->nz;
      d.dense[0] = r->d_buf;
      d.dense[1] = r->d_buf + 5 * n;
      d.clock = s->d_clocks + (int64_t)r->slot * 8;
      d.t_end = r->t_end;
      d.max_steps = (double)r->max_steps;
      d.dt_max = r->dx * r->nx / s->hp.smallc;
      d.dt0 = s->hp.courant_factor * r->dx / s->hp.smallc;
      d.parity0 = 0;
      d.nitems = r->items;
      ho[p] = off;
      off += r->items;
      s->round_members[k].push_back(r);
    }
    ho[nprob] = off;
    RB_CUDA(cudaMemcpyAsync(s->d_desc, hd, nprob * sizeof(rb::BatchDesc), cudaMemcpyHostToDevice, s->stream));
    RB_CUDA(cudaMemcpyAsync(s->d_off, ho, (nprob + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s->stream));
    for (int st = 0; st < s->steps_per_round; st++) {
      cudaError_t e = s->precision == RB_PREC_MIXED
                          ? rb::launch_batch_mixed(s->shape, s->hp, s->d_desc, s->d_off, nprob, nitems, s->stream)
                          : rb::launch_batch_f64(s->shape, s->hp, s->d_desc, s->d_off, nprob, nitems, s->stream);
      if (e != cudaSuccess) return fail(RB_ERR_CUDA, "batched step launch failed: %s", cudaGetErrorString(e));
      rb::batch_clock_kernel<<<nprob, RB_RED_NT, 0, s->stream>>>(s->d_desc, s->d_off);
      RB_CUDA(cudaGetLastError());
      s->batch_launches++;
    }
    int maxslot = 0;
    for (Request* r : s->dense) maxslot = std::max(maxslot, r->slot + 1);
    RB_CUDA(cudaMemcpyAsync(s->h_clocks[k], s->d_clocks, (size_t)maxslot * 8 * sizeof(double),
                            cudaMemcpyDeviceToHost, s->stream));
  }
  RB_CUDA(cudaEventRecord(s->round_ev[k], s->stream));
  s->round_live[k] = true;
  for (Request* r : s->tree) {
    if (r->chunk_in_flight || r->cancel) continue;
    rb_context* c = r->ctx;
    RB_TRY(run_async_chunk(c, 8, true));
    RB_CUDA(cudaMemcpyAsync(c->h_sched, c->d_sched, RB_S_SIZE * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    RB_CUDA(cudaEventRecord(r->ev, c->stream));
    r->chunk_in_flight = true;
  }
  s->round++;
  s->rounds_launched++;
  return RB_OK;
}

// Wait for round k and retire the dense problems that finished in it.
int harvest_dense(rb_server* s, int k, std::vector<int64_t>& done) {
  if (!s->round_live[k]) return RB_OK;
  RB_CUDA(cudaEventSynchronize(s->round_ev[k]));
  s->round_live[k] = false;
  const double* hc = s->h_clocks[k];
  std::vector<Request*> keep;
  keep.reserve(s->dense.size());
  std::vector<Request*> finished;
  for (Request* r : s->round_members[k]) {
    if (r->state != RQ_ACTIVE) continue;  // retired after an earlier round
    const double* ck = hc + (int64_t)r->slot * 8;
    if (ck[6] != 0.0 || r->cancel) finished.push_back(r);
  }
  for (Request* r : finished) {
    const double* ck = hc + (int64_t)r->slot * 8;
    const int64_t n = (int64_t)r->nx * r->ny * r->nz;
    r->t = ck[1];
    r->steps = (int64_t)ck[5];
    r->cell_updates = r->steps * n;
    if (!r->cancel) {
      // the problem's kernels in the round launched since are no-ops, so its
      // final buffer is stable while that round runs
      const double* src = r->d_buf + ((r->steps & 1) ? 5 * n : 0);
      RB_CUDA(cudaMemcpyAsync(r->h_out, src, (size_t)n * 5 * sizeof(double), cudaMemcpyDeviceToHost, s->copy));
      RB_CUDA(cudaStreamSynchronize(s->copy));
      s->total_updates += r->cell_updates;
    }
    release_dense(s, r);
    finish(r, r->cancel ? RQ_CANCELLED : RQ_DONE, RB_OK);
    done.push_back(r->id);
  }
  for (Request* r : s->dense)
    if (r->state == RQ_ACTIVE) keep.push_back(r);
  s->dense.swap(keep);
  return RB_OK;
}

// Retire octree problems whose last chunk has completed and met the stop rule.
int harvest_tree(rb_server* s, bool block, std::vector<int64_t>& done) {
  std::vector<Request*> keep;
  for (Request* r : s->tree) {
    if (r->chunk_in_flight) {
      cudaError_t q = block ? cudaEventSynchronize(r->ev) : cudaEventQuery(r->ev);
      if (q == cudaErrorNotReady) {
        keep.push_back(r);
        continue;
      }
      if (q != cudaSuccess) return fail(RB_ERR_CUDA, "octree request %lld: %s", (long long)r->id, cudaGetErrorString(q));
      r->chunk_in_flight = false;
    }
    const double* h = r->ctx->h_sched;
    const bool over = !(h[RB_S_T] < h[RB_S_TEND]) || !(h[RB_S_COARSE] < h[RB_S_MAXC]);
    if (!over && !r->cancel) {
      keep.push_back(r);
      continue;
    }
    int64_t coarse = 0;
    int rc = run_async_end(r->ctx, &coarse);
    if (!rc && !r->cancel) rc = rb_download_state(r->ctx, r->h_out);
    r->t = r->ctx->t;
    r->steps = coarse;
    r->cell_updates = r->ctx->cell_updates;
    if (!rc && !r->cancel) s->total_updates += r->cell_updates;
    release_tree(s, r);
    finish(r, rc ? RQ_FAILED : (r->cancel ? RQ_CANCELLED : RQ_DONE), rc);
    done.push_back(r->id);
  }
  s->tree.swap(keep);
  return RB_OK;
}

Request* find(rb_server* s, int64_t id) {
  auto it = s->all.find(id);
  return it == s->all.end() ? nullptr : it->second;
}

}  // namespace

extern "C" {

int rb_server_destroy(rb_server* s);

int rb_server_create(const rb_hydro_params* hp, int precision, int64_t hbm_budget_bytes, int steps_per_round,
                     rb_server** out) {
  if (!out) return fail(RB_ERR_INVALID, "null output pointer");
  *out = nullptr;
  if (!hp) return fail(RB_ERR_INVALID, "null hydro parameters");
  rb_mesh_params mp{};
  mp.nx = mp.ny = mp.nz = 1;
  mp.ncoarse = 1;
  mp.ngridmax = 1;
  mp.nlevelmax = 1;
  mp.levelmin = 1;
  mp.nvector = 1;
  mp.boxlen = 1.0;
  RB_TRY(check_params(hp, &mp));  // the parameter rules of rb_create
  if (hp->slope_type == 3)
    return fail(RB_ERR_INVALID, "slope_type 3 (multi-dimensional limiter) is not served: dense problems run the "
                                "z-streaming kernel, which holds axis neighbours only");
  if (hp->pressure_fix)
    return fail(RB_ERR_INVALID, "pressure_fix is not served: the batched z-streaming step keeps no enew/divu");
  if (hp->difmag > 0.0)
    return fail(RB_ERR_INVALID, "difmag > 0 is not served: the batched z-streaming step has no corner divergence");
  if (precision != RB_PREC_FP64 && precision != RB_PREC_MIXED)
    return fail(RB_ERR_INVALID, "precision must be RB_PREC_FP64 or RB_PREC_MIXED");
  if (rb_device_count() == 0) return fail(RB_ERR_NO_DEVICE, "no CUDA device visible");
  if (steps_per_round < 1 || steps_per_round > 1024)
    return fail(RB_ERR_INVALID, "steps_per_round=%d must be in 1..1024", steps_per_round);
  rb_server* s = new rb_server();
  s->hp = *hp;
  s->precision = precision;
  s->steps_per_round = steps_per_round;
  // FP32-mixed schemes that stream2_supports batch with stream2_batch_kernel
  // (the kernel rb_uniform_run picks by default for them)
  if (precision == RB_PREC_MIXED && rb::stream2_supports(*hp)) s->shape = 6;
  auto bail = [&](int rc) {
    rb_server_destroy(s);
    return rc;
  };
  if (cudaGetDevice(&s->device) != cudaSuccess) return bail(fail(RB_ERR_NO_DEVICE, "cudaGetDevice failed"));
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return bail(fail(RB_ERR_CUDA, "cudaMemGetInfo failed"));
  s->budget = hbm_budget_bytes > 0 ? std::min<int64_t>(hbm_budget_bytes, (int64_t)free_b)
                                   : (int64_t)(0.85 * (double)free_b);
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->round_ev[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->round_ev[1], cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(RB_ERR_CUDA, "stream/event creation failed"));
  int rc;
  if ((rc = dalloc(&s->d_clocks, (size_t)kMaxSlots * 8)) || (rc = dalloc(&s->d_smax, (size_t)kMaxSlots)))
    return bail(rc);
  if (cudaMallocHost((void**)&s->h_clocks[0], (size_t)kMaxSlots * 8 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost((void**)&s->h_clocks[1], (size_t)kMaxSlots * 8 * sizeof(double)) != cudaSuccess)
    return bail(fail(RB_ERR_NOMEM, "pinned allocation failed"));
  if (cudaMemsetAsync(s->d_clocks, 0, (size_t)kMaxSlots * 8 * sizeof(double), s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess)
    return bail(fail(RB_ERR_CUDA, "initialising the clock pool failed"));
  s->free_slots.reserve(kMaxSlots);
  for (int i = kMaxSlots - 1; i >= 0; i--) s->free_slots.push_back(i);
  // attribute setup of the batched kernel (shared memory size) before any capture
  cudaError_t e = precision == RB_PREC_MIXED
                      ? rb::launch_batch_mixed(s->shape, s->hp, nullptr, nullptr, 0, 0, s->stream)
                      : rb::launch_batch_f64(s->shape, s->hp, nullptr, nullptr, 0, 0, s->stream);
  if (e != cudaSuccess) return bail(fail(RB_ERR_CUDA, "batched kernel setup failed: %s", cudaGetErrorString(e)));
  *out = s;
  return RB_OK;
}

int rb_server_destroy(rb_server* s) {
  if (!s) return RB_OK;
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (Request* r : s->tree) {
    if (r->ctx) cudaStreamSynchronize(r->ctx->stream);
    release_tree(s, r);
  }
  for (Request* r : s->dense) release_dense(s, r);
  if (s->d_desc) cudaFreeAsync(s->d_desc, s->stream);
  if (s->d_off) cudaFreeAsync(s->d_off, s->stream);
  if (s->d_partial) cudaFreeAsync(s->d_partial, s->stream);
  if (s->stream) cudaStreamSynchronize(s->stream);
  dfree(s->d_clocks);
  dfree(s->d_smax);
  for (int k = 0; k < 2; k++) {
    if (s->h_clocks[k]) cudaFreeHost(s->h_clocks[k]);
    if (s->h_desc[k]) cudaFreeHost(s->h_desc[k]);
    if (s->h_off[k]) cudaFreeHost(s->h_off[k]);
    if (s->round_ev[k]) cudaEventDestroy(s->round_ev[k]);
  }
  if (s->copy) cudaStreamDestroy(s->copy);
  if (s->stream) cudaStreamDestroy(s->stream);
  for (auto& kv : s->all) delete kv.second;
  delete s;
  return RB_OK;
}

static int check_stop(double t_end, int64_t max_steps) {
  if (std::isnan(t_end)) return fail(RB_ERR_INVALID, "t_end is NaN");
  if (max_steps < 0) return fail(RB_ERR_INVALID, "max_steps must be non-negative");
  return RB_OK;
}

int rb_server_submit_dense(rb_server* s, int32_t nx, int32_t ny, int32_t nz, double boxlen, int32_t outflow_mask,
                           const double* u, double t_end, int64_t max_steps, double* result, int64_t* id_out) {
  if (!s || !u || !result || !id_out) return fail(RB_ERR_INVALID, "null argument");
  RB_TRY(check_stop(t_end, max_steps));
  if (outflow_mask < 0 || outflow_mask > 7) return fail(RB_ERR_INVALID, "outflow_mask %d: bits 0-2 only", outflow_mask);
  const int tx = rb::kStreamShapes[s->shape][0], ty = rb::kStreamShapes[s->shape][1];
  if (nx < tx || ny < ty || nz < 2 || nx % tx || ny % ty || nz % 2)
    return fail(RB_ERR_INVALID, "dense grid %dx%dx%d: nx must be a multiple of %d, ny of %d, nz even", nx, ny, nz,
                tx, ty);
  if (!(boxlen > 0.0)) return fail(RB_ERR_INVALID, "boxlen must be positive");
  Request* r = new Request();
  r->id = s->next_id++;
  r->kind = 0;
  r->t_end = t_end;
  r->max_steps = max_steps;
  r->h_in = u;
  r->h_out = result;
  r->nx = nx; r->ny = ny; r->nz = nz;
  r->outflow = outflow_mask;
  r->dx = boxlen / nx;
  if (std::fabs(r->dx * ny - boxlen) > 1e-12 * boxlen || std::fabs(r->dx * nz - boxlen) > 1e-12 * boxlen) {
    delete r;
    return fail(RB_ERR_INVALID, "dense problems are cubes of cubic cells (nx=ny=nz)");
  }
  r->hz = pick_hz(nx, ny, nz, tx, ty);
  r->items = (nx / tx) * (ny / ty) * (nz / r->hz);
  r->bytes = dense_bytes((int64_t)nx * ny * nz);
  if (r->bytes > s->budget) {
    delete r;
    return fail(RB_ERR_CAPACITY, "request needs %lld bytes, the budget is %lld", (long long)dense_bytes((int64_t)nx * ny * nz),
                (long long)s->budget);
  }
  r->t_submit = now_s();
  s->all[r->id] = r;
  s->queue.push_back(r);
  *id_out = r->id;
  return RB_OK;
}

int rb_server_submit_octree(rb_server* s, const rb_mesh_params* mp, const int32_t* son, const int32_t* father,
                            const int32_t* nbor, const int32_t* numbl, const int32_t* active, const double* uold,
                            double t_end, int64_t max_steps, double* result, int64_t* id_out) {
  if (!s || !mp || !son || !father || !nbor || !numbl || !active || !uold || !result || !id_out)
    return fail(RB_ERR_INVALID, "null argument");
  RB_TRY(check_stop(t_end, max_steps));
  RB_TRY(check_params(&s->hp, mp));
  if (max_steps > INT32_MAX) max_steps = INT32_MAX;
  Request* r = new Request();
  r->id = s->next_id++;
  r->kind = 1;
  r->t_end = t_end;
  r->max_steps = max_steps;
  r->h_in = uold;
  r->h_out = result;
  r->mp = *mp;
  r->son = son; r->father = father; r->nbor = nbor; r->numbl = numbl; r->active = active;
  r->bytes = tree_bytes(*mp);
  if (r->bytes > s->budget) {
    delete r;
    return fail(RB_ERR_CAPACITY, "request needs about %lld bytes, the budget is %lld", (long long)tree_bytes(*mp),
                (long long)s->budget);
  }
  r->t_submit = now_s();
  s->all[r->id] = r;
  s->queue.push_back(r);
  *id_out = r->id;
  return RB_OK;
}

int rb_server_submit_octree_bounded(rb_server* s, const rb_mesh_params* mp, const int32_t* son,
                                    const int32_t* father, const int32_t* nbor, const int32_t* numbl,
                                    const int32_t* active, int32_t nboundary, const int32_t* boundary_type,
                                    const int32_t* numbb, const int32_t* boundary_igrid, const double* uold,
                                    double t_end, int64_t max_steps, double* result, int64_t* id_out) {
  if (nboundary < 0 || nboundary > 6 || (nboundary > 0 && (!boundary_type || !numbb || !boundary_igrid)))
    return fail(RB_ERR_INVALID, "bad boundary lists");
  // the boundary-fill tables the admission also allocates: one
  // (boundary oct, reference oct) pair (8 B) and one staged oct state
  // (8 cells x 5 variables, 320 B) per boundary oct
  int64_t nbocts = 0;
  for (int l = 1; l <= mp->nlevelmax; l++)
    for (int ib = 0; ib < nboundary; ib++) {
      const int32_t n = numbb[ib + (int64_t)nboundary * (l - 1)];
      if (n < 0 || n > mp->ngridmax) return fail(RB_ERR_INVALID, "numbb(%d,%d)=%d out of range", ib + 1, l, n);
      nbocts += n;
    }
  const int64_t bbytes = nbocts * (8 + 320);
  if (tree_bytes(*mp) + bbytes > s->budget)
    return fail(RB_ERR_CAPACITY, "request needs about %lld bytes, the budget is %lld",
                (long long)(tree_bytes(*mp) + bbytes), (long long)s->budget);
  RB_TRY(rb_server_submit_octree(s, mp, son, father, nbor, numbl, active, uold, t_end, max_steps, result, id_out));
  Request* r = s->all[*id_out];
  r->bytes += bbytes;
  r->nboundary = nboundary;
  r->btype = boundary_type; r->numbb = numbb; r->bgrid = boundary_igrid;
  return RB_OK;
}

int rb_server_progress(rb_server* s, int64_t* done_ids, int max_ids, int* ndone) {
  if (!s || !ndone || (max_ids > 0 && !done_ids)) return fail(RB_ERR_INVALID, "null argument");
  *ndone = 0;
  std::vector<int64_t> done;
  admit(s);
  const int prev = (s->round + 1) & 1;  // round launched by the previous call
  RB_TRY(launch_round(s));
  RB_TRY(harvest_dense(s, prev, done));
  RB_TRY(harvest_tree(s, false, done));
  admit(s);
  for (int64_t id : done) s->done_pending.push_back(id);
  int n = 0;
  while (n < max_ids && !s->done_pending.empty()) {
    done_ids[n++] = s->done_pending.front();
    s->done_pending.pop_front();
  }
  *ndone = n;
  return RB_OK;
}

int rb_server_request_info(rb_server* s, int64_t id, int* state, double* t, int64_t* steps, int64_t* cell_updates,
                           double* seconds_in_system) {
  if (!s) return fail(RB_ERR_INVALID, "null server");
  Request* r = find(s, id);
  if (!r) return fail(RB_ERR_INVALID, "unknown request id %lld", (long long)id);
  if (state) *state = r->state;
  if (t) *t = r->t;
  if (steps) *steps = r->steps;
  if (cell_updates) *cell_updates = r->cell_updates;
  if (seconds_in_system) *seconds_in_system = (r->t_done > 0.0 ? r->t_done : now_s()) - r->t_submit;
  return r->error;
}

int rb_server_cancel(rb_server* s, int64_t id) {
  if (!s) return fail(RB_ERR_INVALID, "null server");
  Request* r = find(s, id);
  if (!r) return fail(RB_ERR_INVALID, "unknown request id %lld", (long long)id);
  if (r->state == RQ_QUEUED || r->state == RQ_ACTIVE) r->cancel = true;
  return RB_OK;
}

int rb_server_stats(rb_server* s, int* queued, int* active, int64_t* bytes_in_use, int64_t* budget,
                    int64_t* cell_updates, int64_t* batch_launches) {
  if (!s) return fail(RB_ERR_INVALID, "null server");
  if (queued) *queued = (int)s->queue.size();
  if (active) *active = (int)(s->dense.size() + s->tree.size());
  if (bytes_in_use) *bytes_in_use = s->in_use;
  if (budget) *budget = s->budget;
  if (cell_updates) *cell_updates = s->total_updates;
  if (batch_launches) *batch_launches = s->batch_launches;
  return RB_OK;
}

}  // extern "C"
