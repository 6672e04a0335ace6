"""Ensemble serving of independent hydro problems on one GPU.

``Server`` wraps the library's serving engine (``rb_server_*``): problems are
admitted first-come first-served while their device memory fits in an HBM
budget, uniform (dense) problems advance together in packed launches of the
z-streaming kernel, AMR problems run device-scheduled coarse steps on their
own streams, and each finished problem is copied back into its result array.

The rest of the module is the harness of the serving workload: a seeded mix
of planar shock tubes along x and Sedov blasts on 32^3, 64^3 and 128^3 base
grids with 0..2 extra levels, each run to t = 0.1, arriving as a Poisson
process. It reports p50/p99 time-to-solution (arrival -> result in host
memory) and aggregate leaf-cell updates per second, beside the same stream
served one request at a time by the plain FP64 path (``Solver.run``).

Boundaries: uniform tubes have outflow (zero-gradient) boundaries in x and
are periodic in y and z; Sedov blasts are periodic. AMR requests run on the
octree, which is periodic, so an AMR tube sits in a periodic box with its
wrapped second interface half a box away.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import ics, mesh
from .params import HydroParams
from .runtime import (_P32, _P64, _PD, RB_PREC_FP64, RB_PREC_MIXED, RBError, Solver, _check, _ptr, hydro_params_c,
                      load, mesh_params_c)

REQ_QUEUED, REQ_ACTIVE, REQ_DONE, REQ_FAILED, REQ_CANCELLED = 0, 1, 2, 3, 4


# ---------------------------------------------------------------------------
# layouts
# ---------------------------------------------------------------------------
def dense_from_octree(tree: mesh.Octree, level: int, uold: np.ndarray) -> np.ndarray:
    """[5, z, y, x] array of a complete level's cells from uold (5, ncell)."""
    idx = tree.cell_index(level)
    return np.ascontiguousarray(uold[:, idx - 1])


def octree_from_dense(tree: mesh.Octree, level: int, dense: np.ndarray, uold: Optional[np.ndarray] = None
                      ) -> np.ndarray:
    """uold (5, ncell) whose complete level ``level`` holds ``dense`` and whose
    coarser levels hold its restriction (mean of the 8 children)."""
    if uold is None:
        uold = np.zeros((5, tree.ncell))
    cur = dense
    for l in range(level, 0, -1):
        if l < level:
            cur = 0.125 * (cur[:, 0::2, 0::2, 0::2] + cur[:, 1::2, 0::2, 0::2] + cur[:, 0::2, 1::2, 0::2]
                           + cur[:, 1::2, 1::2, 0::2] + cur[:, 0::2, 0::2, 1::2] + cur[:, 1::2, 0::2, 1::2]
                           + cur[:, 0::2, 1::2, 1::2] + cur[:, 1::2, 1::2, 1::2])
        uold[:, tree.cell_index(l) - 1] = cur
    return uold


# ---------------------------------------------------------------------------
# the engine
# ---------------------------------------------------------------------------
class Server:
    """One serving engine (``rb_server``) on the current CUDA device."""

    def __init__(self, hp: HydroParams, precision: str = "mixed", hbm_budget_bytes: int = 0,
                 steps_per_round: int = 8):
        L = load()
        self.hp = hp
        self._hpc = hydro_params_c(hp)
        prec = {"fp64": RB_PREC_FP64, "mixed": RB_PREC_MIXED}[precision]
        h = ctypes.c_void_p()
        _check(L.rb_server_create(ctypes.byref(self._hpc), prec, int(hbm_budget_bytes), int(steps_per_round),
                                  ctypes.byref(h)), "rb_server_create")
        self._h = h
        self._keep = {}  # id -> arrays that must outlive the request
        self.results = {}

    def close(self):
        if getattr(self, "_h", None):
            load().rb_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit_dense(self, u: np.ndarray, boxlen: float = 1.0, t_end: float = math.inf,
                     max_steps: int = 1 << 40, outflow_mask: int = 0) -> int:
        """Queue a uniform problem given as conservative [5, n, n, n];
        outflow_mask bit d: outflow boundaries along axis d, else periodic."""
        u = np.ascontiguousarray(u, np.float64)
        assert u.ndim == 4 and u.shape[0] == 5
        nz, ny, nx = u.shape[1:]
        out = np.empty_like(u)
        rid = ctypes.c_int64()
        _check(load().rb_server_submit_dense(self._h, nx, ny, nz, boxlen, int(outflow_mask), _ptr(u, _PD), float(t_end),
                                             int(max_steps), _ptr(out, _PD), ctypes.byref(rid)),
               "rb_server_submit_dense")
        self._keep[rid.value] = (u, out)
        self.results[rid.value] = out
        return rid.value

    def submit_octree(self, tree: mesh.Octree, uold: np.ndarray, t_end: float = math.inf,
                      max_steps: int = 1 << 30, nsubcycle: Optional[Sequence[int]] = None) -> int:
        """Queue an AMR problem (octree + uold (5, ncell))."""
        mp = mesh_params_c(tree, nsubcycle)
        son = np.ascontiguousarray(tree.son, np.int32)
        father = np.ascontiguousarray(tree.father, np.int32)
        nbor = np.ascontiguousarray(tree.nbor, np.int32)
        numbl = np.array([tree.noct(l) for l in range(1, tree.nlevelmax + 1)], np.int32)
        act, _ = tree.active_concat()
        act = np.ascontiguousarray(act, np.int32)
        u = np.ascontiguousarray(uold, np.float64)
        out = np.empty_like(u)
        rid = ctypes.c_int64()
        bt, boff, bg = tree.boundary_concat()
        numbb = np.diff(boff).astype(np.int32)
        _check(load().rb_server_submit_octree_bounded(
            self._h, ctypes.byref(mp), _ptr(son, _P32), _ptr(father, _P32), _ptr(nbor, _P32), _ptr(numbl, _P32),
            _ptr(act, _P32), len(bt), _ptr(bt, _P32), _ptr(numbb, _P32), _ptr(bg, _P32), _ptr(u, _PD),
            float(t_end), int(max_steps), _ptr(out, _PD), ctypes.byref(rid)), "rb_server_submit_octree_bounded")
        self._keep[rid.value] = (mp, son, father, nbor, numbl, act, bt, numbb, bg, u, out)
        self.results[rid.value] = out
        return rid.value

    def progress(self, max_ids: int = 4096) -> List[int]:
        """One round: admit, enqueue steps, retire; returns completed ids."""
        ids = (ctypes.c_int64 * max_ids)()
        n = ctypes.c_int32()
        _check(load().rb_server_progress(self._h, ids, max_ids, ctypes.byref(n)), "rb_server_progress")
        done = [ids[i] for i in range(n.value)]
        for i in done:
            self._keep.pop(i, None)
        return done

    def info(self, rid: int) -> dict:
        st, t, steps, upd, sec = (ctypes.c_int32(), ctypes.c_double(), ctypes.c_int64(), ctypes.c_int64(),
                                  ctypes.c_double())
        rc = load().rb_server_request_info(self._h, rid, ctypes.byref(st), ctypes.byref(t), ctypes.byref(steps),
                                           ctypes.byref(upd), ctypes.byref(sec))
        return {"state": st.value, "t": t.value, "steps": steps.value, "cell_updates": upd.value,
                "seconds": sec.value, "status": rc}

    def cancel(self, rid: int):
        _check(load().rb_server_cancel(self._h, rid), "rb_server_cancel")

    def stats(self) -> dict:
        q, a = ctypes.c_int32(), ctypes.c_int32()
        used, budget, upd, launches = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(load().rb_server_stats(self._h, ctypes.byref(q), ctypes.byref(a), ctypes.byref(used),
                                      ctypes.byref(budget), ctypes.byref(upd), ctypes.byref(launches)),
               "rb_server_stats")
        return {"queued": q.value, "active": a.value, "bytes_in_use": used.value, "budget": budget.value,
                "cell_updates": upd.value, "batch_launches": launches.value}

    def drain(self, timeout_s: float = 600.0) -> List[int]:
        """Progress until nothing is queued or active."""
        done, t0 = [], time.perf_counter()
        while True:
            done += self.progress()
            s = self.stats()
            if s["queued"] == 0 and s["active"] == 0:
                return done + self.progress()
            if time.perf_counter() - t0 > timeout_s:
                raise TimeoutError("server did not drain in %.0f s" % timeout_s)


# ---------------------------------------------------------------------------
# the request mix
# ---------------------------------------------------------------------------
@dataclass
class RequestSpec:
    kind: str                 # "tube" or "sedov"
    n: int                    # base grid cells per dimension
    extra: int                # levels above the base level
    params: dict = field(default_factory=dict)

    @property
    def levelmin(self) -> int:
        return int(round(math.log2(self.n)))


def draw_requests(count: int, seed: int = 0, sizes: Sequence[int] = (32, 64, 128), max_extra: int = 2
                  ) -> List[RequestSpec]:
    """Seeded request mix: planar tubes along x (rho log-uniform [0.1, 10], P
    log-uniform [0.01, 100], vx uniform [-2, 2] on each side) or Sedov blasts
    (E log-uniform [0.1, 10]), grid uniform over ``sizes``, extra levels
    uniform over 0..max_extra."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice(sizes))
        extra = int(rng.integers(0, max_extra + 1))
        if rng.random() < 0.5:
            lu = lambda lo, hi: float(10 ** rng.uniform(math.log10(lo), math.log10(hi)))  # noqa: E731
            p = {"rho_l": lu(0.1, 10), "p_l": lu(0.01, 100), "u_l": float(rng.uniform(-2, 2)),
                 "rho_r": lu(0.1, 10), "p_r": lu(0.01, 100), "u_r": float(rng.uniform(-2, 2))}
            out.append(RequestSpec("tube", n, extra, p))
        else:
            e = float(10 ** rng.uniform(-1, 1))
            out.append(RequestSpec("sedov", n, extra, {"energy": e}))
    return out


def _prim_fn(spec: RequestSpec, gamma: float, outflow: bool = False):
    if spec.kind == "tube":
        p = spec.params
        # with outflow in x the tube is [0, 1) with one interface at 0.5;
        # in a periodic box its wrapped second interface sits half a box away
        return ics.shock_tube_prim(p["rho_l"], p["p_l"], p["u_l"], p["rho_r"], p["p_r"], p["u_r"],
                                   periodic_mirror=not outflow)
    # blast energy deposited in the cells of the finest level (the region of
    # r < 2.5 finest cells), as a RAMSES run of that levelmax would set it
    return ics.sedov_prim(spec.levelmin + spec.extra, energy=spec.params["energy"], gamma=gamma)


@dataclass
class BuiltRequest:
    spec: RequestSpec
    dense: Optional[np.ndarray] = None   # uniform problems
    outflow_mask: int = 0                # dense problems: bit d = outflow boundaries along axis d
    tree: Optional[mesh.Octree] = None   # AMR problems (and the uniform tree of the baseline)
    uold: Optional[np.ndarray] = None

    @property
    def is_dense(self) -> bool:
        return self.dense is not None


def _tree_key(spec: RequestSpec, refine_threshold: float, outflow: bool):
    """Requests whose initial refinement is the same share one octree: a
    Sedov blast's gradient flags are its blast region for every E of the mix
    (the deposited pressure exceeds the ambient 1e-5 by orders of magnitude),
    a tube's are its interface planes whenever the density or pressure step
    passes the relative-gradient threshold there (hydro_refine's
    |f(i+1)-f(i-1)| / (|f(i+1)|+|f(i)|+|f(i-1)|) at the two cells beside the
    step), else none."""
    if spec.kind == "sedov":
        return ("sedov", spec.n, spec.extra, refine_threshold)
    p = spec.params

    def step_err(a, b):
        return abs(b - a) / (abs(a) + abs(b) + min(abs(a), abs(b)))
    refined = max(step_err(p["rho_l"], p["rho_r"]), step_err(p["p_l"], p["p_r"])) > refine_threshold
    return ("tube", spec.n, spec.extra, refine_threshold, bool(outflow), refined)


_TREE_CACHE: dict = {}


def build_request(spec: RequestSpec, hp: HydroParams, refine_threshold: float = 0.1,
                  outflow: bool = False, cache: bool = True) -> BuiltRequest:
    """Initial state of a request. Uniform requests become dense grids; AMR
    requests a static octree refined on the relative density/pressure
    gradients of the initial state. outflow: a tube request has outflow
    (zero-gradient) boundaries in x instead of a periodic box (uniform
    requests in the z-streaming kernel's plane loads, AMR requests as free
    boundary regions of the octree)."""
    prim = _prim_fn(spec, hp.gamma, outflow and (spec.extra == 0 or spec.kind == "tube"))
    lmin = spec.levelmin
    if spec.extra == 0:
        tree = mesh.uniform_tree(lmin)
        cells, x = tree.cell_centres(lmin)
        q = prim(x)
        u = np.zeros((5, tree.ncell))
        u[:, cells - 1] = ics.prim_to_cons(q, hp.gamma)
        mask = 1 if (outflow and spec.kind == "tube") else 0
        return BuiltRequest(spec, dense=dense_from_octree(tree, lmin, u), outflow_mask=mask)

    def fields(x):
        q = prim(x)
        return [q[0], q[4]]
    ref = mesh.gradient_refine(fields, [refine_threshold, refine_threshold])
    if spec.kind == "sedov":
        ref = mesh.union_refine(ref, mesh.sphere_refine((0.5, 0.5, 0.5), 2.5 * 0.5 ** (lmin + spec.extra)))
    if outflow and spec.kind == "tube":
        # the gradient test wraps around x; with outflow boundaries the box
        # faces are no interface, and refinement keeps clear of them
        grad = ref

        def ref(level, cells):
            n = 2 ** level
            return np.asarray(grad(level, cells), bool) & (cells[:, 0] >= 4) & (cells[:, 0] < n - 4)
    key = _tree_key(spec, refine_threshold, outflow)
    tree = _TREE_CACHE.get(key) if cache else None
    if tree is None:
        tree = mesh.build_tree(lmin, lmin + spec.extra, ref)
        if outflow and spec.kind == "tube":
            tree = mesh.add_boundaries(tree, ("outflow", None, None))
        if cache:
            _TREE_CACHE[key] = tree
    return BuiltRequest(spec, tree=tree, uold=ics.fill_all_levels(tree, prim, hp.gamma))


def leaf_updates_estimate(b: BuiltRequest) -> int:
    if b.is_dense:
        return int(b.dense[0].size)
    return int(sum(b.tree.leaf_cells(l) for l in range(1, b.tree.nlevelmax + 1)))


# ---------------------------------------------------------------------------
# arrivals, latency
# ---------------------------------------------------------------------------
def poisson_arrivals(count: int, rate: float, seed: int = 1) -> np.ndarray:
    """Arrival offsets (seconds) of a Poisson process of ``rate`` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def fifo_completion(arrivals: Sequence[float], service: Sequence[float]) -> np.ndarray:
    """Completion times of one FIFO server with the given service times."""
    t, out = 0.0, []
    for a, s in zip(arrivals, service):
        t = max(t, a) + s
        out.append(t)
    return np.asarray(out)


def percentiles(x: Sequence[float]) -> dict:
    a = np.asarray(x, dtype=float)
    return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)), "mean": float(a.mean()),
            "max": float(a.max())}


def run_stream(server: Server, reqs: Sequence[BuiltRequest], arrivals: Sequence[float], t_end: float,
               timeout_s: float = 3600.0, keep_results: bool = True) -> dict:
    """Serve ``reqs`` arriving at ``arrivals`` (seconds from start) in real
    time; time-to-solution = result in host memory - arrival. With
    ``keep_results`` False each result array is dropped once its request is
    done (long streams)."""
    order = np.argsort(arrivals, kind="stable")
    t0 = time.perf_counter()
    arrive, finish, ids = {}, {}, {}
    k = 0
    n = len(reqs)
    while len(finish) < n:
        now = time.perf_counter() - t0
        while k < n and arrivals[order[k]] <= now:
            i = int(order[k])
            b = reqs[i]
            rid = (server.submit_dense(b.dense, t_end=t_end, outflow_mask=b.outflow_mask) if b.is_dense
                   else server.submit_octree(b.tree, b.uold, t_end=t_end))
            ids[rid] = i
            arrive[i] = arrivals[i]
            k += 1
        for rid in server.progress():
            finish[ids[rid]] = time.perf_counter() - t0
            if not keep_results:
                server.results.pop(rid, None)
        if server.stats()["active"] == 0 and server.stats()["queued"] == 0 and k < n:
            time.sleep(max(0.0, min(0.002, arrivals[order[k]] - (time.perf_counter() - t0))))
        if time.perf_counter() - t0 > timeout_s:
            raise TimeoutError("stream not served in %.0f s" % timeout_s)
    makespan = time.perf_counter() - t0
    tts = [finish[i] - arrive[i] for i in range(n)]
    updates, steps = 0, []
    for rid, i in ids.items():
        inf = server.info(rid)
        if inf["state"] != REQ_DONE:
            raise RuntimeError("request %d ended in state %d (status %d)" % (rid, inf["state"], inf["status"]))
        updates += inf["cell_updates"]
        steps.append(inf["steps"])
    return {"tts": tts, "latency_s": percentiles(tts), "makespan_s": makespan, "cell_updates": updates,
            "cell_updates_per_s": updates / makespan, "steps": steps, "ids": ids}


def one_at_a_time(reqs: Sequence[BuiltRequest], hp: HydroParams, t_end: float, precision: str = "fp64"
                  ) -> dict:
    """The same requests served one at a time by the plain FP64 path: one
    request on the GPU at a time (the FP64 z-streaming step for dense
    problems, device-scheduled coarse steps as Solver.run for AMR ones),
    submission to result in host memory. Returns the service times."""
    service, updates, per = [], 0, []
    with Server(hp, precision=precision) as srv:
        for b in reqs:
            t0 = time.perf_counter()
            rid = (srv.submit_dense(b.dense, t_end=t_end, outflow_mask=b.outflow_mask) if b.is_dense
                   else srv.submit_octree(b.tree, b.uold, t_end=t_end))
            srv.drain()
            service.append(time.perf_counter() - t0)
            per.append(srv.info(rid)["cell_updates"])
            updates += per[-1]
            srv.results.pop(rid, None)
    return {"service_s": service, "cell_updates": updates, "cell_updates_each": per}


def main(argv=None):
    ap = argparse.ArgumentParser(description="ensemble serving of independent hydro problems")
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--rate", type=float, default=100.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--rates", default=None,
                    help="comma-separated arrival rates: the same requests served once per rate (a rate sweep)")
    ap.add_argument("--sizes", default="32,64,128")
    ap.add_argument("--max-extra", type=int, default=2)
    ap.add_argument("--t-end", type=float, default=0.1)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--steps-per-round", type=int, default=8)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--baseline", action="store_true", help="also serve the stream one at a time with plain FP64")
    ap.add_argument("--periodic-tubes", action="store_true",
                    help="tubes in a periodic box instead of outflow boundaries in x")
    ap.add_argument("--ic-pool", type=int, default=0,
                    help="build only this many distinct initial states; request i takes state i mod N "
                         "(long streams: host memory and set-up time)")
    args = ap.parse_args(argv)
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)
    specs = draw_requests(args.requests, args.seed, [int(x) for x in args.sizes.split(",")], args.max_extra)
    t0 = time.perf_counter()
    npool = args.ic_pool if args.ic_pool > 0 else len(specs)
    pool = [build_request(s, hp, outflow=not args.periodic_tubes) for s in specs[:npool]]
    reqs = [pool[i % npool] for i in range(len(specs))]
    build_s = time.perf_counter() - t0
    rates = [float(r) for r in args.rates.split(",")] if args.rates else [args.rate]
    base = None
    if args.baseline:
        # a request's service time is a function of its initial state: the
        # pool's are measured, request i takes the time of state i mod N
        pb = one_at_a_time(pool, hp, args.t_end, "fp64")
        base = {"service_s": [pb["service_s"][i % npool] for i in range(len(reqs))],
                "cell_updates": int(sum(pb["cell_updates_each"][i % npool] for i in range(len(reqs))))}
    sweep = []
    for rate in rates:
        arrivals = poisson_arrivals(len(reqs), rate, args.seed + 1)
        with Server(hp, precision=args.precision, steps_per_round=args.steps_per_round) as srv:
            res = run_stream(srv, reqs, arrivals, args.t_end, keep_results=npool == len(reqs))
            launches = srv.stats()["batch_launches"]
        row = {"rate_per_s": rate, "latency_s": res["latency_s"], "makespan_s": res["makespan_s"],
               "cell_updates_per_s": res["cell_updates_per_s"], "cell_updates": res["cell_updates"],
               "batched_launches": launches}
        if base is not None:
            # the same arrivals through one FIFO server with the measured
            # one-at-a-time FP64 service times
            comp = fifo_completion(arrivals, base["service_s"])
            tts = comp - arrivals
            row["one_at_a_time_fp64"] = {"latency_s": percentiles(tts), "makespan_s": float(comp[-1] - arrivals[0]),
                                         "cell_updates_per_s": base["cell_updates"] / float(sum(base["service_s"])),
                                         "cell_updates": base["cell_updates"]}
        sweep.append(row)
    out = {"workload": "ensemble serving: %d requests (%s, +0..%d levels), Poisson %s req/s, t_end=%g, seed %d%s"
           % (len(reqs), args.sizes, args.max_extra, ",".join("%g" % r for r in rates), args.t_end, args.seed,
              ", initial states from a pool of %d" % npool if npool < len(reqs) else ""),
           "precision": args.precision, "ic_build_s": build_s,
           "dense_requests": sum(r.is_dense for r in reqs), "amr_requests": sum(not r.is_dense for r in reqs)}
    if len(sweep) == 1:
        out.update(sweep[0])
    else:
        out["sweep"] = sweep
    print(json.dumps(out))
    return out


if __name__ == "__main__":
    main()
