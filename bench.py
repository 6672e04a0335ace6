"""Benchmark: hydro leaf-cell-updates/s of the unsplit MUSCL-Hancock step.

Workload (one GPU): the supersonic turbulent box, uniform 256^3
(levelmin=levelmax=8, periodic), ln(rho) and solenoidal velocity seeded
Gaussian fields with P(k) ~ k^-4 (sigma=1, RMS Mach 5), P = 0.01 rho,
gamma = 1.001, hllc, slope_type = 2, courant_factor = 0.8. A "step" is one
coarse hydro step of the whole box (courant_fine, godunov_fine, set_uold).

Headline value: FP32-mixed path, state resident in HBM. Reported beside it:
the FP64 drop-in path, the L1(rho) difference FP32-mixed vs FP64 (the FP64
path is bit-identical to the CPU oracle in the parity tests), an end-to-end
number through the C ABI with host buffers, the roofline of the dominant
kernel and a CPU baseline (the FP64 oracle on the host cores).

--gpus N (under torchrun): N independent replicas (the path runs on one GPU;
there is no data-path collective); value = total cell updates of all ranks
divided by the slowest rank's device time.

--impl reference: the CPU restatement of the reference (oracle) on a bounded
sample of the same workload with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "hydro leaf-cell-updates/s FP32-mix vs FP64 at L1(rho)<=1e-5; %HBM peak; p99"
UNIT = "cell-updates/s"
BYTES_PER_CELL_UPDATE = 80  # read uold (5 x 8 B) + write unew (5 x 8 B) per leaf-cell update
ACCURACY_STEPS = 50         # the turbulent-box configuration runs 50 steps


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--level", type=int, default=8)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-octs", type=int, default=32768)
    ap.add_argument("--only", choices=["mixed", "fp64"], default=None,
                    help="run only one precision's timed steps (for profiling)")
    ap.add_argument("--tile-shape", type=int, default=-1,
                    help="oct-tile method: force a godunov tile shape (default: autotuned on the workload)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="z-streaming method: keep the default configuration instead of autotuning")
    ap.add_argument("--stream-config", default=None, metavar="SHAPE,HZ",
                    help="z-streaming method: use this column shape and z extent instead of autotuning "
                         "(profiling runs replay the autotuned choice without its probe launches)")
    ap.add_argument("--pressure-fix", type=float, default=None, metavar="BETA",
                    help="AMR runs with pressure_fix on and beta_fix=BETA (the dual-energy fix)")
    ap.add_argument("--scheme", choices=["muscl", "plmde"], default="muscl",
                    help="predictor of the headline workload (plmde runs the run-time scheme variant)")
    ap.add_argument("--periodic", action="store_true",
                    help="Sedov AMR run on a periodic box instead of outflow boundaries")
    ap.add_argument("--amr", choices=["sedov", "clumps"], default=None,
                    help="instead of the headline, time device-scheduled coarse steps (rb_run) on a static AMR "
                         "tree: sedov = Sedov levels 6-9 refined on a shell, clumps = blast-clump levels 7-11")
    ap.add_argument("--remesh", type=int, default=0, metavar="K",
                    help="with --amr sedov: the dynamic run of config 1, remeshed from the device's refinement "
                         "flags every K coarse steps until --t-end (periodic box)")
    ap.add_argument("--t-end", type=float, default=0.05, help="end time of the --remesh run")
    ap.add_argument("--remesh-spare", type=int, default=1500000,
                    help="free grids reserved for the --remesh run's growing tree")
    ap.add_argument("--remesh-wall", type=float, default=600.0,
                    help="host wall-time budget (s) of the --remesh run: it reports where it stopped")
    ap.add_argument("--serve-requests", type=int, default=48,
                    help="requests of the bounded serving pass (0: none)")
    ap.add_argument("--tile-order", type=int, default=0, choices=[0, 1],
                    help="AMR runs: launch order of the tiles (0 3D Morton, 1 z slabs)")
    ap.add_argument("--method", choices=["stream", "tiles"], default="stream",
                    help="uniform-level kernel: z-streaming over a dense mirror, or godunov_fine oct tiles")
    return ap.parse_args()


def make_solver(runtime, tree, hp, precision, u, args):
    s = runtime.Solver(tree, hp, precision=precision, uold=u)
    s.set_uniform_method(args.method)
    if args.method == "tiles":
        s.set_tile_shape(tree.nlevelmax, args.tile_shape)
    elif args.stream_config:
        shape, hz = (int(x) for x in args.stream_config.split(","))
        s.set_stream_shape(shape, hz)
    elif not args.no_autotune:
        s.autotune_uniform()
    return s


def workload(level, seed, scheme="muscl"):
    from ramses_b200 import ics, mesh
    from ramses_b200.params import HydroParams
    hp = HydroParams(gamma=1.001, riemann="hllc", slope_type=2, courant_factor=0.8, scheme=scheme)
    tree = mesh.uniform_tree(level)
    q = ics.turbulent_box_prim_grid(2 ** level, seed=seed, gamma=hp.gamma)
    u = ics.fill_uniform_level_from_grid(tree, level, q, hp.gamma)
    return tree, hp, u


def config_dict(level, n_gpus, scheme="muscl"):
    n = 2 ** level
    return {"workload": "turbulent box %d^3 uniform (levelmin=levelmax=%d), periodic, hllc, slope_type=2, "
                        "gamma=1.001, Mach 5, courant 0.8%s" % (n, level, "" if scheme == "muscl" else
                                                                ", scheme=" + scheme),
            "cells": n ** 3, "riemann": "hllc", "slope_type": 2, "precision": "fp32-mixed",
            "l2_policy": "inputs larger than L2 (state %.0f MB per copy > 126 MB L2)" % (n ** 3 * 40 / 1e6),
            "parallelism": "replicas" if n_gpus > 1 else "single-gpu"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def tile_dims(shape):
    import ctypes

    from ramses_b200 import runtime
    v = [ctypes.c_int32() for _ in range(4)]
    if runtime.load().rb_tile_shape_info(shape, *[ctypes.byref(x) for x in v]):
        return "?"
    return "%dx%dx%d cells/%d threads" % tuple(x.value for x in v)


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(method, kernel=""):
    """DRAM bytes per launch of the dominant FP32-mixed kernel on this
    workload, from the committed ncu summary of that kernel (line
    'traffic_bytes_per_launch: N')."""
    if method != "stream":
        name = "godunov_tile_mixed_turb256.md"
    elif kernel.startswith("stream2_step_kernel"):
        name = "stream2_step_mixed_turb256.md"
    else:
        name = "stream_step_mixed_turb256.md"
    f = ROOT / "profiles" / name
    if not f.exists():
        return None
    for ln in f.read_text().splitlines():
        if ln.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(ln.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def opcount_figures():
    """Operation counts per cell update of the turbulent-box scheme (hllc,
    moncen) from the committed summary profiles/opcount_hllc_moncen_turb.md:
    {'algorithmic_ops_per_cell_update': ..., 'algorithmic_fp64_flops_per_cell_update': ...}."""
    f = ROOT / "profiles" / "opcount_hllc_moncen_turb.md"
    out = {}
    if f.exists():
        for ln in f.read_text().splitlines():
            k, _, v = ln.partition(":")
            if k.strip() in ("algorithmic_ops_per_cell_update", "algorithmic_fp64_flops_per_cell_update",
                             "reference_fp64_flops_per_cell_update"):
                try:
                    out[k.strip()] = float(v.strip().split()[0])
                except (ValueError, IndexError):
                    pass
    return out


FP64_NOMINAL_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12   # FP64 FMA lanes per SM x SMs x 2 x max clock


def cpu_sample(tree, hp, u, nocts, reps, warmup):
    """Time the oracle's hydro step (courant_fine, set_unew, godunov_fine,
    set_uold) on the first ``nocts`` octs (Morton order) of the finest level,
    with all host threads. Returns (cell-updates/s, cores, description)."""
    import copy

    import oracle
    level = tree.nlevelmax
    sub = copy.copy(tree)
    sub.active = list(tree.active)
    sub.active[level] = tree.active[level][:nocts]
    cores = os.cpu_count() or 1
    run = oracle.OracleRun(sub, hp, u, nthreads=cores)
    times = []
    for i in range(warmup + reps):
        t0 = time.perf_counter()
        dt, *_ = run.courant_fine(level)
        run.set_unew(level)
        run.godunov_fine(level, dt)
        run.set_uold(level)
        t1 = time.perf_counter()
        if i >= warmup:
            times.append(t1 - t0)
    cells = nocts * 8
    value = cells * len(times) / sum(times)
    desc = ("oracle (C restatement, OpenMP %d threads) hydro step on %d of %d octs (%d cells, Morton-contiguous) "
            "of the same workload, %d timed repetitions" % (cores, nocts, tree.noct(level), cells, len(times)))
    return value, cores, desc


def serving_pass(nreq, rate=100.0, seed=0):
    """A bounded pass of the ensemble-serving workload: ``nreq`` seeded
    requests (shock tubes along x with outflow boundaries and Sedov blasts on
    32^3 / 64^3 base grids with 0..1 extra levels, to t = 0.1) arriving as a
    Poisson process, through the FP32-mixed serving engine; beside it the
    same stream served one at a time by the plain FP64 path (measured service
    times replayed through a FIFO queue with the same arrivals)."""
    from ramses_b200 import serve
    from ramses_b200.params import HydroParams
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)
    specs = serve.draw_requests(nreq, seed, (32, 64), 1)
    t0 = time.perf_counter()
    reqs = [serve.build_request(sp, hp, outflow=True) for sp in specs]
    build_s = time.perf_counter() - t0
    arrivals = serve.poisson_arrivals(nreq, rate, seed + 1)
    with serve.Server(hp, precision="mixed") as srv:
        res = serve.run_stream(srv, reqs, arrivals, 0.1, keep_results=False)
    base = serve.one_at_a_time(reqs, hp, 0.1, "fp64")
    comp = serve.fifo_completion(arrivals, base["service_s"])
    b = serve.percentiles(comp - arrivals)
    return {"workload": "%d requests (tubes with outflow in x, Sedov), 32^3/64^3 base grids +0..1 levels, t_end=0.1, "
                        "Poisson %g req/s, seed %d" % (nreq, rate, seed),
            "dense_requests": sum(r.is_dense for r in reqs), "amr_requests": sum(not r.is_dense for r in reqs),
            "p50_s": res["latency_s"]["p50"], "p99_s": res["latency_s"]["p99"],
            "updates_per_s": res["cell_updates_per_s"], "cell_updates": res["cell_updates"],
            "makespan_s": res["makespan_s"], "precision": "fp32-mixed", "ic_build_s": build_s,
            "one_at_a_time_fp64": {"p50_s": b["p50"], "p99_s": b["p99"],
                                   "updates_per_s": base["cell_updates"] / float(sum(base["service_s"])),
                                   "makespan_s": float(comp[-1] - arrivals[0])}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    tree, hp, u = workload(args.level, args.seed, args.scheme)
    nocts = min(args.cpu_sample_octs, tree.noct(args.level))
    value, cores, desc = cpu_sample(tree, hp, u, nocts, args.steps, args.warmup)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": nocts * 8 / value * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(args.level, 1, args.scheme) | {"precision": "fp64", "sample_octs": nocts},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def prim_errors(u_test, u_ref, cells, gamma):
    """L1 (sum |d| / sum |ref|) and L-inf (max |d| / max |ref|) errors of
    density, pressure and velocity magnitude of u_test against u_ref
    (conservative (5, ncell) arrays) over the given 0-based cells."""
    def prim(u):
        r = u[0, cells]
        v = u[1:4, cells] / r
        p = (gamma - 1.0) * (u[4, cells] - 0.5 * r * (v * v).sum(axis=0))
        return {"rho": r, "P": p, "v": np.sqrt((v * v).sum(axis=0))}
    a, b = prim(u_test), prim(u_ref)
    out = {}
    for k in ("rho", "P", "v"):
        d = np.abs(a[k] - b[k])
        out[k] = {"l1": float(d.sum() / np.abs(b[k]).sum()), "linf": float(d.max() / np.abs(b[k]).max())}
    return out


def leaf_cell_index(tree):
    """0-based Fortran-layout indices of every leaf cell of the tree."""
    out = []
    for l in range(1, tree.nlevelmax + 1):
        if tree.noct(l) == 0:
            continue
        cells, _ = tree.cell_centres(l)
        out.append(cells[tree.son[cells - 1] == 0] - 1)
    return np.concatenate(out)


def amr_workload(name, periodic=False):
    """Static AMR trees of the Sedov and blast-clump configurations.
    sedov: levels 6-9; levels 7-9 on a shell of radius 0.25 around the box
    centre (where the shock of E=1 in rho=1 sits near t=0.02) plus the
    initial blast region; the blast starts at t=0. clumps: levels 7-11 refined
    on the relative density/pressure gradient 0.05 of the initial state
    (2.96 M octs, 20.7 M leaf cells)."""
    from ramses_b200 import ics, mesh
    from ramses_b200.params import HydroParams
    if name == "sedov":
        lmin, lmax = 6, 9
        hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)
        prim = ics.sedov_prim(lmax)
        ref = mesh.union_refine(mesh.shell_refine((0.5, 0.5, 0.5), 0.25, 2.5),
                                mesh.sphere_refine((0.5, 0.5, 0.5), 2.5 * 0.5 ** lmax))
        desc = ("Sedov E=1, rho=1, P=1e-5, levels 6-9 (static: shell of radius 0.25 and the blast region), "
                "hllc, slope_type=1, courant 0.8, nsubcycle 2")
    else:
        lmin, lmax = 7, 11
        hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=2, courant_factor=0.8)
        prim = ics.blast_clumps_prim()

        def fields(x):
            q = prim(x)
            return [q[0], q[4]]
        ref = mesh.gradient_refine(fields, [0.05, 0.05])
        desc = ("blast-clump: 32 seeded clumps (contrast 100) + Sedov E=10, levels 7-11 (static: gradient 0.05 "
                "of the initial state), hllc, slope_type=2, courant 0.8, nsubcycle 2")
    tree = mesh.build_tree(lmin, lmax, ref)
    if name == "sedov" and not periodic:
        # outflow (free, bound_type 2) boundaries on all six faces: one layer
        # of boundary coarse cells, refined to levelmin, refilled after every
        # levelmin step
        tree = mesh.add_boundaries(tree, ("outflow",) * 3)
        desc += ", outflow boundaries on all faces (%d boundary octs)" % sum(
            len(g[l]) for g in tree.boundary for l in range(1, lmax + 1))
    else:
        desc += ", periodic"
    return tree, hp, ics.fill_all_levels(tree, prim, hp.gamma), desc


def run_remesh(args):
    """Config 1 with its refinement criterion, remeshed while it runs: Sedov
    (E=1, rho=1, P=1e-5) on levels 6-9, hllc, slope 1, courant 0.8,
    nsubcycle 2, refined from hydro_flag on the device (err_grad_d =
    err_grad_p = 0.1, the criterion of hydro/hydro_flag.f90) every K coarse
    steps until t_end. The tree is the host's (refine_fine's stand-in,
    mesh.refine_from_flags: surviving octs keep their igrids); each remesh
    re-syncs the library's mirror (levels whose inputs are unchanged keep
    their tables) and prolongs the new octs on the device, so no state crosses
    PCIe. Periodic box: the host remesher keeps igrids on single-coarse-cell
    periodic trees, and the blast stays clear of the faces until t = 0.05
    (shock radius ~0.35 of a unit box). Reports the hydro throughput and the
    per-remesh cost of the flags, the host remesh and the re-sync."""
    from ramses_b200 import ics, mesh, runtime
    from ramses_b200.params import HydroParams, RefineParams
    runtime.load()
    lmin, lmax, K = 6, 9, args.remesh
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)
    rp = RefineParams(err_grad_d=0.1, err_grad_p=0.1)
    prim = ics.sedov_prim(lmax)

    def fields(x):
        q = prim(x)
        return [q[0], q[4]]
    t0 = time.perf_counter()
    ref = mesh.union_refine(mesh.gradient_refine(fields, [0.1, 0.1]),
                            mesh.sphere_refine((0.5, 0.5, 0.5), 2.5 * 0.5 ** lmax))
    tree = mesh.build_tree(lmin, lmax, ref, spare=args.remesh_spare)
    u = ics.fill_all_levels(tree, prim, hp.gamma)
    build_s = time.perf_counter() - t0
    prec = args.only or "mixed"
    s = runtime.Solver(tree, hp, precision=prec, uold=u, nsubcycle=[2] * 33)
    hydro_ms, flag_s, host_s, sync_s = 0.0, 0.0, 0.0, 0.0
    coarse, remeshes, updates0 = 0, 0, s.cell_updates
    syncs = []
    max_coarse = args.steps if args.steps > 0 else 1 << 30
    stop = None
    wall0 = time.perf_counter()
    with ClockSampler(0) as clk:
        while s.t < args.t_end and coarse < max_coarse and time.perf_counter() - wall0 < args.remesh_wall:
            n = s.run(t_end=args.t_end, max_steps=min(K, max_coarse - coarse))
            s.synchronize()
            hydro_ms += s.last_run_ms()
            coarse += n
            if n == 0 or s.t >= args.t_end or coarse >= max_coarse:
                break
            a = time.perf_counter()
            flag1 = s.flag_tree(rp)
            b = time.perf_counter()
            try:
                new = mesh.refine_from_flags(s.tree, flag1)
            except ValueError as e:   # the tree outgrew ngridmax: report where the run stopped
                stop = str(e)
                break
            c = time.perf_counter()
            pro0 = s.transfer_stats()["octs_prolonged"]
            s.sync_tree(new)
            s.synchronize()
            d = time.perf_counter()
            st = s.sync_stats()
            st["octs_prolonged"] = s.transfer_stats()["octs_prolonged"] - pro0
            st["octs"] = int(sum(new.noct(l) for l in range(1, lmax + 1)))
            syncs.append(st)
            flag_s += b - a
            host_s += c - b
            sync_s += d - c
            remeshes += 1
            if remeshes % 10 == 0:
                print("remesh %d: coarse %d t=%.3e octs %d, flags %.1f ms, host %.0f ms, sync %.1f ms (%d built)"
                      % (remeshes, coarse, s.t, st["octs"], 1e3 * (b - a), 1e3 * (c - b), 1e3 * (d - c),
                         st["levels_built"]), file=sys.stderr, flush=True)
    wall = time.perf_counter() - wall0
    if stop is None:
        stop = ("t_end reached" if s.t >= args.t_end else "coarse-step cap" if coarse >= max_coarse
                else "wall-time budget")
    tr = s.tree
    levels = [l for l in range(1, tr.nlevelmax + 1) if tr.noct(l)]
    upd = s.cell_updates - updates0
    xfer = s.transfer_stats()
    s.close()
    mean = lambda k: float(np.mean([x[k] for x in syncs])) if syncs else 0.0
    line = {"metric": METRIC, "value": upd / (hydro_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": coarse,
            "warmup": 0, "ms_per_step": hydro_ms / max(coarse, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if prec == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": "Sedov E=1, rho=1, P=1e-5, levels 6-9 remeshed every %d coarse steps from "
                                   "hydro_flag (err_grad_d=err_grad_p=0.1) to t=%g, hllc, slope_type=1, courant "
                                   "0.8, nsubcycle 2, periodic" % (K, args.t_end),
                       "precision": prec, "path": "rb_run between remeshes; rb_hydro_flag, host remesh, "
                                                  "rb_sync_tree with device prolongation at each remesh",
                       "tree_build_s": build_s},
            "t": s.t, "stopped": stop, "coarse_steps": coarse, "final_octs_per_level": {l: tr.noct(l) for l in levels},
            "final_leaf_cells": int(sum(tr.leaf_cells(l) for l in levels)),
            "remesh": {"count": remeshes, "every_coarse_steps": K,
                       "flag_ms_mean": 1e3 * flag_s / max(remeshes, 1),
                       "host_remesh_ms_mean": 1e3 * host_s / max(remeshes, 1),
                       "sync_ms_mean": 1e3 * sync_s / max(remeshes, 1),
                       "sync_phases_ms_mean": {k: mean(k) for k in ("index_ms", "tables_ms", "boundary_ms",
                                                                     "prolong_ms")},
                       "levels_built_mean": mean("levels_built"), "levels_reused_mean": mean("levels_reused"),
                       "octs_prolonged_mean": mean("octs_prolonged"), "octs_mean": mean("octs"),
                       "state_h2d_bytes": xfer["h2d_state_bytes"], "state_d2h_bytes": xfer["d2h_state_bytes"]},
            "hydro_s": hydro_ms / 1e3, "wall_s": wall, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_amr(args):
    """Leaf-cell updates/s of rb_run (device-scheduled coarse steps from CUDA
    graphs) on a static AMR tree, FP32-mixed and FP64."""
    from ramses_b200 import runtime
    runtime.load()
    t0 = time.perf_counter()
    tree, hp, u, desc = amr_workload(args.amr, args.periodic)
    if args.scheme != "muscl":
        hp.scheme = args.scheme
        desc += ", scheme=" + args.scheme
    if args.pressure_fix is not None:
        hp.pressure_fix = True
        hp.beta_fix = args.pressure_fix
        desc += ", pressure_fix with beta_fix=%g" % args.pressure_fix
    build_s = time.perf_counter() - t0
    levels = [l for l in range(1, tree.nlevelmax + 1) if tree.noct(l)]
    out, states = {}, {}
    for prec in ([args.only] if args.only else ["mixed", "fp64"]):
        s = runtime.Solver(tree, hp, precision=prec, uold=u, nsubcycle=[2] * 33)
        s.set_tile_order(args.tile_order)
        # the cost of a remeshing round trip through the drop-in boundary: a
        # full tree re-sync (tables rebuilt on the host) and a state upload
        t0s = time.perf_counter()
        s.sync_tree()
        s.synchronize()
        t1s = time.perf_counter()
        s.upload_state(u)
        s.synchronize()
        sync = {"sync_tree_s": t1s - t0s, "upload_state_s": time.perf_counter() - t1s}
        for l in levels:
            if l >= tree.levelmin:  # the stepped levels
                s.set_tile_shape(l, args.tile_shape)  # -1: autotuned per level
        s.run(max_steps=args.warmup)
        s.synchronize()
        before = s.cell_updates
        with ClockSampler(0) as clk:
            time.sleep(0.3)
            n = s.run(max_steps=args.steps)
            s.synchronize()
        ms = s.last_run_ms()
        upd = s.cell_updates - before
        out[prec] = {"value": upd / (ms / 1e3), "ms_per_coarse_step": ms / max(n, 1), "coarse_steps": n,
                     "t": s.t, "tile_shapes": {l: s.tile_shape(l) for l in levels}, "clocks": clk.summary(),
                     "remesh_round_trip": sync}
        if prec == "mixed" or args.only:
            # hydro_flag on every level but the finest, on the final state
            # (density and pressure gradients of 0.1): the refinement flags
            # a remeshing step would use
            from ramses_b200.params import RefineParams
            rp = RefineParams(err_grad_d=0.1, err_grad_p=0.1)
            flag1 = np.zeros(tree.ncell + 1, np.int32)
            s.synchronize()
            t0f = time.perf_counter()
            nflag = sum(s.hydro_flag(l, rp, flag1)[1] for l in levels if l < tree.nlevelmax)
            out[prec]["hydro_flag"] = {"ms_all_levels": (time.perf_counter() - t0f) * 1e3, "flagged": nflag,
                                       "cells": int(sum(8 * tree.noct(l) for l in levels if l < tree.nlevelmax)),
                                       "note": "host wall time incl. the flag download and OR into flag1"}
        states[prec] = s.download_state()
        s.close()
    if args.only:
        print(json.dumps({"only": args.only, "amr": args.amr, **out[args.only]}), flush=True)
        return
    line = {"metric": METRIC, "value": out["mixed"]["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": out["mixed"]["ms_per_coarse_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": desc, "octs_per_level": {l: tree.noct(l) for l in levels},
                       "leaf_cells": int(sum(tree.leaf_cells(l) for l in levels)), "path": "rb_run, graphs of 8 "
                       "coarse steps, tile shapes autotuned per level", "tree_build_s": build_s},
            "fp64": out["fp64"], "mixed": out["mixed"], "clocks": out["mixed"]["clocks"],
            "mixed_over_fp64": out["mixed"]["value"] / out["fp64"]["value"],
            "accuracy": {"mixed_vs_fp64_leaf_cells": prim_errors(states["mixed"], states["fp64"],
                                                                 leaf_cell_index(tree), hp.gamma),
                         "coarse_steps_compared": args.warmup + args.steps}}
    print(json.dumps(line), flush=True)


class Replicas:
    """The N>1 path: one process per GPU, each an independent replica of the
    workload (the hydro path has no data-path collective). The only
    collectives are a barrier around the timed region and the max over ranks
    of the device time; the job's value is the units of all ranks divided by
    the slowest rank's time. ``dist`` is torch.distributed (or None for one
    process); ``device`` holds the reduction tensor ('cuda' under NCCL,
    'cpu' under gloo)."""

    def __init__(self, dist=None, device="cuda"):
        self.dist = dist
        self.device = device
        self.world = dist.get_world_size() if dist is not None else 1

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def job_rate(self, units_per_rank: float, seconds: float) -> float:
        """Whole-job units per second: all ranks' units over the slowest rank."""
        return units_per_rank * self.world / self.max(seconds)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.amr and args.remesh > 0:
        if args.amr != "sedov":
            raise SystemExit("--remesh runs the Sedov configuration")
        return run_remesh(args)
    if args.amr:
        return run_amr(args)
    from ramses_b200 import runtime
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    runtime.load()
    runtime.select_device(local)

    tree, hp, u = workload(args.level, args.seed, args.scheme)
    level = args.level
    cells = tree.leaf_cells(level)

    rep = Replicas(dist, "cuda")
    barrier, max_over_ranks = rep.barrier, rep.max

    if args.only:
        # one precision's timed steps only (profiling runs: one solver resident)
        s = make_solver(runtime, tree, hp, args.only, u, args)
        s.uniform_run(args.warmup, graph=False)
        s.uniform_run(args.steps, graph=False)
        print(json.dumps({"only": args.only, "cells": cells, "ms_per_step": s.last_run_ms() / args.steps,
                          "kernel_ms": s.last_kernel_ms(), "kernel": s.uniform_info()["kernel"],
                          "value": cells * args.steps / (s.last_run_ms() / 1e3)}), flush=True)
        s.close()
        return

    # ---- FP32-mixed, device resident (headline) -------------------------
    mixed = make_solver(runtime, tree, hp, "mixed", u, args)
    mixed.uniform_run(args.warmup, graph=False)
    barrier()
    mixed.synchronize()
    with ClockSampler(local) as clk:
        time.sleep(0.3)  # let the sampler start before the timed region
        mixed.uniform_run(args.steps, graph=False)
        mixed.synchronize()
    barrier()
    run_ms = max_over_ranks(mixed.last_run_ms())
    kern_ms = mixed.last_kernel_ms()
    mixed_kernel = mixed.uniform_info()["kernel"]
    value = rep.job_rate(cells * args.steps, run_ms / 1e3)
    # the accuracy comparison covers at least the configuration's 50 steps
    acc_steps = max(ACCURACY_STEPS, args.warmup + args.steps)
    if acc_steps > args.warmup + args.steps:
        mixed.uniform_run(acc_steps - args.warmup - args.steps, graph=False)
    u_mixed = mixed.download_state()

    # ---- FP64 drop-in path on the same steps ----------------------------
    f64 = make_solver(runtime, tree, hp, "fp64", u, args)
    f64.uniform_run(args.warmup, graph=False)
    f64_kernel = f64.uniform_info()["kernel"]
    barrier()
    f64.uniform_run(args.steps, graph=False)
    barrier()
    f64_ms = max_over_ranks(f64.last_run_ms())
    f64_kern = f64.last_kernel_ms()
    f64_value = rep.job_rate(cells * args.steps, f64_ms / 1e3)
    if acc_steps > args.warmup + args.steps:
        f64.uniform_run(acc_steps - args.warmup - args.steps, graph=False)
    u_f64 = f64.download_state()
    idx = tree.cell_index(level).reshape(-1) - 1
    rm, rf = u_mixed[0, idx], u_f64[0, idx]
    l1_rho = float(np.abs(rm - rf).sum() / np.abs(rf).sum())
    linf_rho = float(np.max(np.abs(rm - rf) / np.abs(rf)))
    errs = prim_errors(u_mixed, u_f64, idx, hp.gamma)
    f64.close()

    # ---- end to end through the C ABI with host buffers ------------------
    # every step: H2D of the step's input rows of the Fortran-layout uold
    # (the finest level's octs, rb_upload_level_state) from pinned memory,
    # the coarse step (CFL + fused update), D2H of the same rows of the
    # result (rb_download_level_state).
    import ctypes
    nbytes = 5 * 8 * 8 * tree.noct(level)
    host = np.empty((5, tree.ncell))
    try:
        import torch
        pinned = torch.empty((5, tree.ncell), dtype=torch.float64, pin_memory=True)
        host = pinned.numpy()
    except Exception:
        pass
    host[:] = u_mixed
    mixed.upload_state(host)
    mixed.uniform_run(1, graph=False)
    barrier()
    mixed.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        mixed.upload_level_state(level, host)
        mixed.uniform_run(1, graph=False)
        mixed.download_level_state(level, host)
    mixed.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = rep.job_rate(cells * args.e2e_steps, e2e_s)
    mixed.close()

    peak, peak_kind = hbm_peak()
    achieved = BYTES_PER_CELL_UPDATE * cells / (kern_ms / 1e3) / 1e9
    traffic = ncu_traffic(args.method, mixed_kernel)
    # issue ceiling: one instruction per counted operation at full issue
    # (148 SMs x 4 schedulers x 32 threads per cycle at the sampled SM clock)
    ops = opcount_figures()
    clk_sum = clk.summary()
    sm_hz = (clk_sum.get("sm_mhz") or 1965.0) * 1e6
    issue_ceiling = None
    if "algorithmic_ops_per_cell_update" in ops:
        t_issue = ops["algorithmic_ops_per_cell_update"] * cells / (148 * 4 * 32 * sm_hz)
        t_hbm = BYTES_PER_CELL_UPDATE * cells / (peak * 1e9)
        issue_ceiling = min(1.0, t_hbm / t_issue)
    f64_flops = ops.get("algorithmic_fp64_flops_per_cell_update")
    serving = None
    if world == 1 and args.serve_requests > 0:
        serving = serving_pass(args.serve_requests)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nocts = min(args.cpu_sample_octs, tree.noct(level))
        v, cores, desc = cpu_sample(tree, hp, u, nocts, reps=5, warmup=1)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": run_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": config_dict(level, world, args.scheme),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "steps": args.e2e_steps,
                    "path": "rb_upload_level_state + rb_uniform_run(1) + rb_download_level_state "
                            "(the finest level's rows of the Fortran-layout uold), pinned host buffers"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": mixed_kernel + " (fused godunov + update + CFL partials)",
                         "bytes_per_cell_update": BYTES_PER_CELL_UPDATE, "kernel_ms": kern_ms,
                         "peak_kind": peak_kind, "issue_ceiling_frac": issue_ceiling,
                         "algorithmic_ops_per_cell_update": ops.get("algorithmic_ops_per_cell_update"),
                         "issue_ceiling_note": "HBM time over the issue time of the algorithmic operation "
                                               "count at one instruction per operation "
                                               "(profiles/opcount_hllc_moncen_turb.md)"},
            "cpu_baseline": cpu,
            "clocks": clk_sum,
            "gpu_launches": 2 * args.steps,
            "fp64": {"value": f64_value, "ms_per_step": f64_ms / args.steps, "kernel_ms": f64_kern,
                     "kernel": f64_kernel,
                     "roofline_frac": BYTES_PER_CELL_UPDATE * cells / (f64_kern / 1e3) / 1e9 / peak,
                     "algorithmic_tflops": (f64_flops * cells / (f64_kern / 1e3) / 1e12) if f64_flops else None,
                     "flop_frac": (f64_flops * cells / (f64_kern / 1e3) / 1e12 / FP64_NOMINAL_TFLOPS
                                   if f64_flops else None),
                     "flop_peak": "nominal FP64 %.1f TFLOP/s (64 FMA lanes/SM, 148 SMs, 1.965 GHz)"
                                  % FP64_NOMINAL_TFLOPS},
            "mixed_over_fp64": value / f64_value,
            "serving": serving,
            "accuracy": {"l1_rho_mixed_vs_fp64": l1_rho, "linf_rel_rho_mixed_vs_fp64": linf_rho,
                         "mixed_vs_fp64": errs,
                         "steps_compared": acc_steps,
                         "reference": "FP64 GPU path (bit-identical to the FP64 oracle in the parity tests)"},
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
