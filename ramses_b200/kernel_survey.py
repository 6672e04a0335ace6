"""A profiling workload that launches the library's secondary kernels once
each on states larger than L2, for per-kernel DRAM throughput captures
(``ncu --metrics ... -k regex:<kernel> -c 1``). The headline and AMR kernels
have their own workloads in bench.py; this covers the entry points the
drop-in host calls one at a time and the remesh path:

* ``rb_set_unew`` / ``rb_set_uold`` / ``rb_upload_fine`` standalone
  (copy_octs_kernel, upload_fine_kernel), FP64 and with pressure_fix
  around a ``rb_godunov_fine`` (pf_set_unew_kernel, pdv_kernel,
  pf_fix_kernel), on the 256^3 turbulent box;
* ``rb_download_state`` (permute_d2f_kernel) and a uniform step that leaves
  the dense mirror and comes back (oct_to_dense_kernel, dense_to_oct_kernel);
* ``rb_courant_cells_noalloc`` on the level's 16.7 M cells
  (noalloc_cfl_partial, noalloc_cfl_final);
* ``rb_unsplit`` on 32,768 blocks in the Fortran layout (unsplit_fortran_kernel);
* a remesh of the Sedov shell tree through ``rb_sync_tree``
  (scatter_son_kernel, prolong_new_octs_kernel).

Usage: ``python -m ramses_b200.kernel_survey`` (prints one line per stage).
"""
from __future__ import annotations

import ctypes
import time

import numpy as np


def main() -> None:
    import torch

    from ramses_b200 import ics, mesh, runtime
    from ramses_b200.params import HydroParams

    runtime.load()
    level = 8
    t0 = time.perf_counter()
    hp = HydroParams(gamma=1.001, riemann="hllc", slope_type=2, courant_factor=0.8)
    tree = mesh.uniform_tree(level)
    q = ics.turbulent_box_prim_grid(2 ** level, seed=2024, gamma=hp.gamma)
    u = ics.fill_uniform_level_from_grid(tree, level, q, hp.gamma)
    print("turbulent box 256^3 built in %.1f s" % (time.perf_counter() - t0), flush=True)

    with runtime.Solver(tree, hp, uold=u) as s:
        s.set_unew(level)
        s.set_uold(level)
        s.upload_fine(level - 1)
        s.synchronize()
        print("set_unew, set_uold, upload_fine (FP64)", flush=True)
        out = s.download_state()
        print("download_state", flush=True)
        s.uniform_run(1, graph=False)
        s.download_state(out)
        print("uniform step through the dense mirror and back", flush=True)

    hpf = HydroParams(gamma=1.001, riemann="hllc", slope_type=2, courant_factor=0.8, pressure_fix=True, beta_fix=10.0)
    with runtime.Solver(tree, hpf, uold=u) as s:
        dt, *_ = s.courant_fine(level)
        s.set_unew(level)
        s.godunov_fine(level, dt)
        s.set_uold(level)
        s.synchronize()
        print("set_unew, godunov_fine, set_uold with pressure_fix", flush=True)

    # the allocation-free CFL reduction on the level's cells (Fortran cell order)
    a = tree.active[level].astype(np.int64)
    cells = (tree.ncoarse + np.arange(8)[:, None] * tree.ngridmax + a[None, :]).reshape(-1)
    n = len(cells)
    dev = torch.from_numpy(np.ascontiguousarray(u[:, cells - 1]).reshape(-1)).cuda()
    res = torch.zeros(4, dtype=torch.float64, device="cuda")
    hpc = runtime.hydro_params_c(hp)
    stream = torch.cuda.current_stream().cuda_stream
    rc = runtime.load().rb_courant_cells_noalloc(ctypes.byref(hpc), ctypes.c_void_p(dev.data_ptr()), n, n,
                                                  tree.boxlen * 0.5 ** level, tree.boxlen / hp.smallc,
                                                  ctypes.c_void_p(res.data_ptr()), ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    if rc:
        raise RuntimeError(runtime.load().rb_last_error().decode())
    print("courant_cells_noalloc on %d cells: dt %.6e" % (n, res[0].item()), flush=True)
    del dev

    # unsplit in the Fortran layout on 32,768 random blocks
    rng = np.random.default_rng(7)
    nv = 32768
    uin = np.empty((5, 6, 6, 6, nv))
    uin[0] = 1.0 + 0.3 * rng.random((6, 6, 6, nv))
    uin[1:4] = 0.3 * (rng.random((3, 6, 6, 6, nv)) - 0.5)
    uin[4] = 2.0 + rng.random((6, 6, 6, nv))
    runtime.unsplit(HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8), uin, None,
                    1.0 / 64, 1e-4)
    print("unsplit on %d blocks" % nv, flush=True)

    # a remesh of the Sedov shell tree: son diffs and new octs prolonged on the device
    lmin, lmax = 6, 9
    hps = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)
    centre = (0.5, 0.5, 0.5)

    def shell(r):
        return mesh.union_refine(mesh.shell_refine(centre, r, 2.5), mesh.sphere_refine(centre, 2.5 * 0.5 ** lmax))
    t1 = mesh.build_tree(lmin, lmax, shell(0.25), spare=200000)
    us = ics.fill_all_levels(t1, ics.sedov_prim(lmax), hps.gamma)
    t2 = mesh.remesh(t1, mesh.oct_sets(lmin, lmax, shell(0.26)))
    with runtime.Solver(t1, hps, uold=us) as s:
        before = s.transfer_stats()["octs_prolonged"]
        s.sync_tree(t2)
        s.synchronize()
        print("remesh %d -> %d octs: %d prolonged on the device, %s" % (
            sum(t1.noct(l) for l in range(1, lmax + 1)), sum(t2.noct(l) for l in range(1, lmax + 1)),
            s.transfer_stats()["octs_prolonged"] - before, s.sync_stats()), flush=True)


if __name__ == "__main__":
    main()
