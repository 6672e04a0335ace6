"""The allocation-free CFL reduction (rb_courant_cells_noalloc) against the
regular entry point rb_courant_fine on the same cells.

rb_courant_cells_noalloc exists for callers that cannot call cudaMalloc or
cudaFree mid-run (those calls wait for the whole device to go idle): it keeps
its scratch in a fixed array inside the library. This file is collected last,
so a run that stops at the first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

from ramses_b200 import runtime

from helpers import turbulent_uniform

pytestmark = pytest.mark.gpu


def _level_cells(tree, u, level):
    """(5, n) conservative values of the level's cells in Fortran cell order."""
    a = tree.active[level].astype(np.int64)
    cells = (tree.ncoarse + np.arange(8)[:, None] * tree.ngridmax + a[None, :]).reshape(-1)
    return np.ascontiguousarray(u[:, cells - 1])


def test_noalloc_cfl_matches_courant_fine_twice(cuda_lib):
    import torch
    level = 5
    tree, hp, u = turbulent_uniform(level)
    with runtime.Solver(tree, hp, uold=u) as s:
        dt_ref, mass_ref, ekin_ref, eint_ref = s.courant_fine(level)
    cells = _level_cells(tree, u, level)
    n = cells.shape[1]
    stride = n + 3  # padded rows: the entry point honours the stride
    host = np.zeros((5, stride))
    host[:, :n] = cells
    dev = torch.from_numpy(host.reshape(-1)).cuda()
    out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
    hpc = runtime.hydro_params_c(hp)
    dx = tree.boxlen * 0.5 ** level
    dt_in = tree.boxlen / hp.smallc
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out.fill_(-1.0)
        torch.cuda.synchronize()
        rc = runtime.load().rb_courant_cells_noalloc(ctypes.byref(hpc), ctypes.c_void_p(dev.data_ptr()), n, stride,
                                                      dx, dt_in, ctypes.c_void_p(out.data_ptr()),
                                                      ctypes.c_void_p(stream))
        assert rc == 0, runtime.load().rb_last_error()
        torch.cuda.synchronize()
        dt, mass, ekin, eint = out.cpu().tolist()
        assert dt == dt_ref, (call, dt, dt_ref)              # a min: order independent, exact
        assert abs(mass - mass_ref) <= 1e-12 * abs(mass_ref)  # sums: summation order differs
        assert abs(ekin - ekin_ref) <= 1e-12 * abs(ekin_ref)
        assert abs(eint - eint_ref) <= 1e-12 * abs(eint_ref)


def test_noalloc_rejects_sizes_beyond_capacity(cuda_lib):
    from ramses_b200.params import HydroParams
    hpc = runtime.hydro_params_c(HydroParams())
    big = 16777216 + 1
    rc = runtime.load().rb_courant_cells_noalloc(ctypes.byref(hpc), ctypes.c_void_p(16), big, big, 0.1, 1.0,
                                                  ctypes.c_void_p(16), None)
    assert rc == 8  # RB_ERR_CAPACITY, returned before anything touches the device
    msg = runtime.load().rb_last_error().decode()
    assert "capacity" in msg and str(big) in msg, msg
