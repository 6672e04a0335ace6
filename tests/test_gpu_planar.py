"""GPU: the CUDA path against the pinned 1D/2D whole-run oracle.

oracle/ramses_oracle_amr.c reproduces the reference's own regression
checksums for its 1D Sod tube and 2D implosion
(tests/test_oracle_regression_cpu.py). On one complete level those problems
extended along the missing axes are planar: every transverse term of the 3D
scheme is an exact zero, so the device's FP64 path must reproduce the 1D/2D
restatement bit for bit when both take the same time steps:

* the drop-in level calls (rb_set_unew, rb_godunov_fine with the 1D/2D
  run's own dt, rb_set_uold, rb_make_boundary_hydro) with the regression
  tests' walls;
* the z-streaming kernel (rb_uniform_run) on the periodic versions, the
  1D/2D restatement taking the device run's time steps (its own 3D CFL
  condition); in FP32-mixed within the north-star tolerance.
"""
import numpy as np
import pytest

from ramses_b200 import runtime

from helpers import planar_expected, planar_lowdim_run, planar_tree

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,level,nsteps", [("sod1d", 5, 40), ("implosion2d", 5, 25)])
def test_drop_in_level_calls_equal_pinned_oracle(cuda_lib, oracle_lib, kind, level, nsteps):
    hp, init, final = planar_lowdim_run(kind, level, nsteps)
    tree, u = planar_tree(kind, level, init)
    with runtime.Solver(tree, hp, uold=u) as s:
        for dt in final["dt"]:
            s.set_unew(level)
            s.godunov_fine(level, float(dt))
            s.set_uold(level)
            s.make_boundary_hydro(level)
        got = s.download_state()
    cells, want = planar_expected(kind, level, tree, final)
    np.testing.assert_array_equal(got[:, cells - 1], want)
    assert np.any(want[1] != 0.0)


def _stream_run(tree, hp, u, nsteps, precision):
    """nsteps of rb_uniform_run one at a time: (state, the dt of each step)."""
    dts = []
    with runtime.Solver(tree, hp, uold=u, precision=precision) as s:
        for k in range(nsteps):
            t0 = s.t
            s.uniform_run(1, graph=False)
            if k == 0:
                assert t0 == 0.0
                dts.append(s.t)  # 0 + dt0
            if k + 1 < nsteps:
                dts.append(s.next_dt)
        assert s.uniform_info()["method"] == "stream", s.uniform_info()
        return s.download_state(), np.array(dts), s.t


@pytest.mark.parametrize("kind,level,nsteps", [("sod1d_periodic", 6, 40), ("implosion2d_periodic", 5, 25)])
def test_streaming_kernel_equals_pinned_oracle(cuda_lib, oracle_lib, kind, level, nsteps):
    hp, init, _ = planar_lowdim_run(kind, level, 0)
    tree, u = planar_tree(kind, level, init)
    got, dts, t = _stream_run(tree, hp, u, nsteps, "fp64")
    _, _, final = planar_lowdim_run(kind, level, nsteps, dt_force=dts)
    assert final["t"] == t
    cells, want = planar_expected(kind, level, tree, final)
    np.testing.assert_array_equal(got[:, cells - 1], want)
    assert np.any(want[1] != 0.0)


@pytest.mark.parametrize("kind,level,nsteps", [("sod1d_periodic", 6, 40), ("implosion2d_periodic", 5, 25)])
def test_mixed_streaming_close_to_pinned_oracle(cuda_lib, oracle_lib, kind, level, nsteps):
    """FP32-mixed z-streaming (the headline kernel) against the pinned oracle
    taking the same time steps: L1(rho, P) <= 1e-5, momentum along the
    missing axes exactly zero."""
    hp, init, _ = planar_lowdim_run(kind, level, 0)
    tree, u = planar_tree(kind, level, init)
    got, dts, _ = _stream_run(tree, hp, u, nsteps, "mixed")
    _, _, final = planar_lowdim_run(kind, level, nsteps, dt_force=dts)
    cells, want = planar_expected(kind, level, tree, final)
    g, w = got[:, cells - 1], want
    l1 = np.abs(g[0] - w[0]).sum() / np.abs(w[0]).sum()
    assert l1 <= 1e-5, l1
    ekin = lambda a: 0.5 * (a[1] ** 2 + a[2] ** 2 + a[3] ** 2) / a[0]
    pg, pw = 0.4 * (g[4] - ekin(g)), 0.4 * (w[4] - ekin(w))
    assert np.abs(pg - pw).sum() / np.abs(pw).sum() <= 1e-5
    nd = 1 if kind.startswith("sod") else 2
    assert np.all(g[1 + nd:4] == 0.0)
