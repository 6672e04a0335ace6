"""GPU: coarse steps with the device-resident scheduler (rb_run), against the
host-driven amr_step sequence (rb_coarse_step) and the oracle.

rb_run keeps dtnew/dtold/t/nstep on the device and may replay the steps from
a CUDA graph; the state, the time and the cell-update count must be bitwise
those of the same number of rb_coarse_step calls.
"""
import numpy as np
import pytest

import oracle
from ramses_b200 import runtime

from helpers import leaf_values, sedov_amr, turbulent_uniform

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("nsub", [1, 2])
def test_run_equals_coarse_steps(cuda_lib, graph, nsub):
    tree, hp, u = sedov_amr(4, 6, interpol_var=1 if nsub == 1 else 0, interpol_type=2 if nsub == 1 else 1)
    ns = [nsub] * 33
    with runtime.Solver(tree, hp, nsubcycle=ns, uold=u) as a, runtime.Solver(tree, hp, nsubcycle=ns, uold=u) as b:
        for _ in range(11):
            a.coarse_step()
        assert b.run(max_steps=11, graph=graph) == 11
        np.testing.assert_array_equal(a.download_state(), b.download_state())
        assert a.t == b.t
        assert a.cell_updates == b.cell_updates
        # the host scheduler state was brought back: both continue identically
        a.coarse_step()
        b.coarse_step()
        np.testing.assert_array_equal(a.download_state(), b.download_state())
        assert a.last_dtnew == b.last_dtnew


def test_run_matches_oracle(cuda_lib, oracle_lib):
    tree, hp, u = sedov_amr(4, 6)
    ns = [2] * 33
    orc = oracle.OracleRun(tree, hp, u, nsubcycle=ns)
    for _ in range(4):
        orc.coarse_step()
    with runtime.Solver(tree, hp, nsubcycle=ns, uold=u) as s:
        assert s.run(max_steps=4) == 4
        cells, ref = leaf_values(tree, orc.uold)
        np.testing.assert_array_equal(s.download_state()[:, cells - 1], ref)
        assert s.t == orc.t
        assert s.cell_updates == orc.cell_updates


@pytest.mark.parametrize("graph", [False, True])
def test_run_stops_at_t_end(cuda_lib, graph):
    tree, hp, u = sedov_amr(3, 5)
    with runtime.Solver(tree, hp, uold=u) as a, runtime.Solver(tree, hp, uold=u) as b:
        a.coarse_step()
        t_end = 13.5 * a.t  # a time no step lands on exactly
        n_host = 1
        while a.t < t_end:
            a.coarse_step()
            n_host += 1
        n_dev = b.run(t_end=t_end, graph=graph)
        assert n_dev == n_host
        assert b.t == a.t and b.t >= t_end
        np.testing.assert_array_equal(a.download_state(), b.download_state())
        # a finished run takes no further step
        assert b.run(t_end=t_end, graph=graph) == 0
        assert b.run(max_steps=0) == 0
        np.testing.assert_array_equal(a.download_state(), b.download_state())


def test_run_after_uniform_dense_steps(cuda_lib):
    """rb_run on a complete level picks up a state that the z-streaming path
    left in its dense mirror."""
    tree, hp, u = turbulent_uniform(5)
    with runtime.Solver(tree, hp, uold=u) as a, runtime.Solver(tree, hp, uold=u) as b:
        for _ in range(6):
            a.coarse_step()
        b.uniform_run(3)
        assert b.run(max_steps=3) == 3
        np.testing.assert_array_equal(a.download_state(), b.download_state())
        assert a.t == b.t


def test_run_mixed_precision(cuda_lib):
    tree, hp, u = sedov_amr(4, 6)
    with runtime.Solver(tree, hp, uold=u) as a, runtime.Solver(tree, hp, precision="mixed", uold=u) as b:
        a.run(max_steps=5)
        b.run(max_steps=5)
        cells, ref = leaf_values(tree, a.download_state())
        got = b.download_state()[:, cells - 1]
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got[0] - ref[0]) / ref[0]) < 1e-4
