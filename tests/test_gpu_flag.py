"""GPU: hydro_flag (refinement flags from the gradient criterion) computed on
the device state through the C ABI, against the oracle's restatement of
hydro/hydro_flag.f90 + hydro_refine on the same state: bit-for-bit equal
flag arrays and equal counts of new flags."""
import numpy as np
import pytest

import oracle
from ramses_b200 import runtime
from ramses_b200.params import RefineParams

from helpers import sedov_amr

pytestmark = pytest.mark.gpu

CRITERIA = [RefineParams(err_grad_d=0.02), RefineParams(err_grad_p=0.1),
            RefineParams(err_grad_u=0.05), RefineParams(err_grad_d=0.02, err_grad_p=0.1, err_grad_u=0.05,
                                                        floor_d=1e-3, floor_p=1e-6, floor_u=1e-2)]


@pytest.mark.parametrize("ic", range(len(CRITERIA)))
def test_hydro_flag_matches_oracle(cuda_lib, oracle_lib, ic):
    rp = CRITERIA[ic]
    tree, hp, u = sedov_amr(4, 6)
    ns = [2] * 33
    orc = oracle.OracleRun(tree, hp, u, nsubcycle=ns)
    with runtime.Solver(tree, hp, nsubcycle=ns, uold=u) as s:
        for _ in range(3):
            orc.coarse_step()
            s.coarse_step()
        np.testing.assert_array_equal(s.download_state(), orc.uold)
        total = 0
        for lvl in range(1, tree.nlevelmax + 1):
            want, n_want = orc.hydro_flag(lvl, rp)
            got, n_got = s.hydro_flag(lvl, rp)
            np.testing.assert_array_equal(got, want)
            assert n_got == n_want
            total += n_got
        assert total > 0
        # existing flags are kept and not counted again
        pre = np.zeros(tree.ncell + 1, np.int32)
        pre[1::5] = 1
        want, n_want = orc.hydro_flag(5, rp, pre.copy())
        got, n_got = s.hydro_flag(5, rp, pre.copy())
        np.testing.assert_array_equal(got, want)
        assert n_got == n_want


def test_hydro_flag_after_dense_steps(cuda_lib, oracle_lib):
    """The flags read the newest state also when it lives in the z-streaming
    kernel's dense mirror (flags first, then the state is downloaded)."""
    from helpers import turbulent_uniform
    tree, hp, u = turbulent_uniform(4)
    rp = RefineParams(err_grad_d=0.5, err_grad_p=0.8)
    with runtime.Solver(tree, hp, uold=u) as s:
        s.uniform_run(2)
        got = [s.hydro_flag(lvl, rp) for lvl in (2, 3)]
        orc = oracle.OracleRun(tree, hp, s.download_state())
    for lvl, (g, n) in zip((2, 3), got):
        want, n_want = orc.hydro_flag(lvl, rp)
        np.testing.assert_array_equal(g, want)
        assert n == n_want


def test_hydro_flag_errors(cuda_lib):
    tree, hp, u = sedov_amr(3, 5)
    with runtime.Solver(tree, hp, uold=u) as s:
        with pytest.raises(runtime.RBError):
            s.hydro_flag(9, RefineParams(err_grad_d=0.1))
        f, n = s.hydro_flag(5, RefineParams(err_grad_d=0.0))   # finest level: nothing to do
        assert n == 0 and not f.any()
