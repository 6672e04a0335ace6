"""GPU: pressure_fix (RAMSES's dual-energy fix) against the oracle, FP64
bit for bit: set_unew's internal energy, the velocity-divergence and
internal-energy fluxes of godunov_fine (both levels of the update), the pdV
term and the energy repair of set_uold (hydro/godunov_fine.f90:71-86,
203-227, 287-432, 735-744, 775-789, 831-856, 883-906)."""
import numpy as np
import pytest

import oracle
from ramses_b200 import runtime
from ramses_b200.params import HydroParams

from helpers import leaf_values, sedov_amr, sedov_uniform

pytestmark = pytest.mark.gpu


def _pf(hp, beta):
    hp = HydroParams(**{**hp.__dict__})
    hp.pressure_fix = True
    hp.beta_fix = beta
    return hp


def _active_cells(tree, l):
    a = tree.active[l]
    return (tree.ncoarse + np.arange(8)[:, None] * tree.ngridmax + a[None, :]).reshape(-1) - 1


def test_level_calls_match_oracle(cuda_lib, oracle_lib):
    """The drop-in call sequence on one level (set_unew, godunov_fine with its
    coarse-level corrections, set_uold, upload_fine): uold, unew, divu, enew."""
    tree, hp, u = sedov_amr(3, 5)
    hp = _pf(hp, 10.0)
    orc = oracle.OracleRun(tree, hp, u)
    for _ in range(2):
        orc.coarse_step()
    u1 = orc.uold.copy()
    l, dt = 5, 0.3 * orc.dtnew(5)
    orc.set_unew(l)
    orc.set_unew(l - 1)
    orc.godunov_fine(l, dt)
    with runtime.Solver(tree, hp, uold=u1) as s:
        s.set_unew(l)
        s.set_unew(l - 1)
        s.godunov_fine(l, dt)
        dv, en = s.download_pressure_fix()
        c = np.concatenate([_active_cells(tree, l), _active_cells(tree, l - 1)])
        np.testing.assert_array_equal(s.download_unew()[:, c], orc.unew[:, c])
        np.testing.assert_array_equal(dv[c], orc.divu[c])
        np.testing.assert_array_equal(en[c], orc.enew[c])
        orc.set_uold(l)
        orc.upload_fine(l - 1)
        s.set_uold(l)
        s.upload_fine(l - 1)
        _, en = s.download_pressure_fix()
        c = _active_cells(tree, l)
        np.testing.assert_array_equal(en[c], orc.enew[c])
        np.testing.assert_array_equal(s.download_state(), orc.uold)


@pytest.mark.parametrize("beta", [0.0, 10.0])
def test_coarse_steps_match_oracle(cuda_lib, oracle_lib, beta):
    tree, hp, u = sedov_amr(3, 5)
    hp = _pf(hp, beta)
    orc = oracle.OracleRun(tree, hp, u)
    with runtime.Solver(tree, hp, uold=u) as s:
        for _ in range(5):
            orc.coarse_step()
            s.coarse_step()
        np.testing.assert_array_equal(s.download_state(), orc.uold)
        dv, en = s.download_pressure_fix()
        np.testing.assert_array_equal(dv, orc.divu)
        np.testing.assert_array_equal(en, orc.enew)
        assert s.t == orc.t


@pytest.mark.parametrize("graph", [False, True])
def test_device_scheduled_run_matches_oracle(cuda_lib, oracle_lib, graph):
    tree, hp, u = sedov_amr(3, 5)
    hp = _pf(hp, 10.0)
    orc = oracle.OracleRun(tree, hp, u)
    for _ in range(5):
        orc.coarse_step()
    with runtime.Solver(tree, hp, uold=u) as s:
        assert s.run(max_steps=5, graph=graph) == 5
        np.testing.assert_array_equal(s.download_state(), orc.uold)
        assert s.t == orc.t


def test_uniform_run_matches_oracle(cuda_lib, oracle_lib):
    tree, hp, u = sedov_uniform(4)
    hp = _pf(hp, 10.0)
    orc = oracle.OracleRun(tree, hp, u)
    for _ in range(12):
        orc.coarse_step()
    with runtime.Solver(tree, hp, uold=u) as s:
        s.uniform_run(12)
        np.testing.assert_array_equal(s.download_state(), orc.uold)


def test_fix_is_exercised(oracle_lib):
    """The cases above repair cells: with beta_fix = 10 the run departs from
    the one without the pressure fix."""
    tree, hp, u = sedov_amr(3, 5)
    a = oracle.OracleRun(tree, hp, u)
    b = oracle.OracleRun(tree, _pf(hp, 10.0), u)
    for _ in range(5):
        a.coarse_step()
        b.coarse_step()
    assert np.any(a.uold != b.uold)


def test_mixed_precision_close_to_fp64(cuda_lib):
    tree, hp, u = sedov_amr(3, 5)
    hp = _pf(hp, 10.0)
    with runtime.Solver(tree, hp, uold=u) as a, runtime.Solver(tree, hp, precision="mixed", uold=u) as b:
        for _ in range(5):
            a.coarse_step()
            b.coarse_step()
        cells, ra = leaf_values(tree, a.download_state())
        _, rb_ = leaf_values(tree, b.download_state())
        assert np.all(np.isfinite(rb_))
        assert np.abs(ra[0] - rb_[0]).sum() / np.abs(ra[0]).sum() < 1e-5
