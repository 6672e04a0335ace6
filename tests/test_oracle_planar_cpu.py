"""The 3D oracle against the pinned 1D/2D whole-run oracle on planar data.

oracle/ramses_oracle_amr.c reproduces the reference's own regression
checksums for the 1D Sod tube and the 2D implosion
(tests/test_oracle_regression_cpu.py). On one complete level with walls,
those problems extended along the missing axes (periodic there) are planar:
every transverse slope, face-state term, kinetic-energy term and flux
difference of the 3D scheme is an exact zero. Driven with the 1D/2D run's
own time steps (its 3D CFL condition would differ: cmpdt sums the sound
speed over ndim), the 3D restatement (oracle/ramses_oracle.c:
godunov_fine with trace3d, make_boundary_hydro) must reproduce the 1D/2D
states bit for bit, which ties it to the pinned restatement.
"""
import numpy as np
import pytest

import oracle
from helpers import planar_expected, planar_lowdim_run, planar_tree


@pytest.mark.parametrize("kind,level,nsteps", [("sod1d", 5, 40), ("implosion2d", 5, 25),
                                               ("sod1d_periodic", 5, 30), ("implosion2d_periodic", 4, 20)])
def test_3d_oracle_equals_pinned_lowdim_oracle_on_planar_data(kind, level, nsteps):
    hp, init, final = planar_lowdim_run(kind, level, nsteps)
    tree, u = planar_tree(kind, level, init)
    orc = oracle.OracleRun(tree, hp, u)
    cells, want = planar_expected(kind, level, tree, init)
    np.testing.assert_array_equal(orc.uold[:, cells - 1], want)
    for dt in final["dt"]:
        orc.set_unew(level)
        orc.godunov_fine(level, float(dt))
        orc.set_uold(level)
        orc.make_boundary_hydro(level)
    cells, want = planar_expected(kind, level, tree, final)
    np.testing.assert_array_equal(orc.uold[:, cells - 1], want)
    assert np.any(want[1] != 0.0)  # the waves moved


def test_forced_time_steps_reproduce_the_run():
    """The dt_force hook (used to drive the 1D/2D restatement with another
    code's time steps) given the run's own steps changes nothing."""
    hp, init, final = planar_lowdim_run("implosion2d", 4, 15)
    _, _, again = planar_lowdim_run("implosion2d", 4, 15, dt_force=final["dt"])
    np.testing.assert_array_equal(again["u"], final["u"])
    assert again["t"] == final["t"]
    _, _, other = planar_lowdim_run("implosion2d", 4, 15, dt_force=0.5 * final["dt"])
    assert other["t"] != final["t"]


@pytest.mark.parametrize("riemann", ["llf", "hll", "hllc", "acoustic", "exact"])
@pytest.mark.parametrize("slope_type", [0, 1, 2])
def test_3d_oracle_planar_other_schemes(riemann, slope_type):
    """The same bitwise reduction for every Riemann solver and the slope
    types both restatements take (the Riemann solvers are shared; the
    traces, slopes and updates are not)."""
    kind, level, nsteps = "implosion2d", 4, 10
    hp, init, final = planar_lowdim_run(kind, level, nsteps, riemann=riemann, slope_type=slope_type)
    tree, u = planar_tree(kind, level, init)
    orc = oracle.OracleRun(tree, hp, u)
    for dt in final["dt"]:
        orc.set_unew(level)
        orc.godunov_fine(level, float(dt))
        orc.set_uold(level)
        orc.make_boundary_hydro(level)
    cells, want = planar_expected(kind, level, tree, final)
    np.testing.assert_array_equal(orc.uold[:, cells - 1], want)
