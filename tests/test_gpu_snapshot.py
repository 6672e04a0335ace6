"""Snapshots of device states in the reference's output format, and the
reference's Sod shock tube (tests/hydro/sod-tube/sod-tube.nml: walls at
both x ends, hllc, moncen, courant 0.8, gamma 1.4, to t = 0.245) run as a
planar tube on a uniform 32^3 grid (the device path is NDIM = 3) on the GPU
and by the oracle: the snapshot's regression checksums (the reference's
check_solution sums) agree exactly, and the density profile lies within a
first-order scheme's error of the reference's own exact-solution table."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from ramses_b200 import ics, mesh, runtime, snapshot
from ramses_b200.params import HydroParams

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "sod_tube_ana.csv"


def sod_tube(level):
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=2, courant_factor=0.8)
    tree = mesh.add_boundaries(mesh.build_tree(level, level, None), ("reflexive", None, None))
    prim = ics.shock_tube_prim(1.0, 1.0, 0.0, 0.125, 0.1, 0.0, x0=0.5, periodic_mirror=False)
    return tree, hp, ics.fill_all_levels(tree, prim, hp.gamma)


def test_sod_tube_snapshot_checksums_gpu_equal_oracle(cuda_lib, oracle_lib, tmp_path):
    level, t_end = 5, 0.245
    tree, hp, u = sod_tube(level)
    orc = oracle.OracleRun(tree, hp, u)
    while orc.t < t_end:
        orc.coarse_step()
    with runtime.Solver(tree, hp, uold=u) as s:
        s.run(t_end=t_end)
        assert s.t == orc.t
        s.write_snapshot(tmp_path / "gpu", 1)
    snapshot.write_snapshot(tmp_path / "cpu", 1, tree, orc.uold, hp.gamma, hp.smallr, t=orc.t)
    a = snapshot.read_snapshot(tmp_path / "gpu", 1)
    b = snapshot.read_snapshot(tmp_path / "cpu", 1)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    sa, sb = snapshot.solution_sums(a), snapshot.solution_sums(b)
    assert sa == sb, (sa, sb)
    assert len(a["density"]) == 8 ** level
    # the planar profile against the reference's exact-solution table
    ana = np.loadtxt(GOLDEN, delimiter=",")
    x = a["x"]
    xs = np.unique(x)
    rho = np.array([a["density"][x == xi].mean() for xi in xs])
    assert np.all(np.array([np.ptp(a["density"][x == xi]) for xi in xs]) == 0.0)   # planar to the bit
    ref = np.interp(xs, ana[:, 0], ana[:, 2])
    assert np.abs(rho - ref).mean() / np.abs(ref).mean() < 0.06
