"""GPU: physical boundaries (make_boundary_hydro, hydro/hydro_boundary.f90:
5-260, called after every level step, amr/amr_step.f90:515) against the
oracle, FP64 bit for bit, through the level call, host- and device-scheduled
coarse steps and the uniform run.

The comparison covers the octs of the box and every boundary oct whose
reference oct is one of those or lies in an earlier boundary region: the
cells the box's stencils and interpolations read. The outer layers of a
boundary region copy from octs of the same region; the reference's sweep
updates those in nvector batches, the device in one pass, so they may lag
one fill behind each other without reaching the box."""
import numpy as np
import pytest

import oracle
from ramses_b200 import ics, mesh, runtime
from ramses_b200.params import HydroParams

pytestmark = pytest.mark.gpu


def determined_cells(tree):
    """1-based cells of the octs of the box and of the boundary octs whose
    reference oct is determined before their region is filled."""
    cells = []
    for l in range(1, tree.nlevelmax + 1):
        known = set(tree.active[l].tolist())
        for ib, bt in enumerate(tree.boundary_type):
            if l >= len(tree.boundary[ib]) or len(tree.boundary[ib][l]) == 0:
                continue
            g = tree.boundary[ib][l]
            dirn = bt % 10
            inbor = dirn + 1 if dirn % 2 else dirn - 1
            ref = tree.son[tree.nbor[inbor - 1, g - 1] - 1]
            ok = np.array([r in known for r in ref.tolist()])
            known.update(g[ok].tolist())
        octs = np.array(sorted(known), dtype=np.int64)
        if len(octs):
            cells.append((tree.ncoarse + np.arange(8)[:, None] * tree.ngridmax + octs[None, :]).reshape(-1))
    return np.concatenate(cells)


def tube(level, bounds=("outflow",) * 3, **kw):
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=2, courant_factor=0.8, **kw)
    prim = ics.shock_tube_prim(1.0, 1.0, 0.4, 0.125, 0.1, -0.3, x0=0.5, periodic_mirror=False)
    tree = mesh.add_boundaries(mesh.build_tree(level, level, None), bounds)
    return tree, hp, ics.fill_all_levels(tree, prim, hp.gamma)


def sedov_amr_bounded(bounds, lmin=3, lmax=5, **kw):
    hp = HydroParams(**{"gamma": 1.4, "riemann": "hllc", "slope_type": 1, "courant_factor": 0.8, **kw})
    prim = ics.sedov_prim(lmax)
    ref = mesh.sphere_refine((0.5, 0.5, 0.5), 0.12)
    tree = mesh.add_boundaries(mesh.build_tree(lmin, lmax, ref), bounds)
    return tree, hp, ics.fill_all_levels(tree, prim, hp.gamma)


def check(tree, a, b):
    c = determined_cells(tree) - 1
    np.testing.assert_array_equal(a[:, c], b[:, c])


def test_level_fill_bitwise(cuda_lib, oracle_lib):
    """rb_make_boundary_hydro on a state whose boundary cells hold noise."""
    tree, hp, u = tube(4, ("outflow", "reflexive", "outflow"))
    rng = np.random.default_rng(3)
    for ib in range(len(tree.boundary_type)):
        g = tree.boundary[ib][4].astype(np.int64)
        cells = (tree.ncoarse + np.arange(8)[:, None] * tree.ngridmax + g[None, :]).reshape(-1)
        u[:, cells - 1] = 1.0 + rng.random((5, len(cells)))
    orc = oracle.OracleRun(tree, hp, u)  # fills every level
    with runtime.Solver(tree, hp, uold=u) as s:
        check(tree, s.download_state(), orc.uold)


@pytest.mark.parametrize("bounds", [("outflow",) * 3, ("reflexive",) * 3, ("outflow", None, "reflexive")])
def test_tube_coarse_steps_bitwise(cuda_lib, oracle_lib, bounds):
    tree, hp, u = tube(4, bounds)
    orc = oracle.OracleRun(tree, hp, u)
    with runtime.Solver(tree, hp, uold=u) as s:
        for _ in range(12):
            orc.coarse_step()
            s.coarse_step()
        check(tree, s.download_state(), orc.uold)
        assert s.t == orc.t


@pytest.mark.parametrize("riemann", ["hllc", "llf"])
def test_amr_device_run_bitwise(cuda_lib, oracle_lib, riemann):
    tree, hp, u = sedov_amr_bounded(("outflow",) * 3, riemann=riemann)
    orc = oracle.OracleRun(tree, hp, u)
    for _ in range(4):
        orc.coarse_step()
    with runtime.Solver(tree, hp, uold=u) as s:
        assert s.run(max_steps=4) == 4
        check(tree, s.download_state(), orc.uold)


def test_resync_with_boundaries_keeps_tables_and_results(cuda_lib, oracle_lib):
    """A re-sync of the same bounded tree (rb_set_boundary then
    rb_sync_tree, as the drop-in does after a host tree change) keeps every
    level's tables, and the run stays bit-identical to the oracle; a re-sync
    with other boundary types rebuilds them all."""
    tree, hp, u = sedov_amr_bounded(("outflow",) * 3)
    orc = oracle.OracleRun(tree, hp, u)
    for _ in range(4):
        orc.coarse_step()
    nonempty = sum(1 for lvl in range(1, tree.nlevelmax + 1) if tree.noct(lvl))
    with runtime.Solver(tree, hp, uold=u) as s:
        assert s.run(max_steps=2) == 2
        s.sync_tree(tree)
        st = s.sync_stats()
        assert st["levels_built"] == 0 and st["levels_reused"] == nonempty, st
        assert s.transfer_stats()["octs_prolonged"] == 0
        assert s.run(max_steps=2) == 2
        check(tree, s.download_state(), orc.uold)
    t2, hp2, u2 = sedov_amr_bounded(("reflexive",) * 3)
    with runtime.Solver(tree, hp, uold=u) as s:
        s.sync_tree(t2)   # same octs, walls instead of free boundaries
        st = s.sync_stats()
        assert st["levels_reused"] == 0 and st["levels_built"] == nonempty, st


def test_amr_walls_pressure_fix_bitwise(cuda_lib, oracle_lib):
    tree, hp, u = sedov_amr_bounded(("reflexive",) * 3, pressure_fix=True, beta_fix=0.5)
    orc = oracle.OracleRun(tree, hp, u)
    with runtime.Solver(tree, hp, uold=u) as s:
        for _ in range(3):
            orc.coarse_step()
            s.coarse_step()
        check(tree, s.download_state(), orc.uold)


def test_uniform_run_bitwise(cuda_lib, oracle_lib):
    tree, hp, u = tube(5)
    orc = oracle.OracleRun(tree, hp, u)
    for _ in range(10):
        orc.coarse_step()
    with runtime.Solver(tree, hp, uold=u) as s:
        s.uniform_run(10)
        check(tree, s.download_state(), orc.uold)


def test_mixed_close_to_fp64(cuda_lib):
    tree, hp, u = tube(5)
    with runtime.Solver(tree, hp, uold=u) as a, runtime.Solver(tree, hp, precision="mixed", uold=u) as b:
        for _ in range(10):
            a.coarse_step()
            b.coarse_step()
        idx = tree.cell_index(5) - 1
        ra, rb_ = a.download_state()[0][idx], b.download_state()[0][idx]
        assert np.abs(ra - rb_).sum() / np.abs(ra).sum() < 1e-5


def test_large_region_fill_bitwise(cuda_lib, oracle_lib):
    """Regions larger than one launch's threads (levelmin 6: the z regions
    hold 294,912 octs each)."""
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)
    tree = mesh.add_boundaries(mesh.build_tree(6, 6, None), ("outflow", "reflexive", "outflow"))
    assert max(len(g[6]) for g in tree.boundary) > 148 * 32 * 256 // 8
    u = ics.fill_all_levels(tree, ics.sedov_prim(6), hp.gamma)
    rng = np.random.default_rng(5)
    for ib in range(len(tree.boundary_type)):
        g = tree.boundary[ib][6].astype(np.int64)
        cells = (tree.ncoarse + np.arange(8)[:, None] * tree.ngridmax + g[None, :]).reshape(-1)
        u[:, cells - 1] = 1.0 + rng.random((5, len(cells)))
    orc = oracle.OracleRun(tree, hp, u)
    with runtime.Solver(tree, hp, uold=u) as s:
        check(tree, s.download_state(), orc.uold)
        orc.coarse_step()
        s.coarse_step()
        check(tree, s.download_state(), orc.uold)


def test_boundary_argument_checks(cuda_lib):
    """Imposed boundaries are rejected; a tile shape that would hold octs of
    the box and of the boundary layer is refused."""
    import ctypes
    tree, hp, u = tube(3)
    with runtime.Solver(tree, hp, uold=u) as s:
        L = runtime.load()
        bt = np.array([21], np.int32)
        nb = np.zeros(tree.nlevelmax, np.int32)
        g = np.zeros(1, np.int32)
        P = ctypes.POINTER(ctypes.c_int32)
        rc = L.rb_set_boundary(s._h, 1, bt.ctypes.data_as(P), nb.ctypes.data_as(P), g.ctypes.data_as(P))
        assert rc == 1  # RB_ERR_INVALID
        with pytest.raises(runtime.RBError):
            s.set_tile_shape(1, 3)  # 4x4x2 octs on a level with one oct per coarse cell
