"""Snapshots in the reference's output format (ramses_b200.snapshot), on the
CPU: the writer's files decode to exactly what the reference's own reader
(tests/visu/visu_ramses.py load_snapshot) decoded from them when the fixture
was made (tests/golden/make_snapshot_fixture.py), record by record through
this repository's reader; the checksums follow the reference's regression
check."""
from pathlib import Path

import numpy as np

from ramses_b200 import ics, mesh, snapshot
from ramses_b200.params import HydroParams

GOLDEN = Path(__file__).resolve().parent / "golden" / "snapshot_sedov_l3_4.npz"
FIELDS = ("level", "x", "y", "z", "dx", "density", "velocity_x", "velocity_y", "velocity_z", "pressure")


def snapshot_case():
    """A two-level Sedov state (levels 3-4 on a sphere, seeded velocity noise)
    with spare grids, and the run metadata of the snapshot."""
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)
    tree = mesh.build_tree(3, 4, mesh.sphere_refine((0.5, 0.5, 0.5), 0.2), spare=5)
    u = ics.fill_all_levels(tree, ics.sedov_prim(4), hp.gamma)
    rng = np.random.default_rng(11)
    u[1:4] += 0.01 * rng.standard_normal(u[1:4].shape) * (u[0] > 0)
    meta = {"t": 0.125, "dtold": [0.01] * 4, "dtnew": [0.02] * 4, "nstep": 9, "nstep_coarse": 3}
    return tree, u, hp.gamma, meta


def order(d):
    return np.lexsort((d["z"], d["y"], d["x"], d["level"]))


def test_snapshot_decodes_as_the_reference_reader_did(tmp_path):
    tree, u, gamma, meta = snapshot_case()
    snapshot.write_snapshot(tmp_path, 7, tree, u, gamma, **meta)
    ours = snapshot.read_snapshot(tmp_path, 7)
    ref = np.load(GOLDEN)
    o = order(ours)
    assert len(o) == len(ref["density"])
    for k in FIELDS:
        np.testing.assert_array_equal(np.asarray(ours[k])[o], ref[k], err_msg=k)


def test_snapshot_leaf_cells_and_hydro_variables(tmp_path):
    tree, u, gamma, meta = snapshot_case()
    d = snapshot.write_snapshot(tmp_path, 1, tree, u, gamma, **meta)
    names = sorted(p.name for p in d.iterdir())
    assert names == ["amr_00001.out00001", "header_00001.txt", "hydro_00001.out00001", "hydro_file_descriptor.txt",
                     "info_00001.txt"]
    cells = snapshot.read_snapshot(tmp_path, 1)
    nleaf = sum(tree.leaf_cells(l) for l in range(1, tree.nlevelmax + 1))
    assert len(cells["density"]) == nleaf
    # total mass of the leaf cells = the state's
    mass = float((cells["density"] * cells["dx"] ** 3).sum())
    leaf = np.concatenate([
        (tree.ncoarse + np.arange(8)[:, None] * tree.ngridmax + tree.active[l][None, :]).ravel()
        for l in range(1, tree.nlevelmax + 1) if tree.noct(l)])
    leaf = leaf[tree.son[leaf - 1] == 0]
    lev = np.concatenate([np.full(8 * tree.noct(l), l) for l in range(1, tree.nlevelmax + 1) if tree.noct(l)])
    lev = lev[tree.son[np.concatenate([(tree.ncoarse + np.arange(8)[:, None] * tree.ngridmax
                                        + tree.active[l][None, :]).ravel()
                                       for l in range(1, tree.nlevelmax + 1) if tree.noct(l)]) - 1] == 0]
    ref_mass = float((u[0, leaf - 1] * (0.5 ** lev) ** 3).sum())
    assert abs(mass - ref_mass) <= 1e-14 * ref_mass
    # pressure as backup_hydro forms it
    hv = snapshot.hydro_variables(u[:, leaf - 1], gamma, 1e-10)
    assert np.isclose(np.sort(cells["pressure"]), np.sort(hv[4]), rtol=0, atol=0).all()
    info = (d / "info_00001.txt").read_text()
    assert "time        =  0.125000000000000E+00" in info


def test_solution_sums_follow_the_regression_check():
    cells = {"density": np.array([1.0, 10.0, 100.0]), "pressure": np.array([1.0, 1.0, 1.0]),
             "velocity_x": np.array([1.0, 1e-20, -2.0]), "velocity_y": np.zeros(3), "velocity_z": np.zeros(3)}
    s = snapshot.solution_sums(cells)
    assert s["density"] == 3.0
    assert s["pressure"] == 0.0
    assert s["velocity_x"] == 3.0      # the 1e-20 component is below threshold x |v|: 0
