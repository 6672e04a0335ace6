"""The residency protocol of the drop-in boundary, replayed as the Fortran
host would drive it.

The replay follows adaptive_loop's coarse step (amr/adaptive_loop.f90:143-151)
and amr_step (amr/amr_step.f90:320-445), as the oracle restates them, for a
pure-hydro single-rank run: per level
courant_fine, set_unew, the finer levels, godunov_fine, set_uold,
upload_fine, make_boundary_hydro and hydro_flag, each device call preceded by
rb_ensure_device as the patched routines do. The host's uold array is only
touched through rb_ensure_device / rb_ensure_host. Checked:

* no uold crosses PCIe during coarse steps that do not remesh (one upload
  at start-up, nothing after);
* a remesh that keeps every level's oct count (one oct killed, one created
  elsewhere, igrids reused as kill_grid / make_grid_fine do) is detected
  through rb_note_tree_changed, although the per-level counts and the
  sampled son checksum that the earlier binding relied on are unchanged;
* the new oct gets make_grid_fine's state (interpol_hydro of its father
  cell and the getnborfather neighbours) on the device, bit for bit as the
  oracle computes it, again without a state upload;
* the run continues bit-identical to the oracle on the remeshed tree.
"""
import numpy as np
import pytest

import oracle
from ramses_b200 import ics, mesh, runtime
from ramses_b200.params import HydroParams, RefineParams

pytestmark = pytest.mark.gpu


class FortranHost:
    """The reference's host loop with the patched hydro routines."""

    def __init__(self, solver, u):
        self.s = solver
        self.u = np.ascontiguousarray(u, np.float64).copy()   # the host's uold
        L = solver.tree.nlevelmax
        self.dtnew = [0.0] * (L + 2)
        self.dtold = [0.0] * (L + 2)
        self.t = 0.0
        self.nsub = [2] * (L + 2)
        self.flags = None
        self.rp = RefineParams(err_grad_d=0.1, err_grad_p=0.1)

    def device(self):
        self.s.ensure_device(self.u)

    def amr_step(self, l, icount):
        s, tree = self.s, self.s.tree
        if tree.noct(l) == 0:
            return
        # newdt_fine -> courant_fine (pm/newdt_fine.f90:177)
        self.dtold[l] = self.dtnew[l]
        self.dtnew[l] = tree.boxlen / s.hp.smallc
        self.device()
        dt_all, *_ = s.courant_fine(l, self.dtnew[l])
        self.dtnew[l] = min(self.dtnew[l], dt_all)
        if l > tree.levelmin:
            self.dtnew[l] = min(self.dtnew[l - 1] / float(np.float32(self.nsub[l - 1])), self.dtnew[l])
        self.device()
        s.set_unew(l)
        if l < tree.nlevelmax and tree.noct(l + 1) > 0:
            self.amr_step(l + 1, 1)
            self.amr_step(l + 1, 2)
        else:
            if l < tree.nlevelmax:
                self.dtold[l + 1] = self.dtnew[l] / self.nsub[l]
                self.dtnew[l + 1] = self.dtnew[l] / self.nsub[l]
            self.t += self.dtnew[l]
        self.device()
        s.godunov_fine(l, self.dtnew[l])
        s.set_uold(l)
        s.upload_fine(l)
        # make_boundary_hydro: a periodic box has no boundary regions
        if l < tree.nlevelmax:   # flag_fine -> hydro_flag: flags come back, uold stays
            self.device()
            s.hydro_flag(l, self.rp)
        if l > tree.levelmin and icount == 2:
            self.dtnew[l - 1] = self.dtold[l] + self.dtnew[l]

    def coarse_step(self):
        tree = self.s.tree
        self.amr_step(tree.levelmin, 1)
        # adaptive_loop.f90:146-151: the levels below levelmin are restricted
        # after the base-level step (upload_fine is wrapped to the device)
        if tree.levelmin < tree.nlevelmax:
            for il in range(tree.levelmin - 1, 0, -1):
                self.device()
                self.s.upload_fine(il)

    def refine(self, new_tree):
        """refine_fine changed the tree; its host-side interpolation for the
        new octs works on a stale uold and is never uploaded."""
        self.s.note_tree_changed(new_tree)


def old_binding_stamp(tree):
    """The change stamp of the earlier binding: per-level oct counts and
    every 97th son entry."""
    stamp = 0
    for l in range(1, tree.nlevelmax + 1):
        stamp = (stamp * 31 + tree.noct(l)) & 0xFFFFFFFFFFFFFFFF
    for i in range(0, tree.ncell, 97):
        stamp = (stamp * 7 + int(tree.son[i])) & 0xFFFFFFFFFFFFFFFF
    return stamp


def swap_one_oct(tree, level):
    """Coordinates of every level with one leaf oct of ``level`` killed and
    one created under a level-(level-1) leaf cell away from it, keeping the
    per-level counts, the nesting rule and the sampled stamp."""
    n = 2 ** (level - 1)
    oc = {l: tree.coords[l].copy() for l in range(1, tree.nlevelmax + 1)}
    children = tree.coords[level + 1] // 2 if level < tree.nlevelmax and tree.noct(level + 1) else np.zeros((0, 3))
    ckeys = set(map(tuple, children)) if len(children) else set()
    have = set(map(tuple, oc[level]))
    stamp0 = old_binding_stamp(tree)
    for i in range(len(oc[level]) - 1, -1, -1):
        kill = tuple(oc[level][i])
        if kill in ckeys:
            continue
        # a level-(level-1) cell without an oct, on the far side of the box
        for dz in range(n):
            cand = ((kill[0] + n // 2) % n, (kill[1] + n // 2) % n, (kill[2] + dz) % n)
            if cand in have:
                continue
            new = dict(oc)
            new[level] = np.concatenate([np.delete(oc[level], i, axis=0), np.array([cand], np.int64)])
            try:
                t2 = mesh.remesh(tree, new)
            except ValueError:
                continue
            if old_binding_stamp(t2) == stamp0:
                return t2
    raise RuntimeError("no count-preserving remesh found")


def test_resident_protocol_with_count_preserving_remesh(cuda_lib, oracle_lib):
    lmin, lmax = 3, 5
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)
    tree = mesh.build_tree(lmin, lmax, mesh.sphere_refine((0.5, 0.5, 0.5), 0.15), spare=64)
    u = ics.fill_all_levels(tree, ics.sedov_prim(lmax), hp.gamma)
    orc = oracle.OracleRun(tree, hp, u, nsubcycle=[2] * 33)
    s = runtime.Solver(tree, hp, nsubcycle=[2] * 33)
    host = FortranHost(s, u)
    nbytes = 5 * tree.ncell * 8
    try:
        for _ in range(2):
            host.coarse_step()
            orc.coarse_step()
        st = s.transfer_stats()
        assert st["h2d_state_bytes"] == nbytes and st["d2h_state_bytes"] == 0, st
        assert st["tree_syncs"] == 1, st
        assert host.t == orc.t
        # remesh keeping every level's oct count
        t2 = swap_one_oct(tree, lmin + 1)
        assert [t2.noct(l) for l in range(1, lmax + 1)] == [tree.noct(l) for l in range(1, lmax + 1)]
        assert old_binding_stamp(t2) == old_binding_stamp(tree)
        # the new oct: a grid that was not at this level or had another
        # father (kill_grid freed an igrid, make_grid_fine reused it)
        old_at = set(tree.active[lmin + 1].tolist())
        born = [g for g in t2.active[lmin + 1].tolist()
                if g not in old_at or t2.father[g - 1] != tree.father[g - 1]]
        assert len(born) == 1
        # the oracle side: make_grid_fine's state for the new oct from the
        # pre-remesh state (cell numbering is unchanged by the remesh)
        u_pre = orc.uold.copy()
        orc2 = oracle.OracleRun(t2, hp, u_pre, nsubcycle=[2] * 33)
        g = int(born[0])
        f = int(t2.father[g - 1])
        cells7 = orc2.getnborfather(f, lmin)
        u2 = oracle.interpol_hydro(hp, u_pre[:, cells7 - 1].T[None])[0]   # (8, 5)
        for ind in range(8):
            u_pre[:, t2.ncoarse + ind * t2.ngridmax + g - 1] = u2[ind]
        orc2 = oracle.OracleRun(t2, hp, u_pre, nsubcycle=[2] * 33)
        orc2.m.t = orc.t
        host.refine(t2)
        assert s.tree_needs_sync()
        host.device()               # the next patched call: re-sync, prolongation, no upload
        assert not s.tree_needs_sync()
        st = s.transfer_stats()
        assert st["h2d_state_bytes"] == nbytes and st["d2h_state_bytes"] == 0, st
        assert st["tree_syncs"] == 2 and st["octs_prolonged"] == 1, st
        cells = np.concatenate([(t2.ncoarse + np.arange(8)[:, None] * t2.ngridmax + t2.active[l][None, :]).ravel()
                                for l in range(1, lmax + 1) if t2.noct(l)])
        # the host reads uold (an output): one download
        host_u = np.zeros((5, t2.ncell))
        s.ensure_host(host_u)
        s.ensure_host(host_u)     # nothing newer on the device: no second copy
        assert s.transfer_stats()["d2h_state_bytes"] == nbytes
        new_cells = t2.ncoarse + np.arange(8) * t2.ngridmax + g
        np.testing.assert_array_equal(host_u[:, new_cells - 1], u_pre[:, new_cells - 1])
        diff = np.nonzero(np.any(host_u[:, cells - 1] != u_pre[:, cells - 1], axis=0))[0]
        assert len(diff) == 0, ("cells differing after the re-sync", (cells[diff] - 1 - t2.ncoarse) % t2.ngridmax + 1)
        for _ in range(2):
            host.coarse_step()
            orc2.coarse_step()
        st = s.transfer_stats()
        assert st["h2d_state_bytes"] == nbytes and st["d2h_state_bytes"] == nbytes, st
        s.ensure_host(host_u)
        assert s.transfer_stats()["d2h_state_bytes"] == 2 * nbytes
        diff = np.nonzero(np.any(host_u[:, cells - 1] != orc2.uold[:, cells - 1], axis=0))[0]
        assert len(diff) == 0, ("cells differing after 2 steps on the new tree", len(diff),
                                sorted(set(((cells[diff] - 1 - t2.ncoarse) % t2.ngridmax + 1).tolist())), g)
        assert host.t == orc2.t
    finally:
        s.close()


def test_host_writes_are_uploaded_once(cuda_lib):
    """rb_note_host_state_written makes the next rb_ensure_device upload, and
    only that one."""
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)
    tree = mesh.uniform_tree(3)
    u = ics.fill_all_levels(tree, ics.sedov_prim(3), hp.gamma)
    with runtime.Solver(tree, hp) as s:
        s.ensure_device(u)
        s.ensure_device(u)
        assert s.transfer_stats()["h2d_state_bytes"] == 5 * tree.ncell * 8
        u2 = u.copy()
        u2[0] *= 1.5
        s.note_host_state_written()
        s.ensure_device(u2)
        s.ensure_device(u2)
        assert s.transfer_stats()["h2d_state_bytes"] == 2 * 5 * tree.ncell * 8
        back = np.zeros_like(u2)
        s.ensure_host(back)                       # device not newer: no copy
        assert not back.any()
        s.download_state(back)
        np.testing.assert_array_equal(back, u2)


@pytest.mark.parametrize("case", ["uniform", "amr"])
def test_level_state_transfers_touch_only_the_level_rows(cuda_lib, case):
    """rb_upload_level_state / rb_download_level_state move the rows of one
    level's octs and leave every other row as it is on both sides; the AMR
    level's igrids come in several runs."""
    from helpers import sedov_uniform
    if case == "uniform":
        tree, hp, u = sedov_uniform(4)
    else:  # a remeshed tree: the level's igrids recycled from the free list
        hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)
        t1 = mesh.build_tree(3, 5, mesh.sphere_refine((0.5, 0.5, 0.5), 0.12), spare=3000)
        tree = mesh.remesh(t1, mesh.oct_sets(3, 5, mesh.sphere_refine((0.56, 0.5, 0.5), 0.12)))
        u = ics.fill_all_levels(tree, ics.sedov_prim(5), hp.gamma)
    level = 4
    a = tree.active[level].astype(np.int64)
    rows = (tree.ncoarse + np.arange(8)[:, None] * tree.ngridmax + a[None, :]).reshape(-1) - 1
    other = np.setdiff1d(np.arange(tree.ncell), rows)
    if case == "amr":
        assert np.count_nonzero(np.diff(np.sort(a)) != 1) >= 1
    with runtime.Solver(tree, hp, uold=u) as s:
        b0 = s.transfer_stats()
        h = u.copy()
        h[:, rows] *= 1.25
        h[:, other] = np.nan
        s.upload_level_state(level, h)
        got = s.download_state()
        np.testing.assert_array_equal(got[:, rows], h[:, rows])
        np.testing.assert_array_equal(got[:, other], u[:, other])
        out = np.full_like(u, -7.0)
        s.download_level_state(level, out)
        np.testing.assert_array_equal(out[:, rows], h[:, rows])
        assert np.all(out[:, other] == -7.0)
        b1 = s.transfer_stats()
        nb = rows.size * 5 * 8
        assert b1["h2d_state_bytes"] - b0["h2d_state_bytes"] == nb
        assert b1["d2h_state_bytes"] - b0["d2h_state_bytes"] == nb + 5 * 8 * tree.ncell
        if case == "uniform":  # after steps held in the dense mirror
            s.uniform_run(2, graph=False)
            full = s.download_state()
            out2 = np.full_like(u, -7.0)
            s.download_level_state(level, out2)
            np.testing.assert_array_equal(out2[:, rows], full[:, rows])
            s.upload_level_state(level, full)
            s.uniform_run(1, graph=False)
            ref = np.full_like(u, -7.0)
            s.download_level_state(level, ref)
        if case == "uniform":
            with runtime.Solver(tree, hp, uold=full) as s2:
                s2.uniform_run(1, graph=False)
                np.testing.assert_array_equal(s2.download_state()[:, rows], ref[:, rows])
