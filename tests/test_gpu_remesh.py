"""GPU: remeshing driven by the device's refinement flags, against the oracle.

The host loop of a RAMSES run that remeshes (amr/amr_step.f90:320-445:
flag_fine -> refine_fine between level steps), with the tree kept by the
host and the hydro on the device:

* hydro_flag on the device for every level (the gradient criterion of
  hydro/hydro_flag.f90) gives the same flags as the oracle;
* the host builds the new tree from those flags (refine_fine's role:
  ``mesh.refine_from_flags``, igrids of surviving octs kept, freed igrids
  reused), the library re-synchronises its mirror and fills the new octs on
  the device with make_grid_fine's interpol_hydro state: bit-identical to
  the oracle's prolongation of the same octs, with no state upload;
* levels whose inputs did not change keep their tables (rb_sync_stats), and
  the run continues bit-identical to the oracle on every new tree.
"""
import numpy as np
import pytest

import oracle
from ramses_b200 import ics, mesh, runtime
from ramses_b200.params import HydroParams, RefineParams

from helpers import oct_cells, oracle_prolong_born

pytestmark = pytest.mark.gpu


def _sedov_dynamic(lmin, lmax, spare):
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)
    tree = mesh.build_tree(lmin, lmax, mesh.sphere_refine((0.5, 0.5, 0.5), 0.12), spare=spare)
    u = ics.fill_all_levels(tree, ics.sedov_prim(lmax), hp.gamma)
    return tree, hp, u


@pytest.mark.parametrize("precision", ["fp64"])
def test_flag_driven_remeshes_match_oracle(cuda_lib, oracle_lib, precision):
    lmin, lmax = 3, 6
    tree, hp, u = _sedov_dynamic(lmin, lmax, spare=6000)
    rp = RefineParams(err_grad_d=0.1, err_grad_p=0.1)
    ns = [2] * 33
    orc = oracle.OracleRun(tree, hp, u, nsubcycle=ns)
    born_total = 0
    with runtime.Solver(tree, hp, nsubcycle=ns, uold=u, precision=precision) as s:
        for r in range(3):
            for _ in range(2):
                s.coarse_step()
                orc.coarse_step()
            np.testing.assert_array_equal(s.download_state(), orc.uold)
            # flag_fine: device flags equal the oracle's
            flag1 = s.flag_tree(rp)
            want = np.zeros(tree.ncell + 1, np.int32)
            for lvl in range(lmin, lmax):
                if tree.noct(lvl):
                    want, _ = orc.hydro_flag(lvl, rp, want)
            np.testing.assert_array_equal(flag1, want)
            # refine_fine on the host; the library re-syncs and prolongs
            new = mesh.refine_from_flags(tree, flag1)
            assert any(not np.array_equal(new.active[lvl], tree.active[lvl]) for lvl in range(1, lmax + 1))
            before = s.transfer_stats()
            s.sync_tree(new)
            after = s.transfer_stats()
            assert after["h2d_state_bytes"] == before["h2d_state_bytes"]
            born_total += after["octs_prolonged"] - before["octs_prolonged"]
            st = s.sync_stats()
            # the complete levels up to levelmin are unchanged by any remesh
            assert st["levels_reused"] >= lmin, st
            assert st["levels_built"] >= 1, st
            t = orc.t
            u_new = oracle_prolong_born(tree, new, orc.uold, hp)
            cells = oct_cells(new)
            got = s.download_state()
            np.testing.assert_array_equal(got[:, cells - 1], u_new[:, cells - 1])
            orc = oracle.OracleRun(new, hp, u_new, nsubcycle=ns)
            orc.m.t = t
            tree = new
        for _ in range(2):
            s.coarse_step()
            orc.coarse_step()
        cells = oct_cells(tree)
        got = s.download_state()
        np.testing.assert_array_equal(got[:, cells - 1], orc.uold[:, cells - 1])
        assert s.t == orc.t
    assert born_total > 0


def test_resync_of_the_same_tree_reuses_every_level(cuda_lib, oracle_lib):
    """A re-sync with an unchanged tree rebuilds nothing and changes no
    result; a tree with one oct moved rebuilds only the levels that read it."""
    from helpers import sedov_amr
    tree, hp, u = sedov_amr(3, 5)
    ns = [2] * 33
    orc = oracle.OracleRun(tree, hp, u, nsubcycle=ns)
    with runtime.Solver(tree, hp, nsubcycle=ns, uold=u) as s:
        s.coarse_step()
        orc.coarse_step()
        s.sync_tree(tree)
        st = s.sync_stats()
        nonempty = sum(1 for lvl in range(1, tree.nlevelmax + 1) if tree.noct(lvl))
        assert st["levels_built"] == 0 and st["levels_reused"] == nonempty, st
        assert s.transfer_stats()["octs_prolonged"] == 0
        s.coarse_step()
        orc.coarse_step()
        np.testing.assert_array_equal(s.download_state(), orc.uold)
