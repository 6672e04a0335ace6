"""Shared problem builders for the tests (seeded synthetic inputs)."""
import numpy as np

from ramses_b200 import ics, mesh
from ramses_b200.params import HydroParams


def sedov_uniform(level, riemann="hllc", slope_type=1, courant=0.8):
    hp = HydroParams(gamma=1.4, riemann=riemann, slope_type=slope_type, courant_factor=courant)
    tree = mesh.uniform_tree(level)
    u = ics.fill_all_levels(tree, ics.sedov_prim(level), hp.gamma)
    return tree, hp, u


def sedov_amr(lmin, lmax, riemann="hllc", slope_type=1, courant=0.8, interpol_var=0, interpol_type=1):
    hp = HydroParams(gamma=1.4, riemann=riemann, slope_type=slope_type, courant_factor=courant,
                     interpol_var=interpol_var, interpol_type=interpol_type)
    prim = ics.sedov_prim(lmax)

    def fields(x):
        q = prim(x)
        return [q[0], q[4]]
    ref = mesh.union_refine(mesh.gradient_refine(fields, [0.1, 0.1]),
                            mesh.sphere_refine((0.5, 0.5, 0.5), 2.5 * 0.5 ** lmax))
    tree = mesh.build_tree(lmin, lmax, ref)
    u = ics.fill_all_levels(tree, prim, hp.gamma)
    return tree, hp, u


def turbulent_uniform(level, seed=2024, slope_type=2, riemann="hllc"):
    hp = HydroParams(gamma=1.001, riemann=riemann, slope_type=slope_type, courant_factor=0.8)
    tree = mesh.uniform_tree(level)
    q = ics.turbulent_box_prim_grid(2 ** level, seed=seed, gamma=hp.gamma)
    u = ics.fill_uniform_level_from_grid(tree, level, q, hp.gamma)
    return tree, hp, u


def random_blocks(nv, seed=0, amp=0.3):
    """Random positive states in the Fortran unsplit layout uin(nv,-1:4,-1:4,-1:4,5)
    (C array (5,6,6,6,nv))."""
    rng = np.random.default_rng(seed)
    rho = np.exp(amp * rng.standard_normal((6, 6, 6, nv)))
    vel = amp * rng.standard_normal((3, 6, 6, 6, nv))
    p = np.exp(amp * rng.standard_normal((6, 6, 6, nv)))
    q = np.concatenate([rho[None], vel, p[None]])
    from ramses_b200.ics import prim_to_cons
    return prim_to_cons(q.reshape(5, -1), 1.4).reshape(5, 6, 6, 6, nv)


def leaf_values(tree, u):
    """(cells, values[5,n]) of every leaf cell."""
    cells = []
    for l in range(1, tree.nlevelmax + 1):
        a = tree.active[l]
        if len(a) == 0:
            continue
        c = (tree.ncoarse + np.arange(8)[:, None] * tree.ngridmax + a[None, :]).reshape(-1)
        cells.append(c[tree.son[c - 1] == 0])
    cells = np.concatenate(cells)
    return cells, u[:, cells - 1]


def max_rel(a, b, floor=1e-300):
    return float(np.max(np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), floor)))


def fingerprint(tree, u, gamma):
    """Whole-state fingerprint in the style of the reference's regression
    check (tests/visu/visu_ramses.py check_solution): over the leaf cells,
    sum(log10|x|) for density and pressure and sum(|x|) for each velocity
    component, components below 2e-14 |v| set to zero, summed with fsum."""
    import math
    _, q = leaf_values(tree, u)
    rho = q[0]
    v = q[1:4] / rho
    p = (gamma - 1.0) * (q[4] - 0.5 * rho * (v * v).sum(axis=0))
    vmag = np.sqrt((v * v).sum(axis=0))
    v = np.where(np.abs(v) < 2e-14 * vmag, 0.0, v)
    return {"density": math.fsum(np.log10(np.abs(rho))), "velocity_x": math.fsum(np.abs(v[0])),
            "velocity_y": math.fsum(np.abs(v[1])), "velocity_z": math.fsum(np.abs(v[2])),
            "pressure": math.fsum(np.log10(np.abs(p)))}


def oct_cells(tree):
    """Fortran indices of every cell of the tree's active octs (all levels)."""
    return np.concatenate([(tree.ncoarse + np.arange(8)[:, None] * tree.ngridmax + tree.active[l][None, :]).ravel()
                           for l in range(1, tree.nlevelmax + 1) if tree.noct(l)])


def oracle_prolong_born(old, new, u, hp):
    """make_grid_fine's state for the octs of ``new`` that ``old`` did not
    have at that level under the same father (refine_fine's new octs,
    amr/refine_utils.f90:590-948): interpol_hydro of the father cell and its
    getnborfather neighbours (hydro/interpol_hydro.f90:268-444), level by
    level so that an oct born under a new oct reads its state. The oracle
    restatement; ``u`` is the Fortran-layout state on the pre-remesh tree
    (cell numbering is unchanged by the remesh)."""
    import oracle
    u = np.array(u, np.float64, copy=True)
    old_level = np.zeros(old.ngridmax + 1, np.int64)
    for l in range(1, old.nlevelmax + 1):
        if old.noct(l):
            old_level[old.active[l]] = l
    for l in range(2, new.nlevelmax + 1):
        if not new.noct(l):
            continue
        g = new.active[l].astype(np.int64)
        born = g[(old_level[g] != l) | (old.father[g - 1] != new.father[g - 1])]
        if not len(born):
            continue
        orc = oracle.OracleRun(new, hp, u)
        cells7 = np.stack([orc.getnborfather(int(new.father[b - 1]), l - 1) for b in born])
        u8 = oracle.interpol_hydro(hp, u[:, cells7 - 1].transpose(1, 2, 0))   # (n, 8, 5)
        for ind in range(8):
            u[:, new.ncoarse + ind * new.ngridmax + born - 1] = u8[:, ind, :].T
    return u
