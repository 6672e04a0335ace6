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


# ---- planar problems: the pinned 1D/2D whole-run oracle against the 3D path ----
# The reference's pure-hydro regression setups (tests/hydro/sod-tube, 1D, and
# tests/hydro/implosion, 2D) on one complete level with walls. On data that
# is constant along the missing axes every transverse term of the 3D scheme
# adds an exact zero, so a 3D run driven with the same time steps equals the
# 1D/2D restatement bit for bit.
PLANAR = {
    "sod1d": {"ndim": 1, "gamma": 1.4,
              "regions": [{"x_center": 0.25, "length_x": 0.5, "d": 1.0, "p": 1.0},
                          {"x_center": 0.75, "length_x": 0.5, "d": 0.125, "p": 0.1}],
              "boundaries": [(-1, -1, 0, 0, 1), (1, 1, 0, 0, 1)],
              "bounds3d": ("reflexive", None, None)},
    "implosion2d": {"ndim": 2, "gamma": 1.4,
                    "regions": [{"x_center": 0.5, "y_center": 0.5, "length_x": 1.0, "length_y": 1.0,
                                 "exp_region": 10.0, "d": 1.0, "p": 1.0},
                                {"x_center": 0.0, "y_center": 0.0, "length_x": 1.0, "length_y": 1.0,
                                 "exp_region": 1.0, "d": 0.125, "p": 0.4}],
                    "boundaries": [(-1, -1, 0, 0, 1), (1, 1, 0, 0, 1), (-1, 1, 1, 1, 1), (-1, 1, -1, -1, 1)],
                    "bounds3d": ("reflexive", "reflexive", None)},
}


PLANAR["sod1d_periodic"] = dict(PLANAR["sod1d"], boundaries=[], bounds3d=(None, None, None))
PLANAR["implosion2d_periodic"] = dict(PLANAR["implosion2d"], boundaries=[], bounds3d=(None, None, None))


def planar_lowdim_run(kind, level, nsteps, dt_force=None, riemann="hllc", slope_type=2):
    """The 1D/2D oracle on one complete level: (initial leaves, leaves after
    nsteps coarse steps with the run's own CFL time steps or ``dt_force``,
    the dts taken)."""
    import oracle
    c = PLANAR[kind]
    hp = HydroParams(gamma=c["gamma"], riemann=riemann, slope_type=slope_type, courant_factor=0.8,
                     interpol_var=0, interpol_type=2)
    kw = dict(ndim=c["ndim"], levelmin=level, nlevelmax=level, ngridmax=4 ** level + 64, tout=1e30,
              regions=c["regions"], boundaries=c["boundaries"], nsubcycle=[1] * level, nexpand=[1] * level)
    init = oracle.run_amr(hp, (-1.0, -1.0, -1.0), max_coarse_steps=0, **kw)
    final = oracle.run_amr(hp, (-1.0, -1.0, -1.0), max_coarse_steps=nsteps, dt_force=dt_force, **kw)
    assert final["nstep_coarse"] == nsteps and len(final["dt"]) == nsteps
    return hp, init, final


def _lowdim_grid(res, ndim, level):
    """leaf cells -> dense [y][x][v] (ndim = 2) or [x][v] arrays"""
    n = 2 ** level
    idx = np.floor(res["pos"] * n).astype(np.int64)
    if ndim == 1:
        g = np.zeros((n, 3))
        g[idx[:, 0]] = res["u"]
    else:
        g = np.zeros((n, n, 4))
        g[idx[:, 1], idx[:, 0]] = res["u"]
    return g


def planar_tree(kind, level, init):
    """The 3D tree with the kind's walls (periodic along the missing axes)
    and uold with level ``level`` set from the 1D/2D initial leaves, the
    coarser levels from the same regions at their cell centres."""
    c = PLANAR[kind]
    nd = c["ndim"]
    tree = mesh.build_tree(level, level, None)
    if any(c["bounds3d"]):
        tree = mesh.add_boundaries(tree, c["bounds3d"])

    def prim(x):
        q = np.zeros((5, len(x)))
        for r in c["regions"]:
            xn = 2.0 * np.abs(x[:, 0] - r["x_center"]) / r["length_x"]
            yn = 2.0 * np.abs(x[:, 1] - r.get("y_center", 0.0)) / r.get("length_y", 1.0) if nd > 1 else 0 * xn
            en = r.get("exp_region", 2.0)
            rr = (xn ** en + yn ** en) ** (1.0 / en) if en < 10 else np.maximum(xn, yn)
            q[0] = np.where(rr < 1.0, r["d"], q[0])
            q[4] = np.where(rr < 1.0, r["p"], q[4])
        return q
    u = ics.fill_all_levels(tree, prim, c["gamma"])
    g = _lowdim_grid(init, nd, level)
    idx = tree.cell_index(level)  # [z, y, x]
    if nd == 1:
        for v3, v1 in ((0, 0), (1, 1), (4, 2)):
            u[v3, idx.reshape(-1, idx.shape[2]) - 1] = g[None, :, v1]
        u[2:4, idx.reshape(-1) - 1] = 0.0
    else:
        for v3, v2 in ((0, 0), (1, 1), (2, 2), (4, 3)):
            u[v3, idx - 1] = np.broadcast_to(g[None, :, :, v2], idx.shape)
        u[3, idx.reshape(-1) - 1] = 0.0
    return tree, u


def planar_expected(kind, level, tree, final):
    """(cells, expected uold[5, cells]) of level ``level`` from the 1D/2D
    leaves, constant along the missing axes, zero momenta along them."""
    nd = PLANAR[kind]["ndim"]
    g = _lowdim_grid(final, nd, level)
    idx = tree.cell_index(level)
    exp = np.zeros((5,) + idx.shape)
    if nd == 1:
        for v3, v1 in ((0, 0), (1, 1), (4, 2)):
            exp[v3] = g[None, None, :, v1]
    else:
        for v3, v2 in ((0, 0), (1, 1), (2, 2), (4, 3)):
            exp[v3] = g[None, :, :, v2]
    return idx.reshape(-1), exp.reshape(5, -1)
