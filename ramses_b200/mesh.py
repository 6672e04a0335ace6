"""Octree construction in RAMSES's own index conventions.

The hydro path consumes the tree arrays exactly as RAMSES lays them out
(``amr/amr_commons.f90:67-75``, ``amr/init_amr.f90:37-54,227-233``):

* ``ncoarse = nx*ny*nz`` coarse cells, then ``8*ngridmax`` oct cells;
  the cell of child slot ``ind`` (1..8) of oct ``igrid`` (1-based) is
  ``ncoarse + (ind-1)*ngridmax + igrid``; ``ind = 1 + ix + 2*iy + 4*iz``;
* ``son(icell)`` = the oct refining that cell, or 0;
* ``father(igrid)`` = the cell the oct refines;
* ``nbor(igrid, j)``, j = 1..6 for -x,+x,-y,+y,-z,+z = the cell adjacent
  to ``father(igrid)`` at the father's level (periodic box);
* ``active(ilevel)%igrid`` = the octs of level ``ilevel``.

Levels 1..levelmin are complete; finer levels follow a refinement map that is
closed under RAMSES's nesting rule (every refined cell's 3x3x3 neighbourhood
exists at its level), which is what ``get3cubefather``
(``amr/nbors_utils.f90:5-194``) relies on. Octs of each level are numbered in
creation order (parents in order, children in slot order), which for a
single-cell coarse grid is Morton order.

This module builds inputs; it performs no hydro arithmetic.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Optional, Sequence

import numpy as np

MAXLEVEL = 32


@dataclasses.dataclass
class Octree:
    nx: int
    ny: int
    nz: int
    ncoarse: int
    ngridmax: int
    nlevelmax: int
    levelmin: int
    boxlen: float
    son: np.ndarray          # int32 [ncell]
    father: np.ndarray       # int32 [ngridmax]
    nbor: np.ndarray         # int32 [6, ngridmax]  (Fortran nbor(ngridmax,6))
    active: list             # active[l] = int32 array of 1-based igrids, l=1..nlevelmax
    coords: list             # coords[l] = int64 (n,3) oct coordinates at level l
    # physical boundaries (hydro/read_hydro_params.f90:310-420): the coarse
    # grid carries one layer of boundary coarse cells per bounded side; their
    # octs are listed per boundary region, not in ``active``
    nx_loc: int = 0                      # icoarse_max-icoarse_min+1 (0: nx)
    offset: tuple = (0, 0, 0)            # (icoarse_min, jcoarse_min, kcoarse_min)
    boundary_type: list = dataclasses.field(default_factory=list)   # [nboundary] codes
    boundary: list = dataclasses.field(default_factory=list)        # [ib][l] int32 igrids
    bcoords: list = dataclasses.field(default_factory=list)         # [ib][l] (n,3) coords

    @property
    def ncell(self) -> int:
        return self.ncoarse + 8 * self.ngridmax

    @property
    def scale(self) -> float:
        """boxlen / nx_loc: the length of one coarse cell (amr/init_amr.f90:44)."""
        return self.boxlen / (self.nx_loc or self.nx)

    def boundary_concat(self):
        """(boundary_type int32[nb], off int64[nlevelmax*nb+1], igrid int32[])
        with the grids of (level l, region ib) at [off[k], off[k+1]),
        k = (l-1)*nb + ib (0-based ib)."""
        nb = len(self.boundary_type)
        off = np.zeros(self.nlevelmax * nb + 1, dtype=np.int64)
        parts = []
        for l in range(1, self.nlevelmax + 1):
            for ib in range(nb):
                g = self.boundary[ib][l] if l < len(self.boundary[ib]) else np.zeros(0, np.int32)
                k = (l - 1) * nb + ib
                off[k + 1] = off[k] + len(g)
                parts.append(g)
        cat = np.concatenate(parts) if parts else np.zeros(0, np.int32)
        return np.asarray(self.boundary_type, np.int32), off, cat.astype(np.int32)

    def boundary_octs(self, level: int):
        """(igrid int64[n], coords[n,3]) of the boundary octs of ``level``."""
        g = [self.boundary[ib][level] for ib in range(len(self.boundary)) if level < len(self.boundary[ib])]
        c = [self.bcoords[ib][level] for ib in range(len(self.bcoords)) if level < len(self.bcoords[ib])]
        if not g:
            return np.zeros(0, np.int64), np.zeros((0, 3), np.int64)
        return np.concatenate(g).astype(np.int64), np.concatenate(c)

    def noct(self, level: int) -> int:
        return len(self.active[level]) if level < len(self.active) else 0

    def active_concat(self):
        """(concatenated int32 list, int64 offsets[nlevelmax+2]) with level l's
        list at [off[l], off[l+1])."""
        off = np.zeros(self.nlevelmax + 2, dtype=np.int64)
        for l in range(1, self.nlevelmax + 1):
            off[l + 1] = off[l] + self.noct(l)
        cat = np.concatenate([self.active[l] for l in range(1, self.nlevelmax + 1)
                              if self.noct(l) > 0] or [np.zeros(0, np.int32)])
        return cat.astype(np.int32), off

    def leaf_cells(self, level: int) -> int:
        a = self.active[level]
        if len(a) == 0:
            return 0
        cells = self.ncoarse + np.arange(8)[:, None] * self.ngridmax + a[None, :]
        return int(np.count_nonzero(self.son[cells - 1] == 0))

    def cell_index(self, level: int, order: str = "C") -> np.ndarray:
        """1-based cell indices of level ``level`` arranged as a dense cube
        [z, y, x] (only valid for a complete level)."""
        n = 2 ** level
        a = self.active[level]
        c = self.coords[level] - np.asarray(self.offset, np.int64) * 2 ** (level - 1)
        if len(a) != (n // 2) ** 3:
            raise ValueError("level %d is not complete" % level)
        out = np.zeros((n, n, n), dtype=np.int64)
        for ind in range(8):
            ix, iy, iz = ind & 1, (ind >> 1) & 1, (ind >> 2) & 1
            cell = self.ncoarse + ind * self.ngridmax + a.astype(np.int64)
            out[2 * c[:, 2] + iz, 2 * c[:, 1] + iy, 2 * c[:, 0] + ix] = cell
        return out

    def cell_centres(self, level: int, boundary: bool = True):
        """(cells[1-based], x[n,3]) for every cell of the octs of ``level``
        (with ``boundary``, the boundary octs' cells too), x in user units
        measured from the box corner (init_flow_fine.f90's skip_loc)."""
        a = self.active[level].astype(np.int64)
        c = self.coords[level]
        if boundary and self.boundary:
            bg, bc = self.boundary_octs(level)
            a, c = np.concatenate([a, bg]), np.concatenate([c, bc])
        dx = self.scale * 0.5 ** level
        skip = np.asarray(self.offset, np.float64) * self.scale
        cells, xs = [], []
        for ind in range(8):
            off = np.array([ind & 1, (ind >> 1) & 1, (ind >> 2) & 1])
            cells.append(self.ncoarse + ind * self.ngridmax + a)
            xs.append((2 * c + off + 0.5) * dx - skip)
        return np.concatenate(cells), np.concatenate(xs)


def _keys(c: np.ndarray, n: int) -> np.ndarray:
    return c[:, 0] + n * (c[:, 1] + n * c[:, 2])


def _unique(x: np.ndarray) -> np.ndarray:
    """Sorted unique values (sort-based: much faster than numpy's hashing
    unique on large int64 key arrays)."""
    x = np.sort(np.asarray(x).ravel())
    if len(x) < 2:
        return x
    return x[np.concatenate(([True], x[1:] != x[:-1]))]


def _isin(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Boolean mask of the entries of ``a`` present in ``b`` (sort and
    binary search)."""
    a = np.asarray(a)
    bs = _unique(b)
    if len(bs) == 0:
        return np.zeros(a.shape, bool)
    pos = np.minimum(np.searchsorted(bs, a), len(bs) - 1)
    return bs[pos] == a


def _neighbourhood(cells: np.ndarray) -> np.ndarray:
    offs = np.array([[i, j, k] for k in (-1, 0, 1) for j in (-1, 0, 1) for i in (-1, 0, 1)])
    return (cells[:, None, :] + offs[None, :, :]).reshape(-1, 3)


def _dilated_keys(cells: np.ndarray, n: int) -> np.ndarray:
    """Sorted unique keys of the cells within one cell (26-neighbourhood,
    periodic in n) of ``cells``: three separable one-axis dilations, each
    followed by a unique (a third of the sorting work of the 27-point
    expansion)."""
    k = _unique(_keys(cells % n, n))
    for d in range(3):
        c = np.stack([k % n, (k // n) % n, k // (n * n)], 1)
        parts = []
        for s in (-1, 0, 1):
            cc = c.copy()
            cc[:, d] = (cc[:, d] + s) % n
            parts.append(_keys(cc, n))
        k = _unique(np.concatenate(parts))
    return k


def build_tree(levelmin: int, nlevelmax: Optional[int] = None,
               refine: Optional[Callable[[int, np.ndarray], np.ndarray]] = None,
               boxlen: float = 1.0, nexpand: int = 1, spare: int = 0) -> Octree:
    """Build a periodic single-coarse-cell (nx=ny=nz=1) octree.

    ``refine(level, cell_coords[n,3]) -> bool[n]`` flags level-``level``
    cells (level >= levelmin) for refinement; flags are expanded by
    ``nexpand`` cells and closed under the nesting rule. ``spare`` free
    grids are reserved beyond the octs built (ngridmax, room for
    ``remesh``).
    """
    return _assemble(oct_sets(levelmin, nlevelmax, refine, nexpand), levelmin, nlevelmax or levelmin, boxlen, spare)


def oct_sets(levelmin: int, nlevelmax: Optional[int] = None,
             refine: Optional[Callable[[int, np.ndarray], np.ndarray]] = None, nexpand: int = 1) -> dict:
    """The oct coordinates of every level (dict level -> (n, 3)) of the tree
    that ``build_tree`` assembles: ``refine`` flags, expanded by ``nexpand``
    cells, closed under the nesting rule."""
    if nlevelmax is None:
        nlevelmax = levelmin
    if not (1 <= levelmin <= nlevelmax <= MAXLEVEL - 1):
        raise ValueError("bad level range")
    # -- 1. refined cell sets per level, as integer coords (level-l units) --
    refined = {}
    cur_octs = np.zeros((1, 3), dtype=np.int64)   # level-1 oct(s)
    oct_coords = {1: cur_octs}
    for l in range(1, nlevelmax):
        n = 2 ** l
        octs = oct_coords[l]
        cells = (2 * octs[:, None, :] + np.array([[i & 1, (i >> 1) & 1, (i >> 2) & 1]
                                                   for i in range(8)])[None]).reshape(-1, 3)
        if l < levelmin:
            flag = np.ones(len(cells), dtype=bool)
        elif refine is None:
            flag = np.zeros(len(cells), dtype=bool)
        else:
            flag = np.asarray(refine(l, cells), dtype=bool)
        fc = cells[flag]
        for _ in range(nexpand if l >= levelmin else 0):
            if len(fc) == 0:
                break
            k = _dilated_keys(fc, n)
            ck = _keys(cells, n)
            fc = cells[_isin(ck, k)]
        refined[l] = fc
        oct_coords[l + 1] = fc.copy()
        if len(fc) == 0:
            for ll in range(l + 1, nlevelmax + 1):
                oct_coords.setdefault(ll, np.zeros((0, 3), np.int64))
            break
    for l in range(1, nlevelmax + 1):
        oct_coords.setdefault(l, np.zeros((0, 3), np.int64))
    # -- 2. closure under the nesting rule, finest to coarsest --
    for l in range(nlevelmax - 1, levelmin, -1):
        fc = refined.get(l, np.zeros((0, 3), np.int64))
        if len(fc) == 0:
            continue
        n = 2 ** l
        kd = _dilated_keys(fc, n)
        dc = np.stack([kd % n, (kd // n) % n, kd // (n * n)], 1)
        need = _unique(_keys(dc // 2, n // 2))
        have = _keys(refined[l - 1], n // 2)
        missing = need[~_isin(need, have)]
        if len(missing):
            nn = n // 2
            mc = np.stack([missing % nn, (missing // nn) % nn, missing // (nn * nn)], 1)
            refined[l - 1] = np.concatenate([refined[l - 1], mc])
    # recompute oct sets from the closed refinement sets, keeping only cells
    # whose own oct exists (parents refined)
    oct_coords = {1: np.zeros((1, 3), dtype=np.int64)}
    for l in range(1, nlevelmax):
        n = 2 ** l
        fc = refined.get(l, np.zeros((0, 3), np.int64))
        if len(fc) == 0:
            oct_coords[l + 1] = np.zeros((0, 3), np.int64)
            continue
        parent_keys = _keys(oct_coords[l], n // 2)
        fc = fc[_isin(_keys(fc // 2, n // 2), parent_keys)]
        refined[l] = fc
        oct_coords[l + 1] = fc
    return oct_coords


def flag_refine(tree: "Octree", flag1: np.ndarray) -> Callable[[int, np.ndarray], np.ndarray]:
    """A ``refine`` callback for ``oct_sets`` from per-cell flags of a tree
    (flag1[icell], icell the Fortran cell index, as hydro_flag sets them):
    a level-l cell is flagged when it is a cell of the tree and flagged, or
    when it is refined and one of its children is (so that refined regions
    shrink only from their finest level, one level per remesh)."""
    lookups = {}
    for l in range(1, tree.nlevelmax + 1):
        if tree.noct(l) == 0:
            continue
        n = 2 ** (l - 1)
        k = _keys(tree.coords[l], n)
        srt = np.argsort(k)
        lookups[l] = (k[srt], np.asarray(tree.active[l], np.int64)[srt])

    def cells_of(level, cells):
        """Fortran cell indices of level-``level`` cells (0 where absent)."""
        if level not in lookups:
            return np.zeros(len(cells), np.int64)
        ks, ig = lookups[level]
        n = 2 ** (level - 1)
        k = _keys(cells // 2, n)
        pos = np.minimum(np.searchsorted(ks, k), len(ks) - 1)
        ok = ks[pos] == k
        ind = (cells[:, 0] & 1) + 2 * (cells[:, 1] & 1) + 4 * (cells[:, 2] & 1)
        return np.where(ok, tree.ncoarse + ind * tree.ngridmax + ig[pos], 0)

    def refine(level, cells):
        c = cells_of(level, cells)
        have = c > 0
        flag = np.zeros(len(cells), bool)
        flag[have] = flag1[c[have]] != 0
        if level + 1 <= tree.nlevelmax:
            son = np.zeros(len(cells), np.int64)
            son[have] = tree.son[c[have] - 1]
            kids = son > 0
            if kids.any():
                g = son[kids]
                sub = np.zeros(len(g), bool)
                for ind in range(8):
                    sub |= tree.son[tree.ncoarse + ind * tree.ngridmax + g - 1] > 0
                flag[np.nonzero(kids)[0][sub]] = True
        return flag
    return refine


def _assemble(oct_coords, levelmin, nlevelmax, boxlen, spare=0) -> Octree:
    ncoarse = 1
    counts = [len(oct_coords.get(l, ())) for l in range(1, nlevelmax + 1)]
    ngridmax = int(sum(counts)) + int(spare)
    ncell = ncoarse + 8 * ngridmax
    son = np.zeros(ncell, dtype=np.int32)
    father = np.zeros(ngridmax, dtype=np.int32)
    nbor = np.zeros((6, ngridmax), dtype=np.int32)
    active = [np.zeros(0, np.int32) for _ in range(nlevelmax + 1)]
    coords = [np.zeros((0, 3), np.int64) for _ in range(nlevelmax + 1)]
    # order: level by level; within a level, by (parent igrid, child slot)
    g0 = 0
    parent_lookup = None   # (sorted keys, igrid) for level l-1 octs
    for l in range(1, nlevelmax + 1):
        oc = oct_coords.get(l, np.zeros((0, 3), np.int64))
        n_oct = len(oc)
        if n_oct == 0:
            break
        if l == 1:
            order = np.arange(n_oct)
        else:
            # parent oct at level l-1 and slot of the father cell
            pk = _keys(oc // 2, 2 ** (l - 2))
            keys_sorted, igr = parent_lookup
            pos = np.searchsorted(keys_sorted, pk)
            pg = igr[pos]
            slot = (oc[:, 0] & 1) + 2 * (oc[:, 1] & 1) + 4 * (oc[:, 2] & 1)
            order = np.lexsort((slot, pg))
        oc = oc[order]
        ig = np.arange(g0 + 1, g0 + 1 + n_oct, dtype=np.int64)
        active[l] = ig.astype(np.int32)
        coords[l] = oc
        # father cells and neighbour father cells
        if l == 1:
            father[ig - 1] = 1
            nbor[:, ig - 1] = 1
            son[0] = int(ig[0])
        else:
            keys_sorted, igr = parent_lookup
            nl = 2 ** (l - 1)  # cells per dim at level l-1

            def cell_of(cc):
                cc = cc % nl
                k = _keys(cc // 2, nl // 2)
                pos = np.searchsorted(keys_sorted, k)
                if np.any(pos >= len(keys_sorted)) or np.any(keys_sorted[np.minimum(pos, len(keys_sorted) - 1)] != k):
                    raise ValueError("refinement map violates the nesting rule at level %d" % l)
                slot = (cc[:, 0] & 1) + 2 * (cc[:, 1] & 1) + 4 * (cc[:, 2] & 1)
                return ncoarse + slot * ngridmax + igr[pos]

            fcell = cell_of(oc)
            father[ig - 1] = fcell
            son[fcell - 1] = ig
            for j in range(6):
                d = j // 2
                step = np.zeros(3, np.int64)
                step[d] = 1 if (j % 2) else -1
                nbor[j, ig - 1] = cell_of(oc + step)
        k = _keys(oc, 2 ** (l - 1))
        srt = np.argsort(k)
        parent_lookup = (k[srt], ig[srt])
        g0 += n_oct
    return Octree(nx=1, ny=1, nz=1, ncoarse=ncoarse, ngridmax=ngridmax,
                  nlevelmax=nlevelmax, levelmin=levelmin, boxlen=float(boxlen),
                  son=son, father=father, nbor=nbor, active=active, coords=coords)


def remesh(old: Octree, oct_coords) -> Octree:
    """The tree that refine_fine leaves behind (amr/refine_utils.f90:332-948)
    when the octs of level l become ``oct_coords[l]`` (n,3 oct coordinates):
    an oct present before and after keeps its igrid and its place in the
    level's active list; killed octs free their igrids (kill_grid); new octs
    take free igrids in ascending order and are appended to the list in
    (parent igrid, child slot) order (make_grid_fine). ngridmax and the cell
    numbering are unchanged, so the old tree needs spare grids
    (``build_tree(spare=...)``). Single-coarse-cell periodic trees."""
    if old.ncoarse != 1 or old.boundary_type:
        raise ValueError("remesh: single-coarse-cell periodic trees only")
    L = old.nlevelmax
    ngm, ncoarse = old.ngridmax, old.ncoarse
    new_sets = [np.zeros((0, 3), np.int64)] + [np.asarray(oct_coords.get(l, np.zeros((0, 3), np.int64)),
                                                          np.int64).reshape(-1, 3) for l in range(1, L + 1)]
    keep = {}          # level -> (bool mask over the old active list)
    used = np.zeros(ngm + 1, bool)
    for l in range(1, L + 1):
        if old.noct(l) == 0:
            keep[l] = np.zeros(0, bool)
            continue
        n = 2 ** (l - 1)
        k_old = _keys(old.coords[l], n)
        k_new = _keys(new_sets[l], n) if len(new_sets[l]) else np.zeros(0, np.int64)
        keep[l] = _isin(k_old, k_new)
        used[old.active[l][keep[l]]] = True
    free = np.nonzero(~used[1:])[0] + 1
    fi = 0
    son = np.zeros(ncoarse + 8 * ngm, np.int32)
    father = np.zeros(ngm, np.int32)
    nbor = np.zeros((6, ngm), np.int32)
    active = [np.zeros(0, np.int32) for _ in range(L + 1)]
    coords = [np.zeros((0, 3), np.int64) for _ in range(L + 1)]
    parent_lookup = None
    for l in range(1, L + 1):
        oc_new = new_sets[l]
        if len(oc_new) == 0:
            break
        n = 2 ** (l - 1)
        surv_g = old.active[l][keep[l]] if old.noct(l) else np.zeros(0, np.int32)
        surv_c = old.coords[l][keep[l]] if old.noct(l) else np.zeros((0, 3), np.int64)
        k_surv = _keys(surv_c, n) if len(surv_c) else np.zeros(0, np.int64)
        born = oc_new[~_isin(_keys(oc_new, n), k_surv)]
        if l > 1 and len(born):
            keys_sorted, igr = parent_lookup
            pos = np.searchsorted(keys_sorted, _keys(born // 2, 2 ** (l - 2)))
            slot = (born[:, 0] & 1) + 2 * (born[:, 1] & 1) + 4 * (born[:, 2] & 1)
            born = born[np.lexsort((slot, igr[pos]))]
        if fi + len(born) > len(free):
            raise ValueError("remesh: ngridmax=%d too small" % ngm)
        born_g = free[fi:fi + len(born)].astype(np.int64)
        fi += len(born)
        ig = np.concatenate([surv_g.astype(np.int64), born_g])
        oc = np.concatenate([surv_c, born]) if len(born) else surv_c
        active[l] = ig.astype(np.int32)
        coords[l] = oc
        if l == 1:
            father[ig - 1] = 1
            nbor[:, ig - 1] = 1
            son[0] = int(ig[0])
        else:
            keys_sorted, igr = parent_lookup
            nl = 2 ** (l - 1)

            def cell_of(cc):
                cc = cc % nl
                k = _keys(cc // 2, nl // 2)
                pos = np.searchsorted(keys_sorted, k)
                if np.any(pos >= len(keys_sorted)) or np.any(keys_sorted[np.minimum(pos, len(keys_sorted) - 1)] != k):
                    raise ValueError("remesh: refinement map violates the nesting rule at level %d" % l)
                slot = (cc[:, 0] & 1) + 2 * (cc[:, 1] & 1) + 4 * (cc[:, 2] & 1)
                return ncoarse + slot * ngm + igr[pos]

            fcell = cell_of(oc)
            father[ig - 1] = fcell
            son[fcell - 1] = ig
            for j in range(6):
                step = np.zeros(3, np.int64)
                step[j // 2] = 1 if (j % 2) else -1
                nbor[j, ig - 1] = cell_of(oc + step)
        k = _keys(oc, n)
        srt = np.argsort(k)
        parent_lookup = (k[srt], ig[srt])
    return Octree(nx=1, ny=1, nz=1, ncoarse=ncoarse, ngridmax=ngm, nlevelmax=L, levelmin=old.levelmin,
                  boxlen=old.boxlen, son=son, father=father, nbor=nbor, active=active, coords=coords)


def refine_from_flags(old: Octree, flag1: np.ndarray, nexpand: int = 1) -> Octree:
    """The host's remesh from cell flags (flag_fine -> refine_fine): the
    flagged cells of every level from levelmin (flag1[icell], Fortran cell
    index, as hydro_flag sets them) are refined, expanded by ``nexpand``
    cells and closed under the nesting rule (``oct_sets``); refined regions
    shrink from their finest level; the new tree keeps the igrids of the
    octs that survive (``remesh``)."""
    sets = oct_sets(old.levelmin, old.nlevelmax, flag_refine(old, np.asarray(flag1)), nexpand)
    return remesh(old, sets)


def uniform_tree(level: int, boxlen: float = 1.0) -> Octree:
    """Complete periodic grid of (2**level)^3 leaf cells (levelmin=levelmax)."""
    return build_tree(level, level, None, boxlen)


def gradient_refine(field_fn: Callable[[np.ndarray], Sequence[np.ndarray]],
                    thresholds: Sequence[float], boxlen: float = 1.0,
                    floor: float = 1e-10) -> Callable[[int, np.ndarray], np.ndarray]:
    """Refinement flags from RAMSES's relative-gradient criterion
    (``hydro/godunov_utils.f90:125-263``, ``err_grad_*``) evaluated on an
    analytic field at level-``l`` cell centres: a cell is flagged when
    ``|f(i+1)-f(i-1)| / (|f(i+1)|+|f(i)|+|f(i-1)|+floor)`` exceeds the
    threshold in any direction for any field."""
    def refine(level: int, cells: np.ndarray) -> np.ndarray:
        dx = boxlen * 0.5 ** level
        x0 = (cells + 0.5) * dx
        flag = np.zeros(len(cells), dtype=bool)
        f0 = field_fn(x0 % boxlen)
        for d in range(3):
            e = np.zeros(3)
            e[d] = dx
            fp = field_fn((x0 + e) % boxlen)
            fm = field_fn((x0 - e) % boxlen)
            for a, b, c, thr in zip(fm, f0, fp, thresholds):
                if thr <= 0:
                    continue
                err = np.abs(c - a) / (np.abs(c) + np.abs(b) + np.abs(a) + floor)
                flag |= err > thr
        return flag
    return refine


def sphere_refine(centre, radius: float, boxlen: float = 1.0, pad_cells: float = 2.0
                  ) -> Callable[[int, np.ndarray], np.ndarray]:
    """Geometric refinement: flag level-``l`` cells whose centre lies within
    ``radius + pad_cells*dx_l`` of ``centre`` (periodic distance)."""
    c = np.asarray(centre, dtype=np.float64) * boxlen

    def refine(level: int, cells: np.ndarray) -> np.ndarray:
        dx = boxlen * 0.5 ** level
        x = (cells + 0.5) * dx
        d = np.abs(x - c)
        d = np.minimum(d, boxlen - d)
        return np.sqrt(np.sum(d * d, axis=1)) < radius + pad_cells * dx
    return refine


def shell_refine(centre, radius: float, width_cells: float = 4.0, boxlen: float = 1.0
                 ) -> Callable[[int, np.ndarray], np.ndarray]:
    """Geometric refinement: flag level-``l`` cells whose centre lies within
    ``width_cells*dx_l`` of the sphere of ``radius`` around ``centre``
    (periodic distance): a static stand-in for refinement that follows a
    spherical shock."""
    c = np.asarray(centre, dtype=np.float64) * boxlen

    def refine(level: int, cells: np.ndarray) -> np.ndarray:
        dx = boxlen * 0.5 ** level
        x = (cells + 0.5) * dx
        d = np.abs(x - c)
        d = np.minimum(d, boxlen - d)
        return np.abs(np.sqrt(np.sum(d * d, axis=1)) - radius) < width_cells * dx
    return refine


def union_refine(*fns) -> Callable[[int, np.ndarray], np.ndarray]:
    def refine(level: int, cells: np.ndarray) -> np.ndarray:
        out = np.zeros(len(cells), dtype=bool)
        for f in fns:
            out |= f(level, cells)
        return out
    return refine


# RAMSES boundary_type codes (hydro/read_hydro_params.f90:355-410): side
# 1..6 = -x,+x,-y,+y,-z,+z; + 0 for walls (bound_type 1), + 10 for free
# (zero-gradient, bound_type 2) boundaries.
BOUND_KINDS = {"reflexive": 0, "outflow": 10}


def add_boundaries(tree: Octree, bounds: Sequence[Optional[str]]) -> Octree:
    """Embed a single-coarse-cell tree (``build_tree``) in RAMSES's extended
    coarse grid with physical boundaries: per axis, ``bounds[d]`` is None
    (periodic) or "outflow" / "reflexive" on both sides, which adds one
    boundary coarse cell per side (nx = 3 for a bounded x). The boundary
    coarse cells are refined down to levelmin like every coarse cell
    (amr/refine_utils.f90:86-95); they hold no finer octs, so refinement
    must stay clear of the box faces (the nesting check below fails
    otherwise). Boundary regions are ordered -x, +x, -y, +y, -z, +z over the
    bounded axes; a region spans the coarse cells of its side over the full
    extent of the axes before it and the interior of the axes after it, as
    the usual &BOUNDARY_PARAMS do: the later regions cover the edges and
    corners, whose reference grids then lie in regions filled before."""
    if tree.nx != 1 or tree.ny != 1 or tree.nz != 1 or tree.boundary:
        raise ValueError("add_boundaries takes a single-coarse-cell periodic tree")
    b = [1 if bounds[d] else 0 for d in range(3)]
    for d in range(3):
        if bounds[d] and bounds[d] not in BOUND_KINDS:
            raise ValueError("unknown boundary kind %r" % bounds[d])
    ext = np.array([1 + 2 * b[0], 1 + 2 * b[1], 1 + 2 * b[2]], np.int64)
    lmin, lmax = tree.levelmin, tree.nlevelmax
    regions = []  # (type, axis, side)
    for d in range(3):
        if b[d]:
            for side in (0, 1):
                regions.append((BOUND_KINDS[bounds[d]] + 2 * d + side + 1, d, side))
    # oct sets per level in extended coordinates, tagged -1 (interior) or region
    sets = {}
    for l in range(1, lmax + 1):
        h = 2 ** (l - 1)  # octs per coarse cell along an axis
        inner = tree.coords[l] + np.asarray(b, np.int64) * h if tree.noct(l) else np.zeros((0, 3), np.int64)
        tags = [np.full(len(inner), -1, np.int64)]
        allc = [inner]
        if l <= lmin:
            g = np.stack(np.meshgrid(np.arange(ext[0] * h), np.arange(ext[1] * h), np.arange(ext[2] * h),
                                     indexing="ij"), -1).reshape(-1, 3)
            cc = g // h  # coarse cell of each oct
            interior = np.ones(len(g), bool)
            for d in range(3):
                if b[d]:
                    interior &= (cc[:, d] >= 1) & (cc[:, d] <= ext[d] - 2)
            g, cc = g[~interior], cc[~interior]
            tag = np.full(len(g), -2, np.int64)
            for ir, (_, d, side) in enumerate(regions):
                on = cc[:, d] == (0 if side == 0 else ext[d] - 1)
                for d2 in range(d + 1, 3):  # interior of the axes after this one
                    if b[d2]:
                        on &= (cc[:, d2] >= 1) & (cc[:, d2] <= ext[d2] - 2)
                tag[(tag == -2) & on] = ir
            assert np.all(tag >= 0)
            allc.append(g)
            tags.append(tag)
        sets[l] = (np.concatenate(allc), np.concatenate(tags))
    return _assemble_ext(sets, ext, b, regions, lmin, lmax, tree.boxlen)


def _assemble_ext(sets, ext, b, regions, levelmin, nlevelmax, boxlen) -> Octree:
    nx, ny, nz = (int(e) for e in ext)
    ncoarse = nx * ny * nz
    ngridmax = int(sum(len(sets[l][0]) for l in sets))
    son = np.zeros(ncoarse + 8 * ngridmax, dtype=np.int32)
    father = np.zeros(ngridmax, dtype=np.int32)
    nbor = np.zeros((6, ngridmax), dtype=np.int32)
    active = [np.zeros(0, np.int32) for _ in range(nlevelmax + 1)]
    coords = [np.zeros((0, 3), np.int64) for _ in range(nlevelmax + 1)]
    bnd = [[np.zeros(0, np.int32) for _ in range(nlevelmax + 1)] for _ in regions]
    bco = [[np.zeros((0, 3), np.int64) for _ in range(nlevelmax + 1)] for _ in regions]

    def key(c, l):
        X, Y = nx * 2 ** (l - 1), ny * 2 ** (l - 1)
        return c[:, 0] + X * (c[:, 1] + Y * c[:, 2])

    g0 = 0
    lookup = None  # level l-1: (sorted keys, igrid)
    for l in range(1, nlevelmax + 1):
        oc, tag = sets.get(l, (np.zeros((0, 3), np.int64), np.zeros(0, np.int64)))
        if len(oc) == 0:
            break
        E = ext * 2 ** (l - 1)  # octs per axis at level l; cells at level l-1
        if l == 1:
            order = np.lexsort((oc[:, 0], oc[:, 1], oc[:, 2]))
        else:
            ks, igr = lookup
            pos = np.searchsorted(ks, key(oc // 2, l - 1))
            pg = igr[pos]
            slot = (oc[:, 0] & 1) + 2 * (oc[:, 1] & 1) + 4 * (oc[:, 2] & 1)
            order = np.lexsort((slot, pg))
        oc, tag = oc[order], tag[order]
        ig = np.arange(g0 + 1, g0 + 1 + len(oc), dtype=np.int64)

        def cell_of(cc):
            cc = cc % E
            if l == 1:
                return 1 + cc[:, 0] + nx * (cc[:, 1] + ny * cc[:, 2])
            ks, igr = lookup
            k = key(cc // 2, l - 1)
            pos = np.searchsorted(ks, k)
            if np.any(pos >= len(ks)) or np.any(ks[np.minimum(pos, len(ks) - 1)] != k):
                raise ValueError("refinement reaches the boundary layer at level %d "
                                 "(no boundary octs below levelmin)" % l)
            slot = (cc[:, 0] & 1) + 2 * (cc[:, 1] & 1) + 4 * (cc[:, 2] & 1)
            return ncoarse + slot * ngridmax + igr[pos]

        fc = cell_of(oc)
        father[ig - 1] = fc
        son[fc - 1] = ig
        for j in range(6):
            step = np.zeros(3, np.int64)
            step[j // 2] = 1 if (j % 2) else -1
            nbor[j, ig - 1] = cell_of(oc + step)
        active[l] = ig[tag == -1].astype(np.int32)
        coords[l] = oc[tag == -1]
        for ir in range(len(regions)):
            bnd[ir][l] = ig[tag == ir].astype(np.int32)
            bco[ir][l] = oc[tag == ir]
        k = key(oc, l)
        srt = np.argsort(k)
        lookup = (k[srt], ig[srt])
        g0 += len(oc)
    return Octree(nx=nx, ny=ny, nz=nz, ncoarse=ncoarse, ngridmax=ngridmax, nlevelmax=nlevelmax,
                  levelmin=levelmin, boxlen=float(boxlen), son=son, father=father, nbor=nbor,
                  active=active, coords=coords, nx_loc=1, offset=tuple(b),
                  boundary_type=[r[0] for r in regions], boundary=bnd, bcoords=bco)
