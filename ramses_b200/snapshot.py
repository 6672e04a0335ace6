"""Snapshots in RAMSES's own output format, written from a device download.

``write_snapshot`` writes the directory ``output_NNNNN`` that RAMSES's
``dump_all`` produces for a one-rank pure-hydro run, so that RAMSES's own
tools read it:

* ``amr_NNNNN.out00001``: ``backup_amr`` (``amr/output_amr.f90:5-206``), the
  header records, the coarse ``son``/``flag1``/``cpu_map`` and, per level and
  domain (the rank, then the boundary regions), the grids' linked-list
  indices, ``xg``, ``father``, ``nbor``, ``son``, ``cpu_map`` and ``flag1``;
* ``hydro_NNNNN.out00001``: ``backup_hydro`` (``hydro/output_hydro.f90:1-179``),
  per level and domain the density, velocities and thermal pressure of every
  cell slot, formed as the reference forms them;
* ``hydro_file_descriptor.txt`` (``io/dump_utils.f90:118-139``),
  ``info_NNNNN.txt`` (``output_info``, ``amr/output_amr.f90:411-491``) and
  ``header_NNNNN.txt`` (``output_header``, ``:496-575``, no particles).

All files are Fortran unformatted sequential records (a 4-byte length before
and after each record), little-endian. The grids of a level are listed in the
order of the host's active list; the free list is the unused grids in
ascending order. ``read_snapshot`` parses the records back (independently of
the offsets' arithmetic that RAMSES's readers use).
"""
from __future__ import annotations

import struct
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

from .mesh import Octree


class _Records:
    def __init__(self, f):
        self.f = f

    def raw(self, payload: bytes):
        n = struct.pack("<i", len(payload))
        self.f.write(n + payload + n)

    def ints(self, a):
        self.raw(np.ascontiguousarray(a, "<i4").tobytes())

    def reals(self, a):
        self.raw(np.ascontiguousarray(a, "<f8").tobytes())


def _fortran_e(x: float, w: int = 23, d: int = 15) -> str:
    """Fortran ``Ew.d`` (mantissa in [0.1, 1), two- or three-digit exponent)."""
    if x == 0.0 or not np.isfinite(x):
        s = ("0." + "0" * d + "E+00") if x == 0.0 else repr(x)
        return s.rjust(w)
    m, e = "%.*e" % (d - 1, abs(x)), 0
    digits, exp = m.split("e")
    digits = digits.replace(".", "")
    e = int(exp) + 1
    es = "E%+03d" % e if abs(e) < 100 else "%+04d" % e
    s = ("-" if x < 0 else "") + "0." + digits + es
    return s.rjust(w)


def _level_lists(tree: Octree, level: int):
    """Domains of one level: the active list, then each boundary region."""
    doms = [np.asarray(tree.active[level], np.int64) if level < len(tree.active) else np.zeros(0, np.int64)]
    for ib in range(len(tree.boundary_type)):
        b = tree.boundary[ib]
        doms.append(np.asarray(b[level], np.int64) if level < len(b) else np.zeros(0, np.int64))
    return doms


def _xg(tree: Octree):
    """Oct centres in coarse-cell units from the corner of the coarse grid
    (RAMSES's xg), per grid (ngridmax, 3); zero for unused grids."""
    xg = np.zeros((tree.ngridmax, 3))
    for l in range(1, tree.nlevelmax + 1):
        if l < len(tree.active) and len(tree.active[l]):
            g = np.asarray(tree.active[l], np.int64)
            xg[g - 1] = (np.asarray(tree.coords[l], np.float64) + 0.5) * 0.5 ** (l - 1)
        for ib in range(len(tree.boundary_type)):
            if l < len(tree.boundary[ib]) and len(tree.boundary[ib][l]):
                g = np.asarray(tree.boundary[ib][l], np.int64)
                xg[g - 1] = (np.asarray(tree.bcoords[ib][l], np.float64) + 0.5) * 0.5 ** (l - 1)
    return xg


def hydro_variables(u: np.ndarray, gamma: float, smallr: float) -> np.ndarray:
    """(5, n) conservative -> density, velocity_x/y/z, pressure as
    backup_hydro writes them (hydro/output_hydro.f90:84-120)."""
    rho = u[0]
    den = np.maximum(rho, smallr)
    out = np.empty_like(u)
    out[0] = rho
    out[1] = u[1] / den
    out[2] = u[2] / den
    out[3] = u[3] / den
    p = u[4]
    p = p - 0.5 * u[1] ** 2 / den
    p = p - 0.5 * u[2] ** 2 / den
    p = p - 0.5 * u[3] ** 2 / den
    out[4] = (gamma - 1.0) * p
    return out


def write_snapshot(outdir, nout: int, tree: Octree, uold: np.ndarray, gamma: float, smallr: float = 1e-10,
                   t: float = 0.0, dtold: Optional[Sequence[float]] = None, dtnew: Optional[Sequence[float]] = None,
                   nstep: int = 0, nstep_coarse: int = 0, flag1: Optional[np.ndarray] = None) -> Path:
    """Write ``outdir/output_NNNNN`` (one rank, hilbert ordering) from the
    Fortran-layout ``uold`` (5, ncell) of ``tree``; returns the directory."""
    number = "%05d" % nout
    d = Path(outdir) / ("output_" + number)
    d.mkdir(parents=True, exist_ok=True)
    L = tree.nlevelmax
    nb = len(tree.boundary_type)
    ngm, ncoarse = tree.ngridmax, tree.ncoarse
    dtold = np.zeros(L) if dtold is None else np.asarray(dtold, np.float64)[:L]
    dtnew = np.zeros(L) if dtnew is None else np.asarray(dtnew, np.float64)[:L]
    flag1 = np.zeros(tree.ncell, np.int32) if flag1 is None else np.asarray(flag1, np.int32)
    lists = [_level_lists(tree, l) for l in range(1, L + 1)]
    used = np.zeros(ngm + 1, bool)
    for doms in lists:
        for g in doms:
            used[g] = True
    free = np.nonzero(~used[1:])[0] + 1
    ngrid_current = int(used[1:].sum())
    nxt = np.zeros(ngm, np.int32)
    prv = np.zeros(ngm, np.int32)
    heads = np.zeros((L, 1 + nb), np.int32)
    tails = np.zeros((L, 1 + nb), np.int32)
    counts = np.zeros((L, 1 + nb), np.int32)
    for l, doms in enumerate(lists):
        for j, g in enumerate(doms):
            if len(g) == 0:
                continue
            heads[l, j], tails[l, j], counts[l, j] = g[0], g[-1], len(g)
            nxt[g[:-1] - 1] = g[1:]
            prv[g[1:] - 1] = g[:-1]
    xg = _xg(tree)
    nbor = np.asarray(tree.nbor, np.int32)           # (6, ngridmax)
    son = np.asarray(tree.son, np.int32)
    cpu_map = np.ones(tree.ncell, np.int32)
    with open(d / ("amr_%s.out00001" % number), "wb") as f:
        r = _Records(f)
        r.ints([1])                                   # ncpu
        r.ints([3])                                   # ndim
        r.ints([tree.nx, tree.ny, tree.nz])
        r.ints([L])
        r.ints([ngm])
        r.ints([nb])
        r.ints([ngrid_current])
        r.reals([tree.boxlen])
        r.ints([1, 1, 1])                             # noutput, iout, ifout
        r.reals([t])                                  # tout(1:noutput)
        r.reals([1.0])                                # aout
        r.reals([t])
        r.reals(dtold)
        r.reals(dtnew)
        r.ints([nstep, nstep_coarse])
        r.reals([0.0, 0.0, 0.0])                      # einit, mass_tot_0, rho_tot
        r.reals([1.0, 0.0, 0.0, 0.0, 1.0, 1.0, tree.boxlen])   # omega_m,l,k,b, h0, aexp_ini, boxlen_ini
        r.reals([1.0, 0.0, 1.0, 0.0, 0.0])            # aexp, hexp, aexp_old, epot_tot_int, epot_tot_old
        r.reals([0.0])                                # mass_sph
        r.ints(heads[:, 0])                           # headl(1:ncpu,1:nlevelmax)
        r.ints(tails[:, 0])
        r.ints(counts[:, 0])
        numbtot = np.zeros((L, 10), np.int32)
        numbtot[:, 0] = counts[:, 0]                  # total, min, max, mean over the ranks
        numbtot[:, 1] = counts[:, 0]
        numbtot[:, 2] = counts[:, 0]
        numbtot[:, 3] = counts[:, 0]
        r.ints(numbtot)                               # numbtot(1:10,1:nlevelmax)
        if nb:
            r.ints(heads[:, 1:])                      # headb(1:nboundary,1:nlevelmax)
            r.ints(tails[:, 1:])
            r.ints(counts[:, 1:])
        headf = int(free[0]) if len(free) else 0
        tailf = int(free[-1]) if len(free) else 0
        r.ints([headf, tailf, len(free), ngrid_current, ngrid_current])
        r.raw("hilbert".ljust(128).encode())          # ordering
        r.reals([0.0, float(8 ** L)])                 # bound_key(0:ndomain)
        r.ints(son[:ncoarse])
        r.ints(flag1[:ncoarse])
        r.ints(cpu_map[:ncoarse])
        for l, doms in enumerate(lists):
            for g in doms:
                if len(g) == 0:
                    continue
                gi = g - 1
                r.ints(g)
                r.ints(nxt[gi])
                r.ints(prv[gi])
                for idim in range(3):
                    r.reals(xg[gi, idim])
                r.ints(tree.father[gi])
                for j in range(6):
                    r.ints(nbor[j, gi])
                cell = [ncoarse + ind * ngm + gi for ind in range(8)]
                for ind in range(8):
                    r.ints(son[cell[ind]])
                for ind in range(8):
                    r.ints(cpu_map[cell[ind]])
                for ind in range(8):
                    r.ints(flag1[cell[ind]])
    names = ["density", "velocity_x", "velocity_y", "velocity_z", "pressure"]
    with open(d / ("hydro_%s.out00001" % number), "wb") as f:
        r = _Records(f)
        r.ints([1])
        r.ints([5])
        r.ints([3])
        r.ints([L])
        r.ints([nb])
        r.reals([gamma])
        for l, doms in enumerate(lists):
            for g in doms:
                r.ints([l + 1])
                r.ints([len(g)])
                if len(g) == 0:
                    continue
                for ind in range(8):
                    cells = ncoarse + ind * ngm + (g - 1)
                    hv = hydro_variables(uold[:, cells], gamma, smallr)
                    for v in range(5):
                        r.reals(hv[v])
    with open(d / "hydro_file_descriptor.txt", "w") as f:
        f.write("# version: %2d\n" % 1)
        f.write("# ivar, variable_name, variable_type\n")
        for i, nm in enumerate(names):
            f.write("%2d, %s, %s\n" % (i + 1, nm, "d"))
    nx_loc = tree.nx_loc or tree.nx
    with open(d / ("info_%s.txt" % number), "w") as f:
        for k, v in (("ncpu", 1), ("ndim", 3), ("levelmin", tree.levelmin), ("levelmax", L), ("ngridmax", ngm),
                     ("nstep_coarse", nstep_coarse)):
            f.write("%-12s=%11d\n" % (k, v))
        f.write("\n")
        # output_info writes boxlen/nx_loc: the length of one coarse cell,
        # the unit of xg
        for k, v in (("boxlen", tree.boxlen / nx_loc), ("time", t), ("aexp", 1.0), ("H0", 1.0),
                     ("omega_m", 1.0), ("omega_l", 0.0), ("omega_k", 0.0), ("omega_b", 0.0), ("unit_l", 1.0),
                     ("unit_d", 1.0), ("unit_t", 1.0)):
            f.write("%-12s=%s\n" % (k, _fortran_e(float(v))))
        f.write("\n")
        f.write("ordering type=%-80s\n" % "hilbert")
        f.write("   DOMAIN   ind_min                 ind_max\n")
        f.write("%8d %s %s\n" % (1, _fortran_e(0.0), _fortran_e(float(8 ** L))))
    with open(d / ("header_%s.txt" % number), "w") as f:
        f.write("#%12s%10s\n" % ("Family", "Count"))
        f.write("%13s%10d\n" % ("undefined", 0))
        f.write(" Particle fields\n")
        f.write("pos vel mass iord level family tag \n")
    return d


def _read_records(path):
    data = Path(path).read_bytes()
    out, i = [], 0
    while i < len(data):
        n = struct.unpack_from("<i", data, i)[0]
        out.append(data[i + 4:i + 4 + n])
        if struct.unpack_from("<i", data, i + 4 + n)[0] != n:
            raise ValueError("%s: record markers differ at byte %d" % (path, i))
        i += 8 + n
    return out


def read_snapshot(outdir, nout: int) -> dict:
    """Leaf cells of a snapshot: arrays level, x, y, z, dx (box units) and
    the hydro variables named by the descriptor."""
    number = "%05d" % nout
    d = Path(outdir) / ("output_" + number)
    amr = _read_records(d / ("amr_%s.out00001" % number))
    hyd = _read_records(d / ("hydro_%s.out00001" % number))
    i4 = lambda b: np.frombuffer(b, "<i4")   # noqa: E731
    f8 = lambda b: np.frombuffer(b, "<f8")   # noqa: E731
    ncpu, ndim = int(i4(amr[0])[0]), int(i4(amr[1])[0])
    nx, ny, nz = (int(v) for v in i4(amr[2]))
    L, nb = int(i4(amr[3])[0]), int(i4(amr[5])[0])
    # positions are in coarse cells; the info file's boxlen is one coarse cell
    boxlen = None
    for ln in (d / ("info_%s.txt" % number)).read_text().splitlines():
        if ln.split("=")[0].strip() == "boxlen":
            boxlen = float(ln.split("=")[1].replace("D", "E"))
    if ncpu != 1 or ndim != 3:
        raise ValueError("one-rank 3D snapshots only")
    k = 19                                            # headl, after mass_sph
    numbl = i4(amr[k + 2]).reshape(L, ncpu)
    k += 4                                            # headl, taill, numbl, numbtot
    numbb = np.zeros((L, nb), np.int32)
    if nb:
        numbb = i4(amr[k + 2]).reshape(L, nb)
        k += 3
    k += 1 + 1 + 1 + 3                                # free list, ordering, bound_key, son/flag1/cpu_map
    names = [ln.split(",")[1].strip() for ln in (d / "hydro_file_descriptor.txt").read_text().splitlines()
             if not ln.startswith("#")]
    nvar = int(i4(hyd[1])[0])
    h = 6
    xbound = np.array([nx // 2, ny // 2, nz // 2], np.float64)
    out = {n: [] for n in ["level", "x", "y", "z", "dx"] + names}
    for l in range(1, L + 1):
        dxc = 0.5 ** l
        for dom in range(ncpu + nb):
            ncache = int(numbl[l - 1, dom]) if dom < ncpu else int(numbb[l - 1, dom - ncpu])
            h += 2
            if ncache == 0:
                continue
            recs = amr[k:k + 4 + 3 * ndim + 24]
            k += 4 + 3 * ndim + 24
            xg = np.stack([f8(recs[3 + i]) for i in range(3)], 1)
            son = [i4(recs[4 + 3 * ndim + ind]) for ind in range(8)]
            vals = [[f8(hyd[h + ind * nvar + v]) for v in range(nvar)] for ind in range(8)]
            h += 8 * nvar
            if dom >= ncpu:
                continue                              # boundary grids are not part of the domain
            for ind in range(8):
                off = np.array([(ind & 1) - 0.5, ((ind >> 1) & 1) - 0.5, ((ind >> 2) & 1) - 0.5]) * dxc
                leaf = (son[ind] == 0) | (l == L)
                pos = (xg[leaf] + off - xbound) * boxlen
                out["level"].append(np.full(leaf.sum(), l))
                out["x"].append(pos[:, 0])
                out["y"].append(pos[:, 1])
                out["z"].append(pos[:, 2])
                out["dx"].append(np.full(leaf.sum(), dxc * boxlen))
                for v, n in enumerate(names):
                    out[n].append(vals[ind][v][leaf])
    return {n: np.concatenate(v) if v else np.zeros(0) for n, v in out.items()}


def solution_sums(cells: dict, threshold: float = 2.0e-14, norm_min: float = 1.0e-30,
                  min_variance: float = 1.0e-14) -> dict:
    """Whole-snapshot checksums in the manner of the reference's regression
    check (tests/visu/visu_ramses.py:495-560): per variable a compensated sum
    of log10|x| (density, pressure) or of |x| with components below
    ``threshold`` x |vector| set to zero, values within ``min_variance`` of
    the mean replaced by the mean."""
    import math
    keys = [k for k in cells if k not in ("level", "x", "y", "z", "dx")]
    norms = {k: 1.0 for k in keys}
    if all(("velocity" + s) in cells for s in ("_x", "_y", "_z")):
        vn = np.sqrt(cells["velocity_x"] ** 2 + cells["velocity_y"] ** 2 + cells["velocity_z"] ** 2)
        vn = np.where(vn < norm_min, norm_min, vn)
        for s in ("_x", "_y", "_z"):
            norms["velocity" + s] = vn
    out = {}
    for k in sorted(keys):
        a = np.asarray(cells[k])
        av = np.average(a)
        data = a if av == 0.0 else np.where(np.abs(a - av) / abs(av) < min_variance, av, a)
        if k in ("density", "pressure"):
            sol = np.log10(np.abs(data))
        else:
            sol = np.where(np.abs(data) < threshold * norms[k], 0.0, np.abs(data))
        out[k] = math.fsum(sol)
    return out
