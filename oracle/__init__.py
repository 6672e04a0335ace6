"""ctypes wrapper of the CPU oracle (``ramses_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline / reference arm, as the checker. The product
package ``ramses_b200`` never imports it.

Parity status: restatement of the reference Fortran. Its NDIM=1/2 companion
(``ramses_oracle_amr.c``, ``run_amr``), which shares the Riemann solvers,
reproduces the reference's own regression checksums of the 1D AMR Sod run
and the 2D AMR implosion (tests/hydro/sod-tube, tests/hydro/implosion); the
3D restatement is also pinned
physically to the reference's Sod known-answer table. 3D bit-level parity
with the Fortran binary is unpinned (no Fortran compiler in the build image).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
LIB_PATH = BUILD / "liboracle.so"
SRC = HERE / "ramses_oracle.c"
HDR = HERE / "ramses_oracle.h"
SOURCES = [SRC, HERE / "ramses_oracle_amr.c"]
HEADERS = [HDR, HERE / "ramses_oracle_amr.h"]
CFLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared", "-std=c11"]


def build(force: bool = False) -> Path:
    """Compile the oracle with gcc (no FMA contraction)."""
    BUILD.mkdir(exist_ok=True)
    if (not force and LIB_PATH.exists()
            and LIB_PATH.stat().st_mtime >= max(f.stat().st_mtime for f in SOURCES + HEADERS)):
        return LIB_PATH
    tmp = LIB_PATH.with_suffix(".so.tmp%d" % os.getpid())
    subprocess.run(["gcc", *CFLAGS, *map(str, SOURCES), "-o", str(tmp), "-lm"], check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(build()))
        _declare(_lib)
    return _lib


class OrcParams(ctypes.Structure):
    _fields_ = [("gamma", ctypes.c_double), ("smallr", ctypes.c_double),
                ("smallc", ctypes.c_double), ("courant_factor", ctypes.c_double),
                ("slope_theta", ctypes.c_double), ("riemann", ctypes.c_int32),
                ("slope_type", ctypes.c_int32), ("interpol_var", ctypes.c_int32),
                ("interpol_type", ctypes.c_int32), ("pressure_fix", ctypes.c_int32),
                ("beta_fix", ctypes.c_double), ("niter_riemann", ctypes.c_int32),
                ("difmag", ctypes.c_double), ("scheme", ctypes.c_int32)]


MAXLEVEL = 32
_P32 = ctypes.POINTER(ctypes.c_int32)
_P64 = ctypes.POINTER(ctypes.c_int64)
_PD = ctypes.POINTER(ctypes.c_double)


class OrcRefine(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("err_grad_d", "err_grad_p", "err_grad_u",
                                                "floor_d", "floor_u", "floor_p")]


class OrcMesh(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("ncoarse", ctypes.c_int32), ("ngridmax", ctypes.c_int32),
                ("nlevelmax", ctypes.c_int32), ("levelmin", ctypes.c_int32),
                ("nvector", ctypes.c_int32), ("boxlen", ctypes.c_double),
                ("son", _P32), ("father", _P32), ("nbor", _P32), ("active", _P32),
                ("active_off", _P64), ("uold", _PD), ("unew", _PD),
                ("nsubcycle", ctypes.c_int32 * (MAXLEVEL + 1)),
                ("dtnew", ctypes.c_double * (MAXLEVEL + 1)),
                ("dtold", ctypes.c_double * (MAXLEVEL + 1)),
                ("t", ctypes.c_double), ("nstep", ctypes.c_int64),
                ("mass_tot", ctypes.c_double), ("ekin_tot", ctypes.c_double),
                ("eint_tot", ctypes.c_double), ("cell_updates", ctypes.c_int64),
                ("nthreads", ctypes.c_int32), ("divu", _PD), ("enew", _PD),
                ("nx_loc", ctypes.c_int32), ("nboundary", ctypes.c_int32),
                ("boundary_type", _P32), ("bound_off", _P64), ("bound_igrid", _P32)]


_NREG = 8
_NBND = 4


class OrcAmrParams(ctypes.Structure):
    """orc_amr_params (ramses_oracle_amr.h): the namelist of a 1D or 2D run."""
    _fields_ = [("hydro", OrcParams), ("refine", OrcRefine), ("ndim", ctypes.c_int32),
                ("levelmin", ctypes.c_int32), ("nlevelmax", ctypes.c_int32), ("ngridmax", ctypes.c_int32),
                ("nexpand", ctypes.c_int32 * (MAXLEVEL + 1)), ("nsubcycle", ctypes.c_int32 * (MAXLEVEL + 1)),
                ("boxlen", ctypes.c_double), ("tout", ctypes.c_double), ("nboundary", ctypes.c_int32),
                ("ibound_min", ctypes.c_int32 * _NBND), ("ibound_max", ctypes.c_int32 * _NBND),
                ("jbound_min", ctypes.c_int32 * _NBND), ("jbound_max", ctypes.c_int32 * _NBND),
                ("bound_type", ctypes.c_int32 * _NBND), ("nregion", ctypes.c_int32),
                ("x_center", ctypes.c_double * _NREG), ("y_center", ctypes.c_double * _NREG),
                ("length_x", ctypes.c_double * _NREG), ("length_y", ctypes.c_double * _NREG),
                ("exp_region", ctypes.c_double * _NREG), ("d_region", ctypes.c_double * _NREG),
                ("u_region", ctypes.c_double * _NREG), ("v_region", ctypes.c_double * _NREG),
                ("p_region", ctypes.c_double * _NREG), ("max_coarse_steps", ctypes.c_int64),
                ("dt_force", _PD), ("dt_force_n", ctypes.c_int64)]


class OrcAmrResult(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_int32), ("init_only", ctypes.c_int32),
                ("pos", _PD), ("level", _P32), ("u", _PD), ("ncell", ctypes.c_int32),
                ("taken", ctypes.c_int32), ("t", ctypes.c_double), ("nstep", ctypes.c_int64),
                ("nstep_coarse", ctypes.c_int64), ("noct", ctypes.c_int32 * (MAXLEVEL + 1)),
                ("message", ctypes.c_char * 160), ("dt_log", _PD), ("dt_cap", ctypes.c_int32)]


def run_amr(hp, refine, *, ndim, levelmin, nlevelmax, ngridmax, tout, regions, nsubcycle, nexpand,
            boxlen=1.0, boundaries=(), max_coarse_steps=10_000_000, init_only=False, capacity=1 << 18,
            dt_force=None):
    """A whole 1D or 2D RAMSES hydro run in the oracle (ramses_oracle_amr.c)
    up to the snapshot of the first coarse step starting at t >= tout.

    ``refine``: (err_grad_d, err_grad_p, err_grad_u), -1 for off (floors 1e-10);
    ``regions``: 'square' regions as dicts with x_center, length_x, d, p and
    optionally y_center, length_y, u, v, exp_region (default 2);
    ``boundaries``: (ibound_min, ibound_max, jbound_min, jbound_max,
    bound_type) per region as in the namelist, bound_type 1 reflexive or 2
    outflow; empty: periodic;
    ``nsubcycle``, ``nexpand``: per level from level 1, as RAMSES holds them
    after read_params (entry k of the namelist applies to levelmin + k - 1);
    ``dt_force``: for one complete level, the time steps of the coarse steps
    in place of courant_fine's.
    Returns the leaf cells (pos, level, conservative u), the run's clock and
    the dt of every completed coarse step (``dt``)."""
    p = OrcAmrParams()
    p.hydro = params_struct(hp)
    d, pr, uu = refine
    p.refine = OrcRefine(d, pr, uu, 1e-10, 1e-10, 1e-10)
    p.ndim, p.levelmin, p.nlevelmax, p.ngridmax = ndim, levelmin, nlevelmax, ngridmax
    for lvl in range(1, MAXLEVEL + 1):
        p.nsubcycle[lvl] = nsubcycle[lvl - 1] if lvl - 1 < len(nsubcycle) else 2
        p.nexpand[lvl] = nexpand[lvl - 1] if lvl - 1 < len(nexpand) else 1
    p.boxlen, p.tout = boxlen, tout
    if len(boundaries) > _NBND or len(regions) > _NREG:
        raise ValueError("too many boundary or initial-condition regions")
    p.nboundary = len(boundaries)
    for i, (imin, imax, jmin, jmax, bt) in enumerate(boundaries):
        p.ibound_min[i], p.ibound_max[i], p.jbound_min[i], p.jbound_max[i], p.bound_type[i] = imin, imax, jmin, jmax, bt
    p.nregion = len(regions)
    for k, reg in enumerate(regions):
        p.x_center[k], p.length_x[k] = reg["x_center"], reg["length_x"]
        p.y_center[k], p.length_y[k] = reg.get("y_center", 0.0), reg.get("length_y", 1.0)
        p.exp_region[k] = reg.get("exp_region", 2.0)
        p.d_region[k], p.p_region[k] = reg["d"], reg["p"]
        p.u_region[k], p.v_region[k] = reg.get("u", 0.0), reg.get("v", 0.0)
    p.max_coarse_steps = max_coarse_steps
    if dt_force is not None:
        dtf = np.ascontiguousarray(dt_force, dtype=np.float64)
        p.dt_force, p.dt_force_n = _ptr(dtf, _PD), len(dtf)
    pos = np.zeros((capacity, ndim))
    lv = np.zeros(capacity, np.int32)
    u = np.zeros((capacity, ndim + 2))
    r = OrcAmrResult()
    r.capacity, r.init_only = capacity, 1 if init_only else 0
    r.pos, r.level, r.u = _ptr(pos, _PD), _ptr(lv, _P32), _ptr(u, _PD)
    ncap = int(min(max_coarse_steps, 1 << 20))
    dts = np.full(ncap, np.nan)
    r.dt_log, r.dt_cap = _ptr(dts, _PD), ncap
    rc = lib().orc_amr_run(ctypes.byref(p), ctypes.byref(r))
    if rc != 0:
        raise RuntimeError("orc_amr_run failed (%d): %s" % (rc, r.message.decode()))
    n = r.ncell
    if n > capacity:
        raise RuntimeError("more leaf cells than capacity")
    return {"pos": pos[:n].copy(), "level": lv[:n].copy(), "u": u[:n].copy(), "t": r.t, "taken": bool(r.taken),
            "nstep": r.nstep, "nstep_coarse": r.nstep_coarse,
            "noct": [r.noct[lvl] for lvl in range(1, nlevelmax + 1)],
            "dt": dts[:min(r.nstep_coarse, ncap)].copy()}


def _declare(L):
    P = ctypes.POINTER(OrcParams)
    M = ctypes.POINTER(OrcMesh)
    L.orc_unsplit.argtypes = [P, _PD, _PD, _PD, _PD, ctypes.c_double, ctypes.c_double,
                              ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int]
    L.orc_cmpdt.argtypes = [P, _PD, _PD, ctypes.c_double, ctypes.c_int, ctypes.c_int]
    L.orc_cmpdt.restype = ctypes.c_double
    for name in ("orc_set_unew", "orc_set_uold", "orc_upload_fine"):
        getattr(L, name).argtypes = [P, M, ctypes.c_int]
    L.orc_godunov_fine.argtypes = [P, M, ctypes.c_int, ctypes.c_double]
    L.orc_courant_fine.argtypes = [P, M, ctypes.c_int, _PD, _PD, _PD, _PD]
    L.orc_coarse_step.argtypes = [P, M]
    L.orc_make_boundary_hydro.argtypes = [P, M, ctypes.c_int]
    L.orc_get3cubefather.argtypes = [M, ctypes.c_int, ctypes.c_int, _P32]
    L.orc_getnborfather.argtypes = [M, ctypes.c_int, ctypes.c_int, _P32]
    L.orc_interpol_hydro.argtypes = [P, _PD, _PD, ctypes.c_int]
    L.orc_hydro_flag.argtypes = [P, ctypes.POINTER(OrcRefine), M, ctypes.c_int, _P32]
    L.orc_dense_step.argtypes = [P, _PD, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_int, ctypes.c_int, _PD]
    L.orc_hydro_flag.restype = ctypes.c_int64
    L.orc_riemann_face.argtypes = [P, _PD, _PD, _PD]
    L.orc_amr_run.argtypes = [ctypes.POINTER(OrcAmrParams), ctypes.POINTER(OrcAmrResult)]


def params_struct(hp) -> OrcParams:
    hp.validate()
    return OrcParams(hp.gamma, hp.smallr, hp.smallc, hp.courant_factor, hp.slope_theta,
                     hp.riemann_code, hp.slope_type, hp.interpol_var, hp.interpol_type,
                     1 if hp.pressure_fix else 0, hp.beta_fix, hp.niter_riemann, hp.difmag,
                     hp.scheme_code)


def _ptr(a, t):
    return a.ctypes.data_as(t)


def unsplit(hp, uin, gravin, dx, dt, ngrid=None):
    """Fortran-layout unsplit: uin (5,6,6,6,nvector) C-order == Fortran
    uin(nvector,-1:4,-1:4,-1:4,5). Returns (flux (3,5,3,3,3,nv), tmp (3,2,3,3,3,nv))."""
    uin = np.ascontiguousarray(uin, dtype=np.float64)
    nv = uin.shape[-1]
    if gravin is None:
        gravin = np.zeros((3, 6, 6, 6, nv))
    gravin = np.ascontiguousarray(gravin, dtype=np.float64)
    flux = np.zeros((3, 5, 3, 3, 3, nv))
    tmp = np.zeros((3, 2, 3, 3, 3, nv))
    p = params_struct(hp)
    rc = lib().orc_unsplit(ctypes.byref(p), _ptr(uin, _PD), _ptr(gravin, _PD), _ptr(flux, _PD),
                           _ptr(tmp, _PD), dx, dx, dx, dt, nv if ngrid is None else ngrid, nv)
    if rc:
        raise RuntimeError("orc_unsplit failed: %d" % rc)
    return flux, tmp


def interpol_hydro(hp, u1):
    """interpol_hydro (hydro/interpol_hydro.f90:268-444) of nn father cells:
    u1 (nn, 7, 5) = father cell and its 6 getnborfather neighbours,
    conservative; returns u2 (nn, 8, 5), the 8 children."""
    u1 = np.asarray(u1, np.float64)
    nn = u1.shape[0]
    a = np.ascontiguousarray(np.transpose(u1, (2, 1, 0)))  # Fortran u1(nn,7,5)
    out = np.zeros((5, 8, nn))
    p = params_struct(hp)
    rc = lib().orc_interpol_hydro(ctypes.byref(p), _ptr(a, _PD), _ptr(out, _PD), nn)
    if rc:
        raise RuntimeError("orc_interpol_hydro failed: %d" % rc)
    return np.transpose(out, (2, 1, 0))


def dense_step(hp, u, boxlen=1.0, bc_outflow=0, nvector=32):
    """One coarse step of a complete level given as conservative
    [5, nz, ny, nx] (advanced in place); returns dt. bc_outflow: bit d set
    makes axis d an outflow (zero-gradient) boundary, else periodic."""
    assert u.dtype == np.float64 and u.flags.c_contiguous and u.shape[0] == 5
    nz, ny, nx = u.shape[1:]
    dx = boxlen / nx
    dt = ctypes.c_double()
    p = params_struct(hp)
    rc = lib().orc_dense_step(ctypes.byref(p), _ptr(u, _PD), nx, ny, nz, dx, boxlen / hp.smallc,
                              int(bc_outflow), nvector, ctypes.byref(dt))
    if rc:
        raise RuntimeError("orc_dense_step failed: %d" % rc)
    return dt.value


class OracleRun:
    """One hydro problem held in Fortran-layout host arrays, stepped by the
    oracle with RAMSES's amr_step hydro call sequence."""

    def __init__(self, tree, hp, uold, nsubcycle=None, nvector=32, nthreads=0):
        self.tree = tree
        self.hp = hp
        self.p = params_struct(hp)
        self.son = np.ascontiguousarray(tree.son, dtype=np.int32)
        self.father = np.ascontiguousarray(tree.father, dtype=np.int32)
        self.nbor = np.ascontiguousarray(tree.nbor, dtype=np.int32)
        self.active, self.active_off = tree.active_concat()
        self.uold = np.ascontiguousarray(uold, dtype=np.float64).copy()
        assert self.uold.shape == (5, tree.ncell)
        self.unew = self.uold.copy()
        m = OrcMesh()
        m.nx, m.ny, m.nz = tree.nx, tree.ny, tree.nz
        m.ncoarse, m.ngridmax = tree.ncoarse, tree.ngridmax
        m.nlevelmax, m.levelmin, m.nvector = tree.nlevelmax, tree.levelmin, nvector
        m.boxlen = tree.boxlen
        m.son, m.father, m.nbor = _ptr(self.son, _P32), _ptr(self.father, _P32), _ptr(self.nbor, _P32)
        m.active, m.active_off = _ptr(self.active, _P32), _ptr(self.active_off, _P64)
        m.uold, m.unew = _ptr(self.uold, _PD), _ptr(self.unew, _PD)
        ns = nsubcycle or [2] * (MAXLEVEL + 1)
        for i in range(MAXLEVEL + 1):
            m.nsubcycle[i] = ns[i] if i < len(ns) else 2
        m.nthreads = nthreads
        # pressure_fix: velocity divergence and internal energy per cell
        self.divu = np.zeros(tree.ncell)
        self.enew = np.zeros(tree.ncell)
        m.divu, m.enew = _ptr(self.divu, _PD), _ptr(self.enew, _PD)
        # physical boundaries: filled once per level as init_flow_fine does
        # (hydro/init_flow_fine.f90:19), then after every level step
        m.nx_loc = getattr(tree, "nx_loc", 0)
        self.btype, self.boff, self.bgrid = tree.boundary_concat()
        m.nboundary = len(self.btype)
        m.boundary_type, m.bound_off = _ptr(self.btype, _P32), _ptr(self.boff, _P64)
        m.bound_igrid = _ptr(self.bgrid, _P32)
        self.m = m
        if m.nboundary:
            for l in range(1, tree.nlevelmax + 1):
                self.make_boundary_hydro(l)

    def _check(self, rc, what):
        if rc:
            raise RuntimeError("%s failed: %d" % (what, rc))

    def coarse_step(self):
        self._check(lib().orc_coarse_step(ctypes.byref(self.p), ctypes.byref(self.m)), "coarse_step")

    def godunov_fine(self, ilevel, dt):
        self._check(lib().orc_godunov_fine(ctypes.byref(self.p), ctypes.byref(self.m), ilevel, dt), "godunov_fine")

    def set_unew(self, ilevel):
        lib().orc_set_unew(ctypes.byref(self.p), ctypes.byref(self.m), ilevel)

    def set_uold(self, ilevel):
        lib().orc_set_uold(ctypes.byref(self.p), ctypes.byref(self.m), ilevel)

    def make_boundary_hydro(self, ilevel):
        self._check(lib().orc_make_boundary_hydro(ctypes.byref(self.p), ctypes.byref(self.m), ilevel),
                    "make_boundary_hydro")

    def upload_fine(self, ilevel):
        lib().orc_upload_fine(ctypes.byref(self.p), ctypes.byref(self.m), ilevel)

    def courant_fine(self, ilevel, dt_in=None):
        dt = ctypes.c_double(self.tree.boxlen / self.hp.smallc if dt_in is None else dt_in)
        ma, ek, ei = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(lib().orc_courant_fine(ctypes.byref(self.p), ctypes.byref(self.m), ilevel,
                                           ctypes.byref(dt), ctypes.byref(ma), ctypes.byref(ek),
                                           ctypes.byref(ei)), "courant_fine")
        return dt.value, ma.value, ek.value, ei.value

    @property
    def t(self):
        return self.m.t

    @property
    def cell_updates(self):
        return self.m.cell_updates

    def dtnew(self, level):
        return self.m.dtnew[level]

    def hydro_flag(self, ilevel, rp, flag1=None):
        """hydro_flag(ilevel): returns (flag1 with the level's flagged cells
        set to 1, number newly flagged); flag1 has ncell+1 entries (0..ncell)."""
        f = np.zeros(self.tree.ncell + 1, np.int32) if flag1 is None else flag1
        r = OrcRefine(rp.err_grad_d, rp.err_grad_p, rp.err_grad_u, rp.floor_d, rp.floor_u, rp.floor_p)
        n = lib().orc_hydro_flag(ctypes.byref(self.p), ctypes.byref(r), ctypes.byref(self.m), ilevel,
                                 _ptr(f, _P32))
        return f, int(n)

    def get3cubefather(self, cell, ilevel):
        out = np.zeros(27, np.int32)
        self._check(lib().orc_get3cubefather(ctypes.byref(self.m), cell, ilevel, _ptr(out, _P32)), "get3cubefather")
        return out

    def getnborfather(self, cell, ilevel):
        out = np.zeros(7, np.int32)
        self._check(lib().orc_getnborfather(ctypes.byref(self.m), cell, ilevel, _ptr(out, _P32)), "getnborfather")
        return out
