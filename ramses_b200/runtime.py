"""ctypes binding of the C ABI (``include/ramses_b200.h``) and a small host-side
driver that mirrors the reference's hydro call sites.

The library is the in-tree ``ramses_b200/lib/libramses_b200.so``; there is no
CPU fallback: if it cannot be loaded, or no CUDA device is visible, every
entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

from .mesh import Octree
from .params import HydroParams

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libramses_b200.so"

RB_PREC_FP64 = 0
RB_PREC_MIXED = 1
MAXLEVEL = 32
# z-streaming column shapes (TX, TY, CTAs per SM of register budget), as
# kStreamShapes in csrc/tile_launch.h; STREAM2_SHAPES run stream2_step_kernel
# (FP32-mixed, HLLC with minmod or moncen slopes)
STREAM_SHAPES = [(8, 8, 1), (16, 8, 1), (16, 16, 1), (16, 8, 2), (8, 8, 4), (16, 8, 3), (16, 8, 2)]
STREAM2_SHAPES = (5, 6)

_P32 = ctypes.POINTER(ctypes.c_int32)
_P64 = ctypes.POINTER(ctypes.c_int64)
_PD = ctypes.POINTER(ctypes.c_double)


class HydroParamsC(ctypes.Structure):
    _fields_ = [("gamma", ctypes.c_double), ("smallr", ctypes.c_double), ("smallc", ctypes.c_double),
                ("courant_factor", ctypes.c_double), ("slope_theta", ctypes.c_double),
                ("riemann", ctypes.c_int32), ("slope_type", ctypes.c_int32), ("scheme", ctypes.c_int32),
                ("interpol_var", ctypes.c_int32), ("interpol_type", ctypes.c_int32),
                ("pressure_fix", ctypes.c_int32), ("difmag", ctypes.c_double),
                ("beta_fix", ctypes.c_double), ("niter_riemann", ctypes.c_int32), ("pad_", ctypes.c_int32)]


class RefineParamsC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("err_grad_d", "err_grad_p", "err_grad_u",
                                                "floor_d", "floor_u", "floor_p")]


class MeshParamsC(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("ncoarse", ctypes.c_int32), ("ngridmax", ctypes.c_int32), ("nlevelmax", ctypes.c_int32),
                ("levelmin", ctypes.c_int32), ("nvector", ctypes.c_int32), ("boxlen", ctypes.c_double),
                ("nsubcycle", ctypes.c_int32 * (MAXLEVEL + 1)), ("nx_loc", ctypes.c_int32),
                ("pad_", ctypes.c_int32)]


class RBError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        super().__init__("%s: status %d (%s): %s" % (where, status, status_string(status), detail))
        self.status = status


_lib = None

# name -> (restype, argtypes)
_PROTOS = {
    "rb_version": (ctypes.c_char_p, []),
    "rb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "rb_last_error": (ctypes.c_char_p, []),
    "rb_device_count": (ctypes.c_int, []),
    "rb_select_device": (ctypes.c_int, [ctypes.c_int]),
    "rb_create": (ctypes.c_int, [ctypes.POINTER(HydroParamsC), ctypes.POINTER(MeshParamsC), ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_void_p)]),
    "rb_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rb_sync_tree": (ctypes.c_int, [ctypes.c_void_p, _P32, _P32, _P32, _P32, _P32]),
    "rb_set_boundary": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, _P32, _P32, _P32]),
    "rb_make_boundary_hydro": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "rb_upload_state": (ctypes.c_int, [ctypes.c_void_p, _PD]),
    "rb_download_state": (ctypes.c_int, [ctypes.c_void_p, _PD]),
    "rb_upload_level_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _PD]),
    "rb_download_level_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _PD]),
    "rb_note_tree_changed": (ctypes.c_int, [ctypes.c_void_p]),
    "rb_note_host_state_written": (ctypes.c_int, [ctypes.c_void_p]),
    "rb_tree_needs_sync": (ctypes.c_int, [ctypes.c_void_p, _P32]),
    "rb_ensure_device": (ctypes.c_int, [ctypes.c_void_p, _P32, _P32, _P32, _P32, _P32, ctypes.c_int32, _P32, _P32,
                                        _P32, _PD]),
    "rb_ensure_host": (ctypes.c_int, [ctypes.c_void_p, _PD]),
    "rb_transfer_stats": (ctypes.c_int, [ctypes.c_void_p, _P64, _P64, _P64, _P64]),
    "rb_sync_stats": (ctypes.c_int, [ctypes.c_void_p, _PD, _P32, _P32]),
    "rb_download_pressure_fix": (ctypes.c_int, [ctypes.c_void_p, _PD, _PD]),
    "rb_upload_unew": (ctypes.c_int, [ctypes.c_void_p, _PD]),
    "rb_download_unew": (ctypes.c_int, [ctypes.c_void_p, _PD]),
    "rb_set_unew": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "rb_set_uold": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "rb_godunov_fine": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]),
    "rb_upload_fine": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "rb_courant_fine": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _PD, _PD, _PD, _PD]),
    "rb_coarse_step": (ctypes.c_int, [ctypes.c_void_p, _PD, _PD]),
    "rb_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, _PD, _P32]),
    "rb_hydro_flag": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(RefineParamsC), _P32, _P64]),
    "rb_cell_updates": (ctypes.c_int, [ctypes.c_void_p, _P64]),
    "rb_set_tile_shape": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "rb_set_tile_order": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "rb_get_tile_shape": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _P32]),
    "rb_tile_shape_info": (ctypes.c_int, [ctypes.c_int, _P32, _P32, _P32, _P32]),
    "rb_unsplit": (ctypes.c_int, [ctypes.POINTER(HydroParamsC), _PD, _PD, _PD, _PD, _PD, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int]),
    "rb_uniform_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _PD, _PD]),
    "rb_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "rb_set_uniform_method": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "rb_get_uniform_info": (ctypes.c_int, [ctypes.c_void_p, _P32, _P32, _P32, _P32]),
    "rb_autotune_uniform": (ctypes.c_int, [ctypes.c_void_p, _P32, _P32, ctypes.POINTER(ctypes.c_float)]),
    "rb_set_stream_shape": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "rb_server_create": (ctypes.c_int, [ctypes.POINTER(HydroParamsC), ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "rb_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rb_server_submit_dense": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                              ctypes.c_double, ctypes.c_int32, _PD, ctypes.c_double, ctypes.c_int64,
                                              _PD, _P64]),
    "rb_server_submit_octree": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(MeshParamsC), _P32, _P32, _P32,
                                               _P32, _P32, _PD, ctypes.c_double, ctypes.c_int64, _PD, _P64]),
    "rb_server_submit_octree_bounded": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(MeshParamsC), _P32, _P32,
                                                       _P32, _P32, _P32, ctypes.c_int32, _P32, _P32, _P32, _PD,
                                                       ctypes.c_double, ctypes.c_int64, _PD, _P64]),
    "rb_server_progress": (ctypes.c_int, [ctypes.c_void_p, _P64, ctypes.c_int, _P32]),
    "rb_server_request_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, _P32, _PD, _P64, _P64, _PD]),
    "rb_server_cancel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    "rb_server_stats": (ctypes.c_int, [ctypes.c_void_p, _P32, _P32, _P64, _P64, _P64, _P64]),
    "rb_get_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "rb_last_kernel_ms": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "rb_last_run_ms": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "rb_courant_cells_noalloc": (ctypes.c_int, [ctypes.POINTER(HydroParamsC), ctypes.c_void_p, ctypes.c_int64,
                                                ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                                ctypes.c_void_p]),
}


def load(path: Optional[os.PathLike] = None):
    """Load the CUDA library (build it first with ``ramses_b200.build``)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError("CUDA library %s not built (run python -m ramses_b200.build)" % p)
    L = ctypes.CDLL(str(p))
    for name, (res, args) in _PROTOS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = L
    return L


def status_string(s: int) -> str:
    try:
        return load().rb_status_string(s).decode()
    except Exception:  # pragma: no cover - message formatting only
        return "?"


def _check(rc: int, where: str):
    if rc != 0:
        raise RBError(rc, where, load().rb_last_error().decode())


def hydro_params_c(hp: HydroParams) -> HydroParamsC:
    hp.validate()
    return HydroParamsC(hp.gamma, hp.smallr, hp.smallc, hp.courant_factor, hp.slope_theta, hp.riemann_code,
                        hp.slope_type, hp.scheme_code, hp.interpol_var, hp.interpol_type, int(hp.pressure_fix),
                        hp.difmag,
                        hp.beta_fix, hp.niter_riemann, 0)


def mesh_params_c(tree: Octree, nsubcycle: Optional[Sequence[int]] = None, nvector: int = 32) -> MeshParamsC:
    m = MeshParamsC()
    m.nx, m.ny, m.nz = tree.nx, tree.ny, tree.nz
    m.ncoarse, m.ngridmax = tree.ncoarse, tree.ngridmax
    m.nlevelmax, m.levelmin, m.nvector = tree.nlevelmax, tree.levelmin, nvector
    m.boxlen = tree.boxlen
    m.nx_loc = getattr(tree, "nx_loc", 0)
    ns = list(nsubcycle) if nsubcycle is not None else [2] * (MAXLEVEL + 1)
    for i in range(MAXLEVEL + 1):
        m.nsubcycle[i] = ns[i] if i < len(ns) else 2
    return m


def _ptr(a, t):
    return a.ctypes.data_as(t)


def device_count() -> int:
    return load().rb_device_count()


def select_device(device: int) -> None:
    _check(load().rb_select_device(device), "rb_select_device")


class Solver:
    """One device-resident hydro problem (a ``rb_context``)."""

    def __init__(self, tree: Octree, hp: HydroParams, precision: str = "fp64",
                 nsubcycle: Optional[Sequence[int]] = None, nvector: int = 32, uold: Optional[np.ndarray] = None):
        L = load()
        self.tree = tree
        self.hp = hp
        self.precision = precision
        prec = {"fp64": RB_PREC_FP64, "mixed": RB_PREC_MIXED}[precision]
        self._hpc = hydro_params_c(hp)
        self._mpc = mesh_params_c(tree, nsubcycle, nvector)
        h = ctypes.c_void_p()
        _check(L.rb_create(ctypes.byref(self._hpc), ctypes.byref(self._mpc), prec, ctypes.byref(h)), "rb_create")
        self._h = h
        self.t = 0.0
        self.sync_tree()
        if uold is not None:
            self.upload_state(uold)
            # physical boundaries: one fill per level, as init_flow_fine does
            # (hydro/init_flow_fine.f90:19)
            if tree.boundary_type:
                for l in range(1, tree.nlevelmax + 1):
                    self.make_boundary_hydro(l)

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            load().rb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- tree / state -----------------------------------------------------
    def sync_tree(self, tree: Optional[Octree] = None):
        if tree is not None:
            self.tree = tree
        t = self.tree
        son = np.ascontiguousarray(t.son, np.int32)
        father = np.ascontiguousarray(t.father, np.int32)
        nbor = np.ascontiguousarray(t.nbor, np.int32)
        numbl = np.array([t.noct(l) for l in range(1, t.nlevelmax + 1)], np.int32)
        act, _ = t.active_concat()
        bt, boff, bg = t.boundary_concat()
        numbb = np.diff(boff).astype(np.int32)
        _check(load().rb_set_boundary(self._h, len(bt), _ptr(bt, _P32), _ptr(numbb, _P32), _ptr(bg, _P32)),
               "rb_set_boundary")
        _check(load().rb_sync_tree(self._h, _ptr(son, _P32), _ptr(father, _P32), _ptr(nbor, _P32),
                                   _ptr(numbl, _P32), _ptr(act, _P32)), "rb_sync_tree")

    def make_boundary_hydro(self, ilevel: int):
        _check(load().rb_make_boundary_hydro(self._h, ilevel), "rb_make_boundary_hydro")

    # ---- residency protocol of the drop-in boundary ----
    def note_tree_changed(self, tree: Optional[Octree] = None):
        """The host changed the tree (refine_fine, load_balance, defrag)."""
        if tree is not None:
            self.tree = tree
        _check(load().rb_note_tree_changed(self._h), "rb_note_tree_changed")

    def note_host_state_written(self):
        _check(load().rb_note_host_state_written(self._h), "rb_note_host_state_written")

    def ensure_device(self, uold: np.ndarray):
        """Before a device hydro call: re-sync the tree if the host changed
        it, upload uold only if the host copy is the newer one."""
        t = self.tree
        son = np.ascontiguousarray(t.son, np.int32)
        father = np.ascontiguousarray(t.father, np.int32)
        nbor = np.ascontiguousarray(t.nbor, np.int32)
        numbl = np.array([t.noct(l) for l in range(1, t.nlevelmax + 1)], np.int32)
        act, _ = t.active_concat()
        bt, boff, bg = t.boundary_concat()
        numbb = np.diff(boff).astype(np.int32)
        u = np.ascontiguousarray(uold, np.float64)
        assert u.shape == (5, t.ncell)
        _check(load().rb_ensure_device(self._h, _ptr(son, _P32), _ptr(father, _P32), _ptr(nbor, _P32),
                                       _ptr(numbl, _P32), _ptr(act, _P32), len(bt), _ptr(bt, _P32),
                                       _ptr(numbb, _P32), _ptr(bg, _P32), _ptr(u, _PD)), "rb_ensure_device")

    def write_snapshot(self, outdir, nout: int, nstep_coarse: int = 0):
        """dump_all's amr/hydro files of the current state (downloaded from the
        device) in RAMSES's output format: ramses_b200.snapshot."""
        from . import snapshot
        u = self.download_state()
        return snapshot.write_snapshot(outdir, nout, self.tree, u, self.hp.gamma, self.hp.smallr, t=self.t,
                                       nstep_coarse=nstep_coarse)

    def tree_needs_sync(self) -> bool:
        n = ctypes.c_int32()
        _check(load().rb_tree_needs_sync(self._h, ctypes.byref(n)), "rb_tree_needs_sync")
        return bool(n.value)

    def ensure_host(self, uold: np.ndarray):
        """Before host code reads uold: download it if the device copy is newer."""
        assert uold.dtype == np.float64 and uold.flags.c_contiguous and uold.shape == (5, self.tree.ncell)
        _check(load().rb_ensure_host(self._h, _ptr(uold, _PD)), "rb_ensure_host")

    def transfer_stats(self) -> dict:
        v = [ctypes.c_int64() for _ in range(4)]
        _check(load().rb_transfer_stats(self._h, *[ctypes.byref(x) for x in v]), "rb_transfer_stats")
        return dict(zip(("h2d_state_bytes", "d2h_state_bytes", "tree_syncs", "octs_prolonged"),
                        (x.value for x in v)))

    def sync_stats(self) -> dict:
        """Phases of the last tree synchronisation (host ms) and the levels
        whose tables were rebuilt or kept."""
        ms = (ctypes.c_double * 5)()
        built, reused = ctypes.c_int32(), ctypes.c_int32()
        _check(load().rb_sync_stats(self._h, ms, ctypes.byref(built), ctypes.byref(reused)), "rb_sync_stats")
        d = dict(zip(("total_ms", "index_ms", "tables_ms", "boundary_ms", "prolong_ms"), list(ms)))
        d.update(levels_built=built.value, levels_reused=reused.value)
        return d

    def upload_state(self, uold: np.ndarray):
        u = np.ascontiguousarray(uold, np.float64)
        assert u.shape == (5, self.tree.ncell)
        _check(load().rb_upload_state(self._h, _ptr(u, _PD)), "rb_upload_state")

    def download_state(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Fortran-layout uold (5, ncell); ``out`` (e.g. pinned memory) is
        filled in place when given."""
        u = np.empty((5, self.tree.ncell)) if out is None else out
        assert u.shape == (5, self.tree.ncell) and u.dtype == np.float64 and u.flags.c_contiguous
        _check(load().rb_download_state(self._h, _ptr(u, _PD)), "rb_download_state")
        return u

    def upload_level_state(self, ilevel: int, uold: np.ndarray):
        """The rows of level ``ilevel``'s octs from the Fortran-layout host
        array (5, ncell); the device keeps every other row."""
        assert uold.shape == (5, self.tree.ncell) and uold.dtype == np.float64 and uold.flags.c_contiguous
        _check(load().rb_upload_level_state(self._h, ilevel, _ptr(uold, _PD)), "rb_upload_level_state")

    def download_level_state(self, ilevel: int, out: np.ndarray) -> np.ndarray:
        """The rows of level ``ilevel``'s octs into the Fortran-layout host
        array ``out`` (5, ncell); its other rows are left as they are."""
        assert out.shape == (5, self.tree.ncell) and out.dtype == np.float64 and out.flags.c_contiguous
        _check(load().rb_download_level_state(self._h, ilevel, _ptr(out, _PD)), "rb_download_level_state")
        return out

    def upload_unew(self, unew: np.ndarray):
        u = np.ascontiguousarray(unew, np.float64)
        _check(load().rb_upload_unew(self._h, _ptr(u, _PD)), "rb_upload_unew")

    def download_unew(self) -> np.ndarray:
        u = np.empty((5, self.tree.ncell))
        _check(load().rb_download_unew(self._h, _ptr(u, _PD)), "rb_download_unew")
        return u

    def download_pressure_fix(self):
        """pressure_fix arrays (divu, enew), Fortran layout (ncell,) each."""
        dv, en = np.empty(self.tree.ncell), np.empty(self.tree.ncell)
        _check(load().rb_download_pressure_fix(self._h, _ptr(dv, _PD), _ptr(en, _PD)), "rb_download_pressure_fix")
        return dv, en

    # -- level operations (reference names) ------------------------------
    def set_unew(self, ilevel: int):
        _check(load().rb_set_unew(self._h, ilevel), "rb_set_unew")

    def set_uold(self, ilevel: int):
        _check(load().rb_set_uold(self._h, ilevel), "rb_set_uold")

    def godunov_fine(self, ilevel: int, dt: float):
        _check(load().rb_godunov_fine(self._h, ilevel, dt), "rb_godunov_fine")

    def upload_fine(self, ilevel: int):
        _check(load().rb_upload_fine(self._h, ilevel), "rb_upload_fine")

    def courant_fine(self, ilevel: int, dt_in: Optional[float] = None):
        dt = ctypes.c_double(self.tree.boxlen / self.hp.smallc if dt_in is None else dt_in)
        ma, ek, ei = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(load().rb_courant_fine(self._h, ilevel, ctypes.byref(dt), ctypes.byref(ma), ctypes.byref(ek),
                                      ctypes.byref(ei)), "rb_courant_fine")
        return dt.value, ma.value, ek.value, ei.value

    def coarse_step(self) -> float:
        t = ctypes.c_double(self.t)
        dts = (ctypes.c_double * MAXLEVEL)()
        _check(load().rb_coarse_step(self._h, ctypes.byref(t), dts), "rb_coarse_step")
        self.t = t.value
        self.last_dtnew = list(dts)
        return self.t

    def run(self, t_end: float = float("inf"), max_steps: int = 1 << 30, graph: bool = True) -> int:
        """Coarse steps until t >= t_end or max_steps steps (adaptive_loop over
        amr_step) with the scheduler state on the device; returns the steps taken."""
        t = ctypes.c_double(self.t)
        n = ctypes.c_int32()
        _check(load().rb_run(self._h, int(max_steps), float(t_end), 1 if graph else 0, ctypes.byref(t),
                             ctypes.byref(n)), "rb_run")
        self.t = t.value
        return n.value

    def uniform_run(self, nsteps: int, graph: bool = True) -> float:
        t = ctypes.c_double(self.t)
        dt = ctypes.c_double()
        _check(load().rb_uniform_run(self._h, nsteps, 1 if graph else 0, ctypes.byref(t), ctypes.byref(dt)),
               "rb_uniform_run")
        self.t = t.value
        self.next_dt = dt.value
        return self.t

    @property
    def cell_updates(self) -> int:
        n = ctypes.c_int64()
        _check(load().rb_cell_updates(self._h, ctypes.byref(n)), "rb_cell_updates")
        return n.value

    def set_uniform_method(self, method: str):
        """'stream' (z-streaming over a dense mirror) or 'tiles' (oct tiles)."""
        _check(load().rb_set_uniform_method(self._h, {"stream": 0, "tiles": 1}[method]), "rb_set_uniform_method")

    def autotune_uniform(self) -> dict:
        """Time every z-streaming configuration on the live state; keep the best."""
        s, hz, ms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_float()
        _check(load().rb_autotune_uniform(self._h, ctypes.byref(s), ctypes.byref(hz), ctypes.byref(ms)),
               "rb_autotune_uniform")
        return {"shape": s.value, "hz": hz.value, "ms": ms.value}

    def hydro_flag(self, ilevel: int, rp, flag1: Optional[np.ndarray] = None):
        """hydro_flag(ilevel) on the device: returns (flag1, newly flagged)
        where flag1 (int32, ncell+1 entries, index = Fortran cell index) has
        the level's flagged cells set to 1."""
        f = np.zeros(self.tree.ncell + 1, np.int32) if flag1 is None else flag1
        assert f.dtype == np.int32 and f.shape == (self.tree.ncell + 1,) and f.flags.c_contiguous
        r = RefineParamsC(rp.err_grad_d, rp.err_grad_p, rp.err_grad_u, rp.floor_d, rp.floor_u, rp.floor_p)
        n = ctypes.c_int64()
        _check(load().rb_hydro_flag(self._h, int(ilevel), ctypes.byref(r), _ptr(f, _P32), ctypes.byref(n)),
               "rb_hydro_flag")
        return f, n.value

    def flag_tree(self, rp) -> np.ndarray:
        """hydro_flag on the device for every level from levelmin to
        nlevelmax-1 (flag_fine's criterion): one flag array (int32, ncell+1
        entries, index = Fortran cell index) for the host's remesh."""
        t = self.tree
        f = np.zeros(t.ncell + 1, np.int32)
        for l in range(t.levelmin, t.nlevelmax):
            if t.noct(l):
                self.hydro_flag(l, rp, f)
        return f

    def set_stream_shape(self, shape: int, hz: int):
        """Fix the z-streaming column shape and z extent (no autotuning)."""
        _check(load().rb_set_stream_shape(self._h, int(shape), int(hz)), "rb_set_stream_shape")

    def uniform_info(self) -> dict:
        v = [ctypes.c_int32() for _ in range(4)]
        _check(load().rb_get_uniform_info(self._h, *[ctypes.byref(x) for x in v]), "rb_get_uniform_info")
        method, shape, hz, items = (x.value for x in v)
        if method == 0:
            dims = STREAM_SHAPES[shape] if 0 <= shape < len(STREAM_SHAPES) else (0, 0, 0)
            name = "stream2_step_kernel" if shape in STREAM2_SHAPES else "stream_step_kernel"
            kern = "%s<%s,%d,%d,%d> (z-streaming, hz=%d, %d CTAs)" % (
                name, "float" if self.precision == "mixed" else "double", dims[0], dims[1], dims[2], hz, items)
        else:
            kern = "godunov_tile_kernel<%s> shape %d (%d tiles)" % (
                "float" if self.precision == "mixed" else "double", shape, items)
        return {"method": "stream" if method == 0 else "tiles", "shape": shape, "hz": hz, "items": items,
                "kernel": kern}

    def set_tile_shape(self, ilevel: int, shape: int):
        _check(load().rb_set_tile_shape(self._h, ilevel, shape), "rb_set_tile_shape")

    def set_tile_order(self, order: int):
        """Launch order of the levels' tiles: 0 3D Morton, 1 z slabs."""
        _check(load().rb_set_tile_order(self._h, int(order)), "rb_set_tile_order")

    def tile_shape(self, ilevel: int) -> int:
        s = ctypes.c_int32()
        _check(load().rb_get_tile_shape(self._h, ilevel, ctypes.byref(s)), "rb_get_tile_shape")
        return s.value

    def synchronize(self):
        _check(load().rb_synchronize(self._h), "rb_synchronize")

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(load().rb_get_stream(self._h, ctypes.byref(s)), "rb_get_stream")
        return s.value or 0

    def last_kernel_ms(self) -> float:
        f = ctypes.c_float()
        _check(load().rb_last_kernel_ms(self._h, ctypes.byref(f)), "rb_last_kernel_ms")
        return f.value

    def last_run_ms(self) -> float:
        f = ctypes.c_float()
        _check(load().rb_last_run_ms(self._h, ctypes.byref(f)), "rb_last_run_ms")
        return f.value


def unsplit(hp: HydroParams, uin: np.ndarray, gravin: Optional[np.ndarray], dx: float, dt: float,
            ngrid: Optional[int] = None):
    """GPU ``unsplit`` with the reference's Fortran layouts: uin (5,6,6,6,nvector)
    C-order == Fortran uin(nvector,-1:4,-1:4,-1:4,5). Returns (flux, tmp) with
    shapes (3,5,3,3,3,nv) and (3,2,3,3,3,nv)."""
    L = load()
    uin = np.ascontiguousarray(uin, np.float64)
    nv = uin.shape[-1]
    g = None if gravin is None else np.ascontiguousarray(gravin, np.float64)
    flux = np.zeros((3, 5, 3, 3, 3, nv))
    tmp = np.zeros((3, 2, 3, 3, 3, nv))
    hpc = hydro_params_c(hp)
    _check(L.rb_unsplit(ctypes.byref(hpc), _ptr(uin, _PD), None if g is None else _ptr(g, _PD), None,
                        _ptr(flux, _PD), _ptr(tmp, _PD), dx, dx, dx, dt, nv if ngrid is None else ngrid, nv),
           "rb_unsplit")
    return flux, tmp
