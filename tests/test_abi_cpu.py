"""The C ABI without a GPU: the shared library loads, exports every function
declared in include/ramses_b200.h, and rejects bad input before touching a
device. No compute call is made."""
import ctypes
import re
from pathlib import Path

import pytest

from ramses_b200 import build, runtime
from ramses_b200.params import HydroParams, hydro_params_from_namelist, nsubcycle_from_namelist
from ramses_b200 import mesh

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def lib():
    if not runtime.LIB_PATH.exists():
        build.build()
    return runtime.load()


def header_functions():
    text = (ROOT / "include" / "ramses_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    fns = header_functions()
    for f in ("rb_create", "rb_godunov_fine", "rb_unsplit", "rb_courant_fine", "rb_coarse_step"):
        assert f in fns


def test_library_exports_every_declared_symbol(lib):
    missing = [f for f in header_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_status_strings(lib):
    assert lib.rb_status_string(0) == b"ok"
    assert b"invalid" in lib.rb_status_string(1)
    assert lib.rb_version().startswith(b"ramses_b200")


def test_bad_parameters_rejected_before_device(lib):
    hp = runtime.hydro_params_c(HydroParams(riemann="hllc"))
    hp.riemann = 9
    tree = mesh.uniform_tree(2)
    mp = runtime.mesh_params_c(tree)
    h = ctypes.c_void_p()
    rc = lib.rb_create(ctypes.byref(hp), ctypes.byref(mp), 0, ctypes.byref(h))
    assert rc == 1
    assert b"Riemann" in lib.rb_last_error()


def test_no_device_reported(lib):
    if lib.rb_device_count() > 0:
        pytest.skip("a CUDA device is visible")
    hp = runtime.hydro_params_c(HydroParams(riemann="hllc"))
    mp = runtime.mesh_params_c(mesh.uniform_tree(2))
    h = ctypes.c_void_p()
    assert lib.rb_create(ctypes.byref(hp), ctypes.byref(mp), 0, ctypes.byref(h)) == 7


def test_python_params_validation():
    with pytest.raises(ValueError):
        HydroParams(riemann="roe").validate()
    HydroParams(riemann="exact").validate()
    HydroParams(riemann="acoustic").validate()
    with pytest.raises(ValueError):
        HydroParams(riemann="exact", niter_riemann=0).validate()
    HydroParams(difmag=0.1).validate()
    with pytest.raises(ValueError):
        HydroParams(difmag=-0.1).validate()
    with pytest.raises(ValueError):
        HydroParams(slope_type=4).validate()
    HydroParams(scheme="plmde").validate()
    with pytest.raises(ValueError):
        HydroParams(scheme="induction").validate()
    HydroParams(riemann="hll", slope_type=8).validate()


NML = """&RUN_PARAMS
hydro=.true.
nsubcycle=3*1,2
/
&HYDRO_PARAMS
gamma=1.4
courant_factor=0.8
slope_type=2
riemann='hllc'
/
&REFINE_PARAMS
err_grad_d=0.05
interpol_var=0
interpol_type=2
/
"""


def test_namelist_reader():
    hp = hydro_params_from_namelist(NML)
    assert hp.gamma == 1.4 and hp.courant_factor == 0.8 and hp.slope_type == 2 and hp.riemann == "hllc"
    assert hp.interpol_type == 2
    ns = nsubcycle_from_namelist(NML, 6)
    assert ns[1:6] == [1, 1, 1, 2, 2]


def test_tile_shape_info(lib):
    tx, ty, tz, nt = (ctypes.c_int32() for _ in range(4))
    assert lib.rb_tile_shape_info(4, ctypes.byref(tx), ctypes.byref(ty), ctypes.byref(tz), ctypes.byref(nt)) == 0
    assert (tx.value, ty.value, tz.value) == (8, 8, 8)
    assert lib.rb_tile_shape_info(17, None, None, None, None) == 1


def test_mesh_builder_rules():
    t = mesh.uniform_tree(3)
    assert t.noct(3) == 64 and t.leaf_cells(3) == 512
    tree = mesh.build_tree(3, 5, mesh.sphere_refine((0.5, 0.5, 0.5), 0.05))
    # every oct's 27 father-neighbour cells exist (nesting rule)
    for l in range(4, 6):
        for c in tree.coords[l]:
            for off in [(i, j, k) for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)]:
                cc = (c + off) % (2 ** (l - 1))
                po = cc // 2
                keys = tree.coords[l - 1]
                assert ((keys == po).all(axis=1)).any()


def test_boundary_tree_layout():
    """mesh.add_boundaries: RAMSES's extended coarse grid (one boundary coarse
    cell per bounded side), regions ordered -x,+x,-y,+y,-z,+z with the later
    regions covering edges and corners, every boundary oct's reference oct
    (son(nbor(igrid,inbor))) present at its level, cell centres measured from
    the box corner."""
    import numpy as np

    from ramses_b200 import mesh
    t = mesh.add_boundaries(mesh.build_tree(3, 3, None), ("outflow", None, "reflexive"))
    assert (t.nx, t.ny, t.nz, t.nx_loc, t.offset) == (3, 1, 3, 1, (1, 0, 1))
    assert t.boundary_type == [11, 12, 5, 6]
    # x regions: the x column over the interior z; z regions: all x
    assert [len(g[3]) for g in t.boundary] == [64, 64, 192, 192]
    for ib, bt in enumerate(t.boundary_type):
        d = bt % 10
        inbor = d + 1 if d % 2 else d - 1
        for l in range(1, 4):
            g = t.boundary[ib][l]
            ref = t.son[t.nbor[inbor - 1, g - 1] - 1]
            assert np.all(ref > 0)
    cells, x = t.cell_centres(3, boundary=False)
    assert x.min() > 0 and x.max() < 1 and len(cells) == 8 * 64
    _, xb = t.cell_centres(3)
    assert xb[:, 0].min() < 0 and xb[:, 2].max() > 1 and np.all((xb[:, 1] > 0) & (xb[:, 1] < 1))
    with pytest.raises(ValueError):
        mesh.add_boundaries(mesh.build_tree(3, 3, None), ("inflow", None, None))
