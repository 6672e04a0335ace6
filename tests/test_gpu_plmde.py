"""GPU: the PLMDE predictor (scheme='plmde': tracexyz, hydro/uplmde.f90:375-696,
selected in unsplit, hydro/umuscl.f90:73-94) against the oracle, FP64 bit for
bit, through the Fortran-layout unsplit, the octree level step, the
device-scheduled run, the dense uniform path and the serving engine."""
import numpy as np
import pytest

import oracle
from ramses_b200 import runtime, serve
from ramses_b200.params import HydroParams

from helpers import leaf_values, random_blocks, sedov_amr, sedov_uniform, turbulent_uniform

pytestmark = pytest.mark.gpu


def _plm(hp, **kw):
    return HydroParams(**{**hp.__dict__, "scheme": "plmde", **kw})


@pytest.mark.parametrize("riemann", ["hllc", "llf", "acoustic"])
@pytest.mark.parametrize("slope_type", [1, 2, 3])
def test_unsplit_bitwise(cuda_lib, oracle_lib, riemann, slope_type):
    hp = HydroParams(gamma=1.4, riemann=riemann, slope_type=slope_type, courant_factor=0.5, scheme="plmde")
    nv = 32
    uin = random_blocks(nv, seed=11 + slope_type)
    rng = np.random.default_rng(8)
    grav = 0.1 * rng.standard_normal((3, 6, 6, 6, nv))
    f_gpu, t_gpu = runtime.unsplit(hp, uin, grav, dx=1.0 / 64, dt=2e-3, ngrid=29)
    f_cpu, t_cpu = oracle.unsplit(hp, uin, grav, dx=1.0 / 64, dt=2e-3, ngrid=29)
    f_muscl, _ = oracle.unsplit(_plm(hp, scheme="muscl"), uin, grav, dx=1.0 / 64, dt=2e-3, ngrid=29)
    for d in range(3):
        sl = [slice(0, 2)] * 3
        sl[2 - d] = slice(0, 3)
        idx = (d, slice(None), *sl, slice(0, 29))
        np.testing.assert_array_equal(f_gpu[idx], f_cpu[idx])
        assert np.any(f_cpu[idx] != f_muscl[idx])


@pytest.mark.parametrize("slope_type", [1, 2, 3])
def test_amr_coarse_steps_bitwise(cuda_lib, oracle_lib, slope_type):
    tree, hp, u = sedov_amr(3, 5, slope_type=slope_type)
    hp = _plm(hp)
    orc = oracle.OracleRun(tree, hp, u)
    with runtime.Solver(tree, hp, uold=u) as s:
        for _ in range(4):
            orc.coarse_step()
            s.coarse_step()
        np.testing.assert_array_equal(s.download_state(), orc.uold)
        assert s.t == orc.t


def test_device_scheduled_run_bitwise(cuda_lib, oracle_lib):
    tree, hp, u = sedov_amr(3, 5)
    hp = _plm(hp, riemann="llf")
    orc = oracle.OracleRun(tree, hp, u)
    for _ in range(4):
        orc.coarse_step()
    with runtime.Solver(tree, hp, uold=u) as s:
        assert s.run(max_steps=4) == 4
        np.testing.assert_array_equal(s.download_state(), orc.uold)


def test_with_pressure_fix_and_difmag_bitwise(cuda_lib, oracle_lib):
    """PLMDE, the dual-energy fix and the artificial diffusion together."""
    tree, hp, u = sedov_amr(3, 5)
    hp = _plm(hp, pressure_fix=True, beta_fix=0.5, difmag=0.1)
    orc = oracle.OracleRun(tree, hp, u)
    with runtime.Solver(tree, hp, uold=u) as s:
        for _ in range(3):
            orc.coarse_step()
            s.coarse_step()
        np.testing.assert_array_equal(s.download_state(), orc.uold)


@pytest.mark.parametrize("method", ["stream", "tiles"])
def test_uniform_run_bitwise(cuda_lib, oracle_lib, method):
    tree, hp, u = sedov_uniform(4, slope_type=2)
    hp = _plm(hp)
    orc = oracle.OracleRun(tree, hp, u)
    for _ in range(6):
        orc.coarse_step()
    with runtime.Solver(tree, hp, uold=u) as s:
        s.set_uniform_method(method)
        s.uniform_run(6)
        np.testing.assert_array_equal(s.download_state(), orc.uold)


def test_served_dense_equals_uniform_run(cuda_lib):
    tree, hp, u = turbulent_uniform(5)
    hp = _plm(hp)
    with runtime.Solver(tree, hp, uold=u) as s:
        s.uniform_run(5, graph=False)
        ref = serve.dense_from_octree(tree, 5, s.download_state())
    with serve.Server(hp, precision="fp64") as srv:
        rid = srv.submit_dense(serve.dense_from_octree(tree, 5, u), max_steps=5)
        srv.drain()
        np.testing.assert_array_equal(srv.results[rid], ref)


@pytest.mark.parametrize("path", ["amr", "uniform"])
def test_mixed_close_to_fp64(cuda_lib, path):
    if path == "amr":
        tree, hp, u = sedov_amr(3, 5)
    else:
        tree, hp, u = turbulent_uniform(5)
    hp = _plm(hp)
    with runtime.Solver(tree, hp, uold=u) as a, runtime.Solver(tree, hp, precision="mixed", uold=u) as b:
        for _ in range(4):
            a.coarse_step()
            b.coarse_step()
        _, ra = leaf_values(tree, a.download_state())
        _, rb_ = leaf_values(tree, b.download_state())
        assert np.abs(ra[0] - rb_[0]).sum() / np.abs(ra[0]).sum() < 1e-5


def test_compiled_variant_with_pressure_fix_bitwise(cuda_lib, oracle_lib):
    """hllc + minmod + PLMDE with the dual-energy fix: the compiled PLMDE
    variant of the pressure_fix tile kernel."""
    tree, hp, u = sedov_amr(3, 5)
    hp = _plm(hp, pressure_fix=True, beta_fix=0.5)
    orc = oracle.OracleRun(tree, hp, u)
    with runtime.Solver(tree, hp, uold=u) as s:
        for _ in range(3):
            orc.coarse_step()
            s.coarse_step()
        np.testing.assert_array_equal(s.download_state(), orc.uold)
