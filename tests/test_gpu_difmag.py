"""GPU: artificial diffusion (difmag > 0: cmpdivu and consup,
hydro/uplmde.f90:702-866, called from unsplit, hydro/umuscl.f90:166-169)
against the oracle, FP64 bit for bit, through the Fortran-layout unsplit,
the octree level step and the uniform path."""
import numpy as np
import pytest

import oracle
from ramses_b200 import runtime
from ramses_b200.params import HydroParams

from helpers import leaf_values, random_blocks, sedov_amr, sedov_uniform

pytestmark = pytest.mark.gpu


def _dm(hp, difmag=0.1):
    hp = HydroParams(**{**hp.__dict__})
    hp.difmag = difmag
    return hp


@pytest.mark.parametrize("riemann", ["hllc", "llf"])
@pytest.mark.parametrize("slope_type", [1, 2, 3])
def test_unsplit_bitwise(cuda_lib, oracle_lib, riemann, slope_type):
    hp = HydroParams(gamma=1.4, riemann=riemann, slope_type=slope_type, courant_factor=0.5, difmag=0.2)
    nv = 32
    uin = random_blocks(nv, seed=5 + slope_type)
    rng = np.random.default_rng(4)
    grav = 0.1 * rng.standard_normal((3, 6, 6, 6, nv))
    f_gpu, t_gpu = runtime.unsplit(hp, uin, grav, dx=1.0 / 64, dt=2e-3, ngrid=29)
    f_cpu, t_cpu = oracle.unsplit(hp, uin, grav, dx=1.0 / 64, dt=2e-3, ngrid=29)
    hp0 = HydroParams(**{**hp.__dict__})
    hp0.difmag = 0.0
    f_ref0, _ = oracle.unsplit(hp0, uin, grav, dx=1.0 / 64, dt=2e-3, ngrid=29)
    for d in range(3):
        sl = [slice(0, 2)] * 3
        sl[2 - d] = slice(0, 3)
        idx = (d, slice(None), *sl, slice(0, 29))
        np.testing.assert_array_equal(f_gpu[idx], f_cpu[idx])
    assert np.any(f_cpu != f_ref0)  # the diffusion acts on these blocks


@pytest.mark.parametrize("slope_type", [1, 2])
def test_amr_coarse_steps_bitwise(cuda_lib, oracle_lib, slope_type):
    tree, hp, u = sedov_amr(3, 5, slope_type=slope_type)
    hp = _dm(hp)
    orc = oracle.OracleRun(tree, hp, u)
    with runtime.Solver(tree, hp, uold=u) as s:
        for _ in range(4):
            orc.coarse_step()
            s.coarse_step()
        np.testing.assert_array_equal(s.download_state(), orc.uold)
        assert s.t == orc.t


def test_device_scheduled_run_bitwise(cuda_lib, oracle_lib):
    tree, hp, u = sedov_amr(3, 5)
    hp = _dm(hp)
    orc = oracle.OracleRun(tree, hp, u)
    for _ in range(4):
        orc.coarse_step()
    with runtime.Solver(tree, hp, uold=u) as s:
        assert s.run(max_steps=4) == 4
        np.testing.assert_array_equal(s.download_state(), orc.uold)


def test_uniform_run_bitwise(cuda_lib, oracle_lib):
    tree, hp, u = sedov_uniform(4, slope_type=2)
    hp = _dm(hp)
    orc = oracle.OracleRun(tree, hp, u)
    for _ in range(6):
        orc.coarse_step()
    with runtime.Solver(tree, hp, uold=u) as s:
        s.uniform_run(6)
        np.testing.assert_array_equal(s.download_state(), orc.uold)


def test_mixed_close_to_fp64(cuda_lib):
    tree, hp, u = sedov_amr(3, 5)
    hp = _dm(hp)
    with runtime.Solver(tree, hp, uold=u) as a, runtime.Solver(tree, hp, precision="mixed", uold=u) as b:
        for _ in range(4):
            a.coarse_step()
            b.coarse_step()
        _, ra = leaf_values(tree, a.download_state())
        _, rb_ = leaf_values(tree, b.download_state())
        assert np.abs(ra[0] - rb_[0]).sum() / np.abs(ra[0]).sum() < 1e-5
