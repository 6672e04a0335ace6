"""The benchmark configurations' own physics against the FP64 CPU oracle.

The headline configuration (the supersonic turbulent box: gamma = 1.001,
RMS Mach 5, P = 0.01 rho, hllc, moncen slopes) and the blast-clump AMR
configuration (32 seeded dense clumps around a Sedov blast, hllc, moncen,
subcycled levels) at reduced size, stepped on the GPU through the C ABI and
by the oracle on the same seeded inputs:

* FP64: bit-identical to the oracle after 1 and after 50 steps; the per-cell
  relative tolerances of the drop-in (1e-12 after one step, 1e-9 after many)
  are asserted as well;
* FP32-mixed (every z-streaming column shape that takes the scheme): L1 and
  L-inf relative errors of rho, P and |v| against the oracle, with
  L1(rho) <= 1e-5;
* the Sedov blast stays mirror symmetric about the box centre (exactly in
  FP64, as the oracle does).
"""
import numpy as np
import pytest

import oracle
from ramses_b200 import ics, mesh, runtime
from ramses_b200.params import HydroParams

from helpers import leaf_values, max_rel, sedov_uniform, turbulent_uniform

pytestmark = pytest.mark.gpu


def prim_errors(u_test, u_ref, cells, gamma):
    """L1 (sum|d| / sum|ref|) and L-inf (max|d| / max|ref|) of rho, P, |v|
    over the given 1-based cells."""
    def prim(u):
        r = u[0, cells - 1]
        v = u[1:4, cells - 1] / r
        p = (gamma - 1.0) * (u[4, cells - 1] - 0.5 * r * (v * v).sum(axis=0))
        return {"rho": r, "P": p, "v": np.sqrt((v * v).sum(axis=0))}
    a, b = prim(u_test), prim(u_ref)
    out = {}
    for k in ("rho", "P", "v"):
        d = np.abs(a[k] - b[k])
        out[k] = (float(d.sum() / np.abs(b[k]).sum()), float(d.max() / np.abs(b[k]).max()))
    return out


def oracle_steps(tree, hp, u, steps, nsubcycle=None):
    orc = oracle.OracleRun(tree, hp, u, nsubcycle=nsubcycle)
    for _ in range(steps):
        orc.coarse_step()
    return orc


_TURB_REF = {}


def turbulent_reference(level, steps):
    """(tree, hp, u0, oracle state after ``steps`` steps), computed once."""
    key = (level, steps)
    if key not in _TURB_REF:
        tree, hp, u = turbulent_uniform(level)
        _TURB_REF[key] = (tree, hp, u, oracle_steps(tree, hp, u, steps).uold.copy())
    return _TURB_REF[key]


@pytest.mark.parametrize("level", [5, 6])
def test_turbulent_box_fp64_equals_oracle_1_and_50_steps(cuda_lib, oracle_lib, level):
    tree, hp, u = turbulent_uniform(level)
    cells = tree.cell_index(level).reshape(-1)
    orc = oracle.OracleRun(tree, hp, u)
    with runtime.Solver(tree, hp, uold=u) as s:
        s.uniform_run(1, graph=False)
        orc.coarse_step()
        got = s.download_state()
        assert max_rel(got[:, cells - 1], orc.uold[:, cells - 1]) <= 1e-12
        np.testing.assert_array_equal(got, orc.uold)
        assert s.t == orc.t
        s.uniform_run(49, graph=True)
        for _ in range(49):
            orc.coarse_step()
        got = s.download_state()
        assert max_rel(got[:, cells - 1], orc.uold[:, cells - 1]) <= 1e-9
        np.testing.assert_array_equal(got, orc.uold)
        assert s.t == orc.t


@pytest.mark.parametrize("shape", [None, 1, 5, 6])
def test_turbulent_box_mixed_vs_oracle_50_steps(cuda_lib, oracle_lib, shape):
    """FP32-mixed through the z-streaming kernels (None: the default choice;
    1: stream_step_kernel 16x8; 5, 6: stream2_step_kernel at 3 and 2 CTAs per
    SM) against the FP64 oracle after 50 steps of the 64^3 box."""
    level, steps = 6, 50
    tree, hp, u, ref = turbulent_reference(level, steps)
    cells = tree.cell_index(level).reshape(-1)
    with runtime.Solver(tree, hp, precision="mixed", uold=u) as s:
        if shape is not None:
            s.set_stream_shape(shape, 16)
        s.uniform_run(steps, graph=True)
        got = s.download_state()
        if shape in (5, 6) or shape is None:
            assert s.uniform_info()["kernel"].startswith("stream2_step_kernel")
    err = prim_errors(got, ref, cells, hp.gamma)
    print("mixed shape %s vs oracle after %d steps: %s" % (shape, steps, err))
    assert err["rho"][0] <= 1e-5, err
    for k in ("rho", "P", "v"):
        assert err[k][0] <= 1e-5 and err[k][1] <= 1e-4, (k, err)
    # conservation of the mixed path: FP64 accumulation of widened face fluxes
    _, a0 = leaf_values(tree, u)
    _, a1 = leaf_values(tree, got)
    scale = np.abs(a0).sum(axis=1)
    assert np.all(np.abs(a1.sum(axis=1) - a0.sum(axis=1)) <= 1e-13 * scale)


def blast_clumps_small():
    """The blast-clump configuration on levels 4-7 with moncen slopes: the
    blast radius widened to 0.06 so that the coarser finest level resolves
    it (the full configuration deposits E = 10 within 0.01 on levels up to
    11)."""
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=2, courant_factor=0.8)
    prim = ics.blast_clumps_prim(r_blast=0.06)

    def fields(x):
        q = prim(x)
        return [q[0], q[4]]
    tree = mesh.build_tree(4, 7, mesh.gradient_refine(fields, [0.05, 0.05]))
    return tree, hp, ics.fill_all_levels(tree, prim, hp.gamma)


def test_blast_clumps_amr_fp64_equals_oracle(cuda_lib, oracle_lib):
    tree, hp, u = blast_clumps_small()
    assert tree.noct(7) > 0
    orc = oracle.OracleRun(tree, hp, u, nsubcycle=[2] * 33)
    with runtime.Solver(tree, hp, uold=u, nsubcycle=[2] * 33) as s:
        for step in range(5):
            s.coarse_step()
            orc.coarse_step()
            assert s.t == orc.t, step
        got = s.download_state()
        cells, vo = leaf_values(tree, orc.uold)
        assert max_rel(got[:, cells - 1], vo) <= 1e-9
        np.testing.assert_array_equal(got[:, cells - 1], vo)
        # the device-scheduled path (CUDA graphs of coarse steps) continues it
        s.run(max_steps=3)
        for _ in range(3):
            orc.coarse_step()
        np.testing.assert_array_equal(s.download_state()[:, cells - 1], orc.uold[:, cells - 1])


def test_blast_clumps_amr_mixed_vs_oracle(cuda_lib, oracle_lib):
    tree, hp, u = blast_clumps_small()
    orc = oracle_steps(tree, hp, u, 5, nsubcycle=[2] * 33)
    with runtime.Solver(tree, hp, precision="mixed", uold=u, nsubcycle=[2] * 33) as s:
        for _ in range(5):
            s.coarse_step()
        got = s.download_state()
    cells, _ = leaf_values(tree, u)
    err = prim_errors(got, orc.uold, cells, hp.gamma)
    print("blast-clump AMR mixed vs oracle after 5 coarse steps: %s" % err)
    for k in ("rho", "P", "v"):
        assert err[k][0] <= 1e-5, (k, err)


def mirror_errors(tree, level, u):
    """max |u - mirror(u)| / max |u| per variable for the three reflections
    x -> 1-x, y -> 1-y, z -> 1-z (the reflected momentum component negated)."""
    U = u[:, tree.cell_index(level) - 1]       # (5, z, y, x)
    out = []
    for axis, mom in ((3, 1), (2, 2), (1, 3)):
        M = np.flip(U, axis=axis).copy()
        M[mom] = -M[mom]
        out.append(np.abs(M - U).max(axis=(1, 2, 3)) / np.abs(U).max(axis=(1, 2, 3)))
    return np.array(out)


def test_sedov_mirror_symmetry(cuda_lib, oracle_lib):
    level = 5
    tree, hp, u = sedov_uniform(level, slope_type=2)
    orc = oracle_steps(tree, hp, u, 30)
    assert np.all(mirror_errors(tree, level, orc.uold) == 0.0)
    with runtime.Solver(tree, hp, uold=u) as s:
        s.uniform_run(30)
        f64 = s.download_state()
    assert np.all(mirror_errors(tree, level, f64) == 0.0)
    np.testing.assert_array_equal(f64, orc.uold)
    with runtime.Solver(tree, hp, precision="mixed", uold=u) as s:
        s.uniform_run(30)
        mixed = s.download_state()
    err = mirror_errors(tree, level, mixed)
    print("mixed mirror asymmetry per variable:", err.max(axis=0))
    assert np.all(err <= 1e-6)
