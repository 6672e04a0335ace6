"""CPU: host logic of the serving harness and the server ABI's argument
checks (no GPU needed)."""
import ctypes

import numpy as np
import pytest

from ramses_b200 import ics, mesh, runtime, serve
from ramses_b200.params import HydroParams


def test_request_mix_is_seeded_and_in_range():
    a = serve.draw_requests(400, seed=11)
    b = serve.draw_requests(400, seed=11)
    assert [(r.kind, r.n, r.extra, r.params) for r in a] == [(r.kind, r.n, r.extra, r.params) for r in b]
    assert {r.n for r in a} == {32, 64, 128} and {r.extra for r in a} == {0, 1, 2}
    tubes = [r for r in a if r.kind == "tube"]
    sedovs = [r for r in a if r.kind == "sedov"]
    assert 150 < len(tubes) < 250 and len(tubes) + len(sedovs) == 400
    for r in tubes:
        p = r.params
        assert 0.1 <= p["rho_l"] <= 10 and 0.1 <= p["rho_r"] <= 10
        assert 0.01 <= p["p_l"] <= 100 and 0.01 <= p["p_r"] <= 100
        assert -2 <= p["u_l"] <= 2 and -2 <= p["u_r"] <= 2
    assert all(0.1 <= r.params["energy"] <= 10 for r in sedovs)


def test_poisson_arrivals_rate():
    t = serve.poisson_arrivals(20000, rate=250.0, seed=5)
    assert np.all(np.diff(t) > 0)
    assert abs(np.mean(np.diff(t)) - 1 / 250.0) < 0.05 / 250.0


def test_fifo_completion_known_answer():
    comp = serve.fifo_completion([0.0, 0.5, 0.6, 5.0], [1.0, 1.0, 0.2, 0.1])
    np.testing.assert_allclose(comp, [1.0, 2.0, 2.2, 5.1])
    p = serve.percentiles(comp - np.array([0.0, 0.5, 0.6, 5.0]))
    assert p["max"] == pytest.approx(1.6) and p["p50"] == pytest.approx(1.25)


def test_dense_octree_round_trip():
    tree = mesh.uniform_tree(3)
    rng = np.random.default_rng(0)
    d = rng.random((5, 8, 8, 8))
    u = serve.octree_from_dense(tree, 3, d)
    np.testing.assert_array_equal(serve.dense_from_octree(tree, 3, u), d)
    # the coarser levels hold the restriction, as fill_uniform_level_from_grid sets it
    q = rng.random((5, 8, 8, 8)) + 0.5
    u2 = ics.fill_uniform_level_from_grid(tree, 3, q, 1.4)
    d2 = serve.dense_from_octree(tree, 3, u2)
    np.testing.assert_allclose(serve.octree_from_dense(tree, 3, d2), u2, rtol=1e-15, atol=0)


def test_build_request_kinds():
    hp = HydroParams(gamma=1.4, riemann="hllc", slope_type=1)
    spec = serve.RequestSpec("sedov", 32, 0, {"energy": 2.0})
    b = serve.build_request(spec, hp)
    assert b.is_dense and b.dense.shape == (5, 32, 32, 32)
    # total energy of the blast plus the ambient thermal energy
    e_amb = 1e-5 / 0.4 * (32 ** 3 - np.count_nonzero(b.dense[4] > 1e-3)) / 32 ** 3
    assert b.dense[4].sum() / 32 ** 3 == pytest.approx(2.0 + e_amb, rel=1e-12)
    spec = serve.RequestSpec("tube", 32, 1, {"rho_l": 1.0, "p_l": 1.0, "u_l": 0.0, "rho_r": 0.125, "p_r": 0.1,
                                             "u_r": 0.0})
    b = serve.build_request(spec, hp)
    assert not b.is_dense and b.tree.nlevelmax == 6 and b.tree.noct(6) > 0
    assert serve.leaf_updates_estimate(b) > 32 ** 3


def test_server_without_device():
    lib = runtime.load()
    if lib.rb_device_count() > 0:
        pytest.skip("a CUDA device is visible")
    hp = runtime.hydro_params_c(HydroParams(riemann="hllc"))
    h = ctypes.c_void_p()
    assert lib.rb_server_create(ctypes.byref(hp), 0, 0, 8, ctypes.byref(h)) == 7
    bad = runtime.hydro_params_c(HydroParams(riemann="hllc"))
    bad.riemann = 9
    assert lib.rb_server_create(ctypes.byref(bad), 0, 0, 8, ctypes.byref(h)) == 1
    assert lib.rb_server_create(ctypes.byref(hp), 5, 0, 8, ctypes.byref(h)) == 1
    # null server handles are rejected, not dereferenced
    n = ctypes.c_int32()
    assert lib.rb_server_progress(None, None, 0, ctypes.byref(n)) == 1
    assert lib.rb_server_cancel(None, 1) == 1
    assert lib.rb_server_destroy(None) == 0
