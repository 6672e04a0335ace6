"""GPU: the serving engine (rb_server_*) through its C ABI.

A served problem must give bitwise the result of the single-problem paths
(rb_uniform_run for dense problems, rb_run for octree problems), and the same
result alone as mixed with any other problems: no reduction or atomic spans
problems, so packing cannot change a bit.
"""

import numpy as np
import pytest

from ramses_b200 import mesh, runtime, serve
from ramses_b200.params import HydroParams

from helpers import sedov_amr, turbulent_uniform

pytestmark = pytest.mark.gpu

HP = HydroParams(gamma=1.4, riemann="hllc", slope_type=1, courant_factor=0.8)


def dense_problem(kind, n, seed):
    spec = serve.draw_requests(1, seed, sizes=(n,), max_extra=0)[0]
    spec.kind = kind
    if kind == "tube":
        spec.params = {"rho_l": 1.0 + seed % 3, "p_l": 1.0, "u_l": 0.3, "rho_r": 0.125, "p_r": 0.1, "u_r": -0.2}
    else:
        spec.params = {"energy": 0.5 + seed % 4}
    return serve.build_request(spec, HP).dense


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dense_request_equals_uniform_run(cuda_lib, precision):
    tree, hp, u = turbulent_uniform(5)
    lvl = 5
    with runtime.Solver(tree, hp, precision=precision, uold=u) as s:
        s.uniform_run(7, graph=False)
        ref = serve.dense_from_octree(tree, lvl, s.download_state())
        t_ref = s.t
    with serve.Server(hp, precision=precision) as srv:
        rid = srv.submit_dense(serve.dense_from_octree(tree, lvl, u), max_steps=7)
        srv.drain()
        inf = srv.info(rid)
        assert inf["state"] == serve.REQ_DONE and inf["steps"] == 7
        assert inf["t"] == t_ref
        np.testing.assert_array_equal(srv.results[rid], ref)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_alone_equals_mixed(cuda_lib, precision):
    """A problem's result does not depend on the problems it is batched with."""
    a = dense_problem("sedov", 32, 1)
    others = [dense_problem("tube", 64, 2), dense_problem("sedov", 64, 3), dense_problem("tube", 32, 4),
              dense_problem("sedov", 32, 5)]
    tree, hp_amr, u_amr = sedov_amr(3, 5)
    t_end = 2e-3
    with serve.Server(HP, precision=precision, steps_per_round=3) as srv:
        ra = srv.submit_dense(a, t_end=t_end)
        srv.drain()
        alone = srv.results[ra].copy()
        steps_alone = srv.info(ra)["steps"]
    with serve.Server(HP, precision=precision, steps_per_round=5) as srv:
        ids = [srv.submit_dense(o, t_end=t_end * (1 + i)) for i, o in enumerate(others[:2])]
        srv.progress()
        rb = srv.submit_dense(a, t_end=t_end)          # joins a batch already running
        ids += [srv.submit_dense(o, t_end=t_end / 2) for o in others[2:]]
        ids.append(srv.submit_octree(tree, u_amr, t_end=1e-3))
        srv.drain()
        assert srv.info(rb)["steps"] == steps_alone
        np.testing.assert_array_equal(srv.results[rb], alone)
        for i in ids:
            assert srv.info(i)["state"] == serve.REQ_DONE
        assert srv.stats()["batch_launches"] > 0


def test_dense_request_runs_to_t_end(cuda_lib):
    """The dense clock: steps until t >= t_end, like rb_run on the octree."""
    d = dense_problem("sedov", 32, 0)
    tree = mesh.uniform_tree(5)
    u = serve.octree_from_dense(tree, 5, d)
    t_end = 3e-3
    with runtime.Solver(tree, HP, uold=u) as s:
        n = s.run(t_end=t_end)
        ref = serve.dense_from_octree(tree, 5, s.download_state())
        t_ref = s.t
    with serve.Server(HP, precision="fp64") as srv:
        rid = srv.submit_dense(d, t_end=t_end)
        srv.drain()
        inf = srv.info(rid)
        assert inf["steps"] == n and inf["t"] == t_ref and inf["t"] >= t_end
        np.testing.assert_array_equal(srv.results[rid], ref)


def test_octree_request_equals_run(cuda_lib):
    tree, hp, u = sedov_amr(4, 6)
    with runtime.Solver(tree, HP, uold=u) as s:
        n = s.run(t_end=4e-3)
        ref = s.download_state()
        t_ref = s.t
    with serve.Server(HP, precision="fp64") as srv:
        rid = srv.submit_octree(tree, u, t_end=4e-3)
        srv.drain()
        inf = srv.info(rid)
        assert inf["state"] == serve.REQ_DONE and inf["steps"] == n and inf["t"] == t_ref
        np.testing.assert_array_equal(srv.results[rid], ref)


def test_admission_by_budget(cuda_lib):
    """With room for one 32^3 problem at a time every request still completes,
    in arrival order, with the same results; an oversize request is refused."""
    probs = [dense_problem("sedov", 32, i) for i in range(4)]
    one = 2 * 5 * 32 ** 3 * 8
    with serve.Server(HP, precision="fp64") as srv:
        ref_ids = [srv.submit_dense(p, max_steps=6) for p in probs]
        srv.drain()
        refs = [srv.results[i].copy() for i in ref_ids]
    with serve.Server(HP, precision="fp64", hbm_budget_bytes=one + one // 2) as srv:
        ids = [srv.submit_dense(p, max_steps=6) for p in probs]
        srv.progress()
        st = srv.stats()
        assert st["active"] == 1 and st["queued"] == 3 and st["bytes_in_use"] <= st["budget"]
        order = srv.drain()
        assert [i for i in order if i in ids] == ids
        for i, r in zip(ids, refs):
            np.testing.assert_array_equal(srv.results[i], r)
        with pytest.raises(runtime.RBError) as e:
            srv.submit_dense(dense_problem("sedov", 64, 0), max_steps=1)
        assert e.value.status == 8  # RB_ERR_CAPACITY


def test_cancel(cuda_lib):
    probs = [dense_problem("tube", 32, i) for i in range(3)]
    with serve.Server(HP, precision="mixed", hbm_budget_bytes=2 * 5 * 32 ** 3 * 8) as srv:
        ids = [srv.submit_dense(p, max_steps=50) for p in probs]
        srv.cancel(ids[2])        # still queued
        srv.progress()
        srv.cancel(ids[0])        # active
        srv.drain()
        assert srv.info(ids[0])["state"] == serve.REQ_CANCELLED
        assert srv.info(ids[1])["state"] == serve.REQ_DONE and srv.info(ids[1])["steps"] == 50
        assert srv.info(ids[2])["state"] == serve.REQ_CANCELLED


def test_stream_harness(cuda_lib):
    """A short Poisson stream through the harness: every request completes and
    latencies are measured from arrival."""
    specs = serve.draw_requests(6, seed=3, sizes=(32,), max_extra=1)
    reqs = [serve.build_request(s, HP) for s in specs]
    arr = serve.poisson_arrivals(len(reqs), 200.0, seed=4)
    with serve.Server(HP, precision="mixed") as srv:
        res = serve.run_stream(srv, reqs, arr, t_end=2e-3)
    assert len(res["tts"]) == 6 and min(res["tts"]) > 0
    assert res["cell_updates"] > 0 and res["latency_s"]["p99"] >= res["latency_s"]["p50"]


@pytest.mark.parametrize("mask", [0, 1, 7])
def test_dense_request_matches_dense_oracle(cuda_lib, oracle_lib, mask):
    """Dense problems with periodic (0), x-outflow (1) or all-outflow (7)
    boundaries: the served FP64 state equals the oracle's dense step bit for
    bit (outflow = the zero-gradient ghost cells of bound_type 2)."""
    import oracle
    spec = serve.RequestSpec("tube", 32, 0, {"rho_l": 2.0, "p_l": 3.0, "u_l": 0.4, "rho_r": 0.5, "p_r": 0.2,
                                             "u_r": -0.3})
    d = serve.build_request(spec, HP, outflow=True).dense
    ref = d.copy()
    t = 0.0
    for _ in range(6):
        t += oracle.dense_step(HP, ref, bc_outflow=mask)
    with serve.Server(HP, precision="fp64", steps_per_round=4) as srv:
        rid = srv.submit_dense(d, max_steps=6, outflow_mask=mask)
        srv.drain()
        inf = srv.info(rid)
        assert inf["steps"] == 6 and inf["t"] == t
        np.testing.assert_array_equal(srv.results[rid], ref)


def test_outflow_mixed_close_to_fp64(cuda_lib):
    spec = serve.RequestSpec("tube", 64, 0, {"rho_l": 1.0, "p_l": 1.0, "u_l": 0.0, "rho_r": 0.125, "p_r": 0.1,
                                             "u_r": 0.0})
    d = serve.build_request(spec, HP, outflow=True).dense
    out = {}
    for prec in ("fp64", "mixed"):
        with serve.Server(HP, precision=prec) as srv:
            rid = srv.submit_dense(d, t_end=0.05, outflow_mask=1)
            srv.drain()
            out[prec] = srv.results[rid].copy()
    r64, r32 = out["fp64"][0], out["mixed"][0]
    assert np.abs(r32 - r64).sum() / np.abs(r64).sum() < 1e-5
    # nothing re-entered through the x boundaries: the far left and right
    # states are still the initial ones
    assert r64[0, 0, 0] == pytest.approx(1.0, abs=1e-10) and r64[0, 0, -1] == pytest.approx(0.125, abs=1e-10)


def test_outflow_octree_tube_request_equals_run(cuda_lib, oracle_lib):
    """An AMR shock-tube request with outflow boundaries in x (free boundary
    regions of the octree): the served state equals rb_run's and, in the box
    and the boundary layers next to it, the oracle's."""
    import oracle
    spec = serve.RequestSpec("tube", 16, 1, {"rho_l": 2.0, "p_l": 3.0, "u_l": 0.4, "rho_r": 0.5, "p_r": 0.2,
                                             "u_r": -0.3})
    b = serve.build_request(spec, HP, outflow=True)
    tree, u = b.tree, b.uold
    assert tree.boundary_type == [11, 12]
    with runtime.Solver(tree, HP, uold=u) as s:
        n = s.run(max_steps=6)
        ref = s.download_state()
    with serve.Server(HP, precision="fp64") as srv:
        rid = srv.submit_octree(tree, u, max_steps=6)
        srv.drain()
        assert srv.info(rid)["steps"] == n == 6
        np.testing.assert_array_equal(srv.results[rid], ref)
    orc = oracle.OracleRun(tree, HP, u)
    for _ in range(6):
        orc.coarse_step()
    from test_gpu_boundary import determined_cells
    c = determined_cells(tree) - 1
    np.testing.assert_array_equal(ref[:, c], orc.uold[:, c])
