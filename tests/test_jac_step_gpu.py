"""jac1's update and the res that follows it as one launch (k_jac_step:
tiles of nodes, each recomputing the updated u of the neighbours its res
reads, u and du written to second buffers), against the reference's
sequential build: u bit-identical, and in SEQ mode u_sum and u_max too.
The fused form runs when reductions are deferred (the update waits for the
next res call) and when the iteration is captured as a graph."""
import hashlib

import numpy as np
import pytest

from conftest import load_golden
from oplus2_matlab_b200 import api, apps
from oplus2_matlab_b200 import mesh as M

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def fused_calls():
    import ctypes as C
    cnt = C.c_int(0)
    t = api.lib().op2b_loop_time(b"update+res", C.byref(cnt))
    return cnt.value if t >= 0 else 0


@pytest.mark.parametrize("knobs", [{}, {"jac_tile_nodes": 64}, {"jac_tile_nodes": 300},
                                   {"jac_step_threads": 1024}, {"jac_step_threads": 256,
                                                                "jac_tile_nodes": 4096}])
def test_deferred_jac1_step_matches_reference(op2, knobs):
    g = load_golden("jac1_nn64")
    lib = api.lib()
    op2.set_strategy(op2.STRATEGY_GATHER)
    op2.set_reduction(op2.REDUCE_SEQ)
    for k, v in knobs.items():
        lib.op2b_set_tuning(k.encode(), v)
    try:
        jm = M.jac(g["NN"], g["variant"])
        J = apps.Jac(jm, g["variant"])
        api.set_gbl_deferred(1)
        for _ in range(g["niter"]):
            J.iteration()  # no synchronisation: each update waits for the next res
        api.sync()
        um, us = float(J.u_max[0]), float(J.u_sum[0])
        u = J.fetch()
        assert fused_calls() == g["niter"] - 1
    finally:
        api.set_gbl_deferred(0)
        for k in knobs:
            lib.op2b_set_tuning(k.encode(), {"jac_tile_nodes": 0, "jac_step_threads": 512}[k])
    assert op2.last_error() == ""
    assert sha(u) == g["u_sha256"]
    gm, grms = g["u_max_rms"][-1]
    assert np.float32(um) == np.float32(gm)
    assert np.float32(np.sqrt(np.float32(us) / np.float32(jm.nnode))) == np.float32(grms)


def test_jac1_step_graph_is_one_launch(op2):
    """The rotated iteration (update, then the next res) captured as a graph
    is one kernel, and launching it repeatedly gives the reference's u."""
    g = load_golden("jac1_nn64")
    lib = api.lib()
    op2.set_strategy(op2.STRATEGY_GATHER)
    op2.set_reduction(op2.REDUCE_TREE)
    jm = M.jac(g["NN"], g["variant"])
    J = apps.Jac(jm, g["variant"])
    api.set_gbl_deferred(1)
    try:
        res = lambda: api.op_par_loop("res", J.edges, *J.res_args)
        upd = lambda: api.op_par_loop("update", J.nodes, *J.upd_args)
        res()
        upd()
        res()  # plans built: update + res ran fused once
        api.sync()
        assert lib.op2b_capture_begin(0) == 1, op2.last_error()
        upd()
        res()
        h = lib.op2b_capture_end()
        assert h, op2.last_error()
        assert lib.op2b_graph_nkernels(h) == 1
        for _ in range(g["niter"] - 2):
            assert lib.op2b_graph_launch(h) == 0
        lib.op2b_graph_destroy(h)
        upd()
        api.sync()
    finally:
        api.set_gbl_deferred(0)
    assert op2.last_error() == ""
    assert sha(J.fetch()) == g["u_sha256"]


def test_jac1_step_larger_grid_tree(op2):
    """NN=256 (tiles of a few rows): u bit-identical to the
    two-launch form; the TREE sum within summation order."""
    jm = M.jac(256, 1)
    op2.set_strategy(op2.STRATEGY_GATHER)
    op2.set_reduction(op2.REDUCE_TREE)
    J = apps.Jac(jm, 1)
    ref = [J.iteration() for _ in range(20)]
    u_ref = J.fetch().copy()
    api.op_exit()
    api.op_init([], 0)
    api.set_strategy(api.STRATEGY_GATHER)
    J = apps.Jac(jm, 1)
    api.set_gbl_deferred(1)
    try:
        for _ in range(20):
            J.iteration()
        api.sync()
        um, us = float(J.u_max[0]), float(J.u_sum[0])
        u = J.fetch()
    finally:
        api.set_gbl_deferred(0)
    assert np.array_equal(u, u_ref)
    # deferred TREE results are added to the host variables when delivered
    # (at the sync), so u_sum holds the 20 iterations' sums together and
    # u_max the largest
    assert um == max(r[0] for r in ref)
    total = sum(r[1] for r in ref)
    assert abs(us - total) <= 1e-5 * total
