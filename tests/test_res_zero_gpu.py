"""res known to hold zeros: airfoil's update leaves res = 0 on every cell and
res_calc and bres_calc only add to it, so the next fused res_calc chain
starts its fold from +0.0 in registers instead of reading res, and leaves
res as it is instead of writing the zeros again (op2b_res_skips counts
those launches).  Any other loop call that writes res makes the next chain
read it.  A graph captured while res was known zero is set at each launch to
read res when res may hold other values then, and back when the zeros are
known again.  Every field is compared with the same calls run eagerly, bit
for bit."""
import numpy as np
import pytest

from oplus2_matlab_b200 import api, apps
from oplus2_matlab_b200 import mesh as M

pytestmark = pytest.mark.gpu

CHAIN = ("adt_calc", "res_calc", "bres_calc", "update")


def start(m, dt, knobs=None):
    api.set_error_mode(api.ERRORS_RETURN)
    api.op_init([], 0)
    api.set_strategy(api.STRATEGY_GATHER)
    api.set_reduction(api.REDUCE_TREE)
    for k, v in (knobs or {}).items():
        api.lib().op2b_set_tuning(k.encode(), v)
    return apps.Airfoil(m, dt)


DEFAULTS = {"chain_tiled": 0, "known_zero": 1}


def finish(A, knobs=None):
    st = {k: v.copy() for k, v in A.fetch().items()}
    err = api.last_error()
    for k in knobs or {}:
        api.lib().op2b_set_tuning(k.encode(), DEFAULTS[k])
    api.op_exit()
    assert err == "", err
    return st


def disturb(A):
    """res_calc and bres_calc without update: res holds their sums."""
    A.loop("res_calc")
    A.loop("bres_calc")
    api.op_fetch_data(A.p_res)
    assert np.any(A.res != 0)


def chain(A):
    A.rms[0] = 0
    for n in CHAIN:
        A.loop(n)


def eager_case(m, dt, knobs):
    """3 iterations, res written by res_calc and bres_calc alone, a chain,
    2 iterations; the skips counted after the 3 iterations and after the
    chain"""
    lib = api.lib()
    A = start(m, dt, knobs)
    lib.op2b_res_skips(1)
    A.iterate(3)
    api.sync()
    first = lib.op2b_res_skips(1)
    disturb(A)
    chain(A)
    api.sync()
    after = lib.op2b_res_skips(1)
    A.iterate(2)
    return finish(A, knobs), first, after


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("tiled", [0, 1])
def test_eager_chain_skips_res_only_when_zero(dt, tiled):
    m = M.naca0012(41, 61)
    st, first, after = eager_case(m, dt, {"chain_tiled": tiled})
    assert first > 0   # res zeroed by each update: the chains after it skip it
    assert after == 0  # res written by other calls: the chain read it
    st0, first0, _ = eager_case(m, dt, {"chain_tiled": tiled, "known_zero": 0})
    assert first0 == 0
    for k in ("q", "qold", "res", "adt"):
        assert np.array_equal(st[k], st0[k]), k


def run_graph_case(m, dt, use_graph):
    """3 iterations, then [disturb, chain] and [chain] twice each, the
    chain eagerly or as a graph captured after the 3 iterations."""
    lib = api.lib()
    A = start(m, dt)
    A.iterate(3)
    api.sync()
    h = None
    if use_graph:
        assert lib.op2b_capture_begin(0) == 1, api.last_error()
        chain(A)
        h = lib.op2b_capture_end()
        assert h, api.last_error()

    def go():
        if use_graph:
            assert lib.op2b_graph_launch(h) == 0, api.last_error()
        else:
            chain(A)

    snaps = []
    for step in ("disturb", "chain", "chain", "disturb", "chain", "chain"):
        if step == "disturb":
            disturb(A)
        else:
            go()
            api.sync()
            snaps.append({k: v.copy() for k, v in A.fetch().items()})
    if h:
        lib.op2b_graph_destroy(h)
    finish(A)
    return snaps


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_graph_reads_res_when_it_may_not_be_zero(dt):
    m = M.naca0012(41, 61)
    eager = run_graph_case(m, dt, False)
    graph = run_graph_case(m, dt, True)
    assert len(eager) == len(graph) == 4
    for i, (a, b) in enumerate(zip(eager, graph)):
        for k in ("q", "qold", "res", "adt"):
            assert np.array_equal(a[k], b[k]), (i, k)


def test_graph_captured_while_res_is_not_known_zero():
    """Captured after res_calc and bres_calc alone wrote res: the graph
    reads res at every launch and matches the eager chains."""
    m = M.naca0012(30, 40)
    out = []
    for use_graph in (False, True):
        lib = api.lib()
        A = start(m, np.float32)
        A.iterate(1)
        disturb(A)
        if use_graph:
            lib.op2b_res_skips(1)
            assert lib.op2b_capture_begin(0) == 1, api.last_error()
            chain(A)
            h = lib.op2b_capture_end()
            assert h, api.last_error()
            assert lib.op2b_res_skips(1) == 0
            for _ in range(5):
                assert lib.op2b_graph_launch(h) == 0, api.last_error()
            api.sync()
            lib.op2b_graph_destroy(h)
        else:
            for _ in range(5):
                chain(A)
        out.append(finish(A))
    for k in ("q", "qold", "res", "adt"):
        assert np.array_equal(out[0][k], out[1][k]), k
