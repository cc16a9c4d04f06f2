"""Deferred reductions and CUDA graphs against the reference's sequential
build.  With reductions deferred, the library holds loops back and runs them
fused: save_soln+adt_calc, res_calc+bres_calc+update+adt_calc, and across
the outer-iteration boundary res_calc+bres_calc+update+save_soln+adt_calc
(one flux pass, one per-cell pass).  The fused chains must leave every field
bit-identical to op_seq.h after the reference's 1000 iterations, called one
by one or replayed from a captured graph of the steady-state iteration."""
import hashlib

import numpy as np
import pytest

from conftest import load_golden
from oplus2_matlab_b200 import api, apps
from oplus2_matlab_b200 import mesh as M

pytestmark = pytest.mark.gpu

RK = ("adt_calc", "res_calc", "bres_calc", "update")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def check(g, A, dt):
    st = A.fetch()
    for f, key in (("p_q", "q"), ("p_qold", "qold"), ("p_res", "res"), ("p_adt", "adt")):
        assert sha(st[key]) == g["final"][f]["sha256"], f
    rms = float(np.sqrt(A.rms[0] / dt(A.mesh.ncell)))
    want = g["rms"][-1][1]
    tol = 5e-5 if dt == np.float32 else 1e-12  # TREE: summation order only
    assert abs(rms - want) / want < tol, (rms, want)


def last_update(A):
    """The run's last update, its rms alone: deferred OP_INC results add to
    the host value when delivered, so deliver the earlier ones first."""
    api.sync()
    A.rms[0] = 0
    A.loop("update")


def setup(op2, case):
    g = load_golden(case)
    m = M.naca0012(g["I"], g["J"], scramble=g["scramble"])
    dt = np.float32 if g["dtype"] == "f32" else np.float64
    op2.set_strategy(op2.STRATEGY_GATHER)
    op2.set_reduction(op2.REDUCE_TREE)
    return g, m, dt


@pytest.mark.parametrize("case", ["airfoil_40x60_f32", "airfoil_40x60_f64", "airfoil_40x60s_f32"])
def test_deferred_loop_calls(op2, case):
    g, m, dt = setup(op2, case)
    api.set_gbl_deferred(1)
    try:
        A = apps.Airfoil(m, dt)
        for it in range(g["niter"]):
            A.loop("save_soln")
            for k in range(2):
                for nm in RK:
                    if nm == "update" and it == g["niter"] - 1 and k == 1:
                        last_update(A)
                    else:
                        A.loop(nm)
        api.sync()
        assert op2.last_error() == ""
        check(g, A, dt)
    finally:
        api.set_gbl_deferred(0)


@pytest.mark.parametrize("case,fold_variant", [("airfoil_40x60_f32", 0), ("airfoil_40x60_f64", 0),
                                               ("airfoil_40x60_f32", 4), ("airfoil_40x60_f32", 5),
                                               ("airfoil_40x60_f64", 5)])
def test_graph_of_rotated_iteration(op2, case, fold_variant):
    """The first iteration as loop calls (they build the plans, which a
    capture cannot), then a graph of res_calc, bres_calc, update, adt_calc,
    res_calc, bres_calc, update, save_soln, adt_calc (one outer iteration,
    rotated so that the next iteration's first loops fuse with this one's
    last update) replayed niter - 2 times, then the last iteration's
    remaining loops.  Every per-cell pass form that takes save_soln
    (fold_variant 0, 4, 5) gives the same fields."""
    g, m, dt = setup(op2, case)
    lib = api.lib()
    A = apps.Airfoil(m, dt)
    lib.op2b_set_tuning(b"fold_variant", fold_variant)
    api.set_gbl_deferred(1)
    try:
        for nm in ("save_soln",) + RK + RK + ("save_soln", "adt_calc"):
            A.loop(nm)
        api.sync()
        assert lib.op2b_capture_begin(0) == 1, op2.last_error()
        for nm in RK[1:] + RK + ("save_soln", "adt_calc"):
            A.loop(nm)
        h = lib.op2b_capture_end()
        assert h, op2.last_error()
        # res_calc+bres_calc+update+adt_calc and
        # res_calc+bres_calc+update+save_soln+adt_calc, two launches each
        assert lib.op2b_graph_nkernels(h) == 4
        for _ in range(g["niter"] - 2):
            assert lib.op2b_graph_launch(h) == 0
        for nm in RK[1:] + RK[:-1]:
            A.loop(nm)
        last_update(A)
        api.sync()
        lib.op2b_graph_destroy(h)
    finally:
        api.set_gbl_deferred(0)
        lib.op2b_set_tuning(b"fold_variant", 0)
    assert op2.last_error() == ""
    assert lib.op2b_wait_timeouts(1) == 0
    check(g, A, dt)
