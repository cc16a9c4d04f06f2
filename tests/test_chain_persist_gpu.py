"""The persistent res_calc chain (one launch: flux tiles and cell tiles from
one dependency-ordered queue, k_chain_persist) against the two-launch chain
(flux pass, then per-cell pass) it replaces:
  - q, qold, res, adt bit-identical after every iteration on meshes whose
    sizes are not multiples of the tiles, FP32 and FP64, for several flux
    tile sizes, cells per thread and queue lags (lag 0 makes nearly every
    cell tile wait for flux tiles still running);
  - the rms within summation order (both are fixed-shape tree sums);
  - no bounded wait ran out (op2b_wait_timeouts);
  - with reductions deferred and the iteration captured as a graph, one
    outer iteration is two launches."""
import numpy as np
import pytest

from conftest import load_golden
from oplus2_matlab_b200 import api, apps
from oplus2_matlab_b200 import mesh as M

pytestmark = pytest.mark.gpu

RK = ("adt_calc", "res_calc", "bres_calc", "update")
DEFAULTS = {"chain_persist": 0, "persist_u": 1, "persist_et": 1024, "persist_lag": -1}


def solve(m, dt, niter, knobs):
    lib = api.lib()
    api.op_init([], 0)
    api.set_strategy(api.STRATEGY_GATHER)
    api.set_reduction(api.REDUCE_TREE)
    for k, v in knobs.items():
        lib.op2b_set_tuning(k.encode(), v)
    try:
        A = apps.Airfoil(m, dt)
        rms = A.iterate(niter)
        st = {k: v.copy() for k, v in A.fetch().items()}
        assert api.last_error() == "", api.last_error()
        assert lib.op2b_wait_timeouts(1) == 0
    finally:
        for k in knobs:
            lib.op2b_set_tuning(k.encode(), DEFAULTS[k])
        api.op_exit()
    return rms, st


@pytest.mark.parametrize("I,J", [(41, 61), (13, 7), (40, 60)])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_persistent_chain_bit_identical_to_two_launches(I, J, dt):
    api.set_error_mode(api.ERRORS_RETURN)
    m = M.naca0012(I, J)
    rms0, st0 = solve(m, dt, 40, {"chain_persist": 0})
    for knobs in ({"chain_persist": 1}, {"chain_persist": 1, "persist_u": 2},
                  {"chain_persist": 1, "persist_et": 256}, {"chain_persist": 1, "persist_et": 4096},
                  {"chain_persist": 1, "persist_lag": 0},
                  {"chain_persist": 1, "persist_lag": 1, "persist_u": 2, "persist_et": 512}):
        rms, st = solve(m, dt, 40, knobs)
        for k in ("q", "qold", "res", "adt"):
            assert np.array_equal(st[k], st0[k]), (knobs, k)
        tol = 5e-6 if dt == np.float32 else 1e-13
        assert np.max(np.abs(rms - rms0) / rms0) < tol, knobs


@pytest.mark.parametrize("case", ["airfoil_40x60_f32", "airfoil_40x60_f64"])
def test_persistent_chain_graph_is_two_launches(op2, case):
    g = load_golden(case)
    m = M.naca0012(g["I"], g["J"])
    dt = np.float32 if g["dtype"] == "f32" else np.float64
    lib = api.lib()
    op2.set_strategy(op2.STRATEGY_GATHER)
    lib.op2b_set_tuning(b"chain_persist", 1)
    A = apps.Airfoil(m, dt)
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
        assert lib.op2b_graph_nkernels(h) == 2
        for _ in range(g["niter"] - 2):
            assert lib.op2b_graph_launch(h) == 0
        for nm in RK[1:] + RK[:-1]:
            A.loop(nm)
        api.sync()
        A.rms[0] = 0
        A.loop("update")
        api.sync()
        lib.op2b_graph_destroy(h)
    finally:
        api.set_gbl_deferred(0)
        lib.op2b_set_tuning(b"chain_persist", 0)
    assert op2.last_error() == ""
    assert lib.op2b_wait_timeouts(1) == 0
    st = A.fetch()
    import hashlib
    for f, key in (("p_q", "q"), ("p_qold", "qold"), ("p_res", "res"), ("p_adt", "adt")):
        assert hashlib.sha256(np.ascontiguousarray(st[key]).tobytes()).hexdigest() == \
            g["final"][f]["sha256"], f
