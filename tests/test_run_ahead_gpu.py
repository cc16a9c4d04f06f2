"""Loops run ahead of their calls.  With reductions returned at every call
(the reference's semantics), an update cannot wait for the adt_calc that
follows it, so its per-cell pass computes that adt_calc (and, at the end of
an outer iteration, the next save_soln) into spare buffers, swapped in when
the matching call comes; the next res_calc + bres_calc's flux pass is
queued behind it.  Whatever the app calls instead, every dataset must
read exactly as it would without run-ahead: each sequence below runs twice,
with the "run_ahead" knob on and off, and every field is compared bit for
bit at each fetch and at the end."""
import ctypes as C

import numpy as np
import pytest

from oplus2_matlab_b200 import _lib, api, apps
from oplus2_matlab_b200 import mesh as M

pytestmark = pytest.mark.gpu

IT = ["save_soln"] + ["adt_calc", "res_calc", "bres_calc", "update"] * 2

SEQUENCES = {
    # the app's own order: adt_calc and save_soln are committed from run-ahead
    "airfoil": IT * 4,
    # a fetch of adt between the update and its adt_calc sees the old adt
    "fetch_between": IT * 2 + ["adt_calc", "res_calc", "bres_calc", "update", "fetch",
                               "adt_calc", "fetch"] + IT,
    # the adt_calc never comes: res_calc reads the old adt
    "skip_adt": IT + ["adt_calc", "res_calc", "bres_calc", "update", "res_calc", "bres_calc",
                      "update"] + IT,
    # save_soln comes, then not adt_calc
    "save_then_other": IT * 2 + ["save_soln", "res_calc", "bres_calc", "update"] + IT,
    # the constants change between the update and its adt_calc
    "const_change": IT * 2 + ["cfl"] + ["adt_calc", "res_calc", "bres_calc", "update"] + IT,
    # adt_calc twice, save_soln twice
    "repeats": IT * 2 + ["save_soln", "save_soln", "adt_calc", "adt_calc"] + IT,
    # the next res_calc's flux pass also runs ahead: res_calc called twice,
    # bres_calc skipped, a fetch between res_calc and bres_calc
    "res_twice": IT * 2 + ["adt_calc", "res_calc", "res_calc", "bres_calc", "update"] + IT,
    "bres_skipped": IT * 2 + ["adt_calc", "res_calc", "update"] + IT,
    "fetch_in_chain": IT * 2 + ["adt_calc", "res_calc", "fetch", "bres_calc", "update"] + IT,
}


def run(op2, seq, ahead, dt):
    lib = _lib.load()
    lib.op2b_set_tuning(b"run_ahead", 1 if ahead else 0)
    op2.set_strategy(op2.STRATEGY_GATHER)
    op2.set_reduction(op2.REDUCE_TREE)
    A = apps.Airfoil(M.naca0012(30, 45, scramble=True), dt)
    snaps, rms = [], []
    try:
        for step in seq:
            if step == "fetch":
                snaps.append({k: v.copy() for k, v in A.fetch().items()})
            elif step == "cfl":
                api.op_decl_const("cfl", 1, A.tn, A.dtype.type(0.8))
            else:
                if step == "update":
                    A.rms[0] = 0
                A.loop(step)
                if step == "update":
                    rms.append(A.rms[0])
        snaps.append({k: v.copy() for k, v in A.fetch().items()})
    finally:
        lib.op2b_set_tuning(b"run_ahead", 1)
    assert op2.last_error() == ""
    return snaps, np.array(rms)


def loop_count(name):
    cnt = C.c_int(0)
    _lib.load().op2b_loop_time(name.encode(), C.byref(cnt))
    return cnt.value


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("seq", sorted(SEQUENCES))
def test_same_fields_with_and_without_run_ahead(op2, seq, dt):
    with_ahead, rms_a = run(op2, SEQUENCES[seq], True, dt)
    api.op_exit()
    api.op_init([], 0)
    without, rms_b = run(op2, SEQUENCES[seq], False, dt)
    assert np.array_equal(rms_a, rms_b)
    assert len(with_ahead) == len(without)
    for a, b in zip(with_ahead, without):
        for k in ("q", "qold", "adt", "res"):
            assert np.array_equal(a[k], b[k]), (seq, k)


def test_run_ahead_replaces_the_calls(op2):
    """In the app's order, after the first iteration every adt_calc and
    save_soln comes from the update before it: the fused launches run and
    the separate kernels do not."""
    run(op2, IT * 6, True, np.float32)
    assert loop_count("res_calc+bres_calc+update+adt_calc") >= 6
    assert loop_count("res_calc+bres_calc+update+save_soln+adt_calc") >= 4
    assert loop_count("save_soln+adt_calc") <= 2
    assert loop_count("adt_calc") <= 2


JAC_SEQUENCES = {
    "plain": ["iter"] * 12,
    # a fetch between update and res, then beta changed before a res
    "fetch_and_beta": ["iter"] * 4 + ["update", "fetch", "res", "update", "beta", "res",
                                      "update"] + ["iter"] * 3,
    # update twice, res twice
    "repeats": ["iter"] * 3 + ["update", "update", "res", "res", "update"] + ["iter"] * 2,
}


def run_jac(op2, seq, ahead, variant, reduction=None):
    lib = _lib.load()
    lib.op2b_set_tuning(b"run_ahead", 1 if ahead else 0)
    op2.set_strategy(op2.STRATEGY_GATHER)
    op2.set_reduction(op2.REDUCE_TREE if reduction is None else reduction)
    J = apps.Jac(M.jac(40, variant), variant)
    out, snaps = [], []

    def update():
        J.u_sum[0] = 0
        J.u_max[0] = 0
        api.op_par_loop("update", J.nodes, *J.upd_args)
        out.append((float(J.u_sum[0]), float(J.u_max[0])))
    try:
        for step in seq:
            if step == "iter":
                api.op_par_loop("res", J.edges, *J.res_args)
                update()
            elif step == "res":
                api.op_par_loop("res", J.edges, *J.res_args)
            elif step == "update":
                update()
            elif step == "beta":
                J.beta[0] = np.float32(0.75)
            elif step == "fetch":
                api.op_fetch_data(J.p_du)
                snaps.append((J.fetch().copy(), J.du.copy()))
        api.op_fetch_data(J.p_du)
        snaps.append((J.fetch().copy(), J.du.copy()))
    finally:
        lib.op2b_set_tuning(b"run_ahead", 1)
    assert op2.last_error() == ""
    return out, snaps


@pytest.mark.parametrize("variant", [1, 2])
@pytest.mark.parametrize("seq", sorted(JAC_SEQUENCES))
@pytest.mark.parametrize("reduction", ["tree", "seq"])
def test_jac_same_results_with_and_without_run_ahead(op2, seq, variant, reduction):
    """u and du bit-identical at every snapshot, u_max and u_sum exact, in
    TREE and in SEQ mode."""
    red = op2.REDUCE_TREE if reduction == "tree" else op2.REDUCE_SEQ
    a_out, a_snaps = run_jac(op2, JAC_SEQUENCES[seq], True, variant, red)
    api.op_exit()
    api.op_init([], 0)
    b_out, b_snaps = run_jac(op2, JAC_SEQUENCES[seq], False, variant, red)
    assert len(a_out) == len(b_out)
    for (sa, ma), (sb, mb) in zip(a_out, b_out):
        assert ma == mb and sa == sb
    for (ua, dua), (ub, dub) in zip(a_snaps, b_snaps):
        assert np.array_equal(ua, ub) and np.array_equal(dua, dub)
