"""Per-loop timing for op_timing_output (op2b_set_timing).

Call counts are exact in every mode; the sampled mode (default) times a
loop's first call and every 16th call and estimates the total from them, so
its totals track the every-call totals; mode 0 records no device time.
"""
import ctypes as C

import numpy as np
import pytest

from oplus2_matlab_b200 import _lib, apps
from oplus2_matlab_b200 import mesh as M

pytestmark = pytest.mark.gpu


def loop_times(names):
    lib = _lib.load()
    out = {}
    for n in names:
        cnt = C.c_int(0)
        out[n] = (lib.op2b_loop_time(n.encode(), C.byref(cnt)), cnt.value)
    return out


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_counts_exact_and_sampled_totals_track(op2, mode):
    lib = _lib.load()
    old = lib.op2b_set_timing(mode)
    # the loops as called, without the next adt_calc / save_soln run ahead
    # inside the update's launch (tests/test_run_ahead_gpu.py covers that)
    lib.op2b_set_tuning(b"run_ahead", 0)
    try:
        op2.set_strategy(op2.STRATEGY_GATHER)
        A = apps.Airfoil(M.naca0012(40, 60), np.float32)
        A.iterate(48)
        assert op2.last_error() == ""
        t = loop_times(["save_soln+adt_calc", "adt_calc", "res_calc+bres_calc+update"])
        assert t["save_soln+adt_calc"][1] == 48
        assert t["adt_calc"][1] == 48
        assert t["res_calc+bres_calc+update"][1] == 96
        for name, (sec, cnt) in t.items():
            if mode == 0:
                assert sec == 0.0, name
            else:
                assert 0.0 < sec < 1.0, name
                assert sec / cnt < 5e-3, name
    finally:
        lib.op2b_set_timing(old)
        lib.op2b_set_tuning(b"run_ahead", 1)
