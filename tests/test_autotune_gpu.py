"""op2b_autotune: the plain path's launch-shape autotuner.

It times its candidates on the app's own data and puts the data back, so a
solve that tunes after its first iteration must end bit-identical to one
that never tuned (the candidates change launch shapes, not the arithmetic or
a cell's order of contributions).  The choice is cached per device, real
type and mesh: a second session finds it without timing.  Without a chain
run first, it refuses."""
import numpy as np
import pytest

from conftest import scratch_dir
from oplus2_matlab_b200 import api, apps
from oplus2_matlab_b200 import mesh as M

pytestmark = pytest.mark.gpu

KNOBS = ("chain_persist", "persist_et", "persist_u", "persist_lag", "fold_variant",
         "flux_ctas_per_sm")
DEFAULTS = {"chain_persist": 0, "persist_et": 1024, "persist_u": 1, "persist_lag": -1,
            "fold_variant": 0, "flux_ctas_per_sm": 16}


def session(m, dt, niter, cache=None, allow_reorder=0):
    """op_init, declare, one iteration, [autotune], niter - 1 more, fetch."""
    lib = api.lib()
    api.op_init([], 0)
    api.set_strategy(api.STRATEGY_GATHER)
    api.set_reduction(api.REDUCE_TREE)
    try:
        A = apps.Airfoil(m, dt)
        A.iterate(1)
        rc, knobs = None, None
        if cache is not None:
            rc = lib.op2b_autotune(cache.encode(), 2, allow_reorder)
            assert rc in (0, 1), api.last_error()
            knobs = {k: lib.op2b_get_tuning(k.encode(), -99) for k in KNOBS}
        A.iterate(niter - 1)
        st = {k: v.copy() for k, v in A.fetch().items()}
        assert api.last_error() == "", api.last_error()
        assert lib.op2b_wait_timeouts(1) == 0
    finally:
        for k, v in DEFAULTS.items():
            lib.op2b_set_tuning(k.encode(), v)
        api.set_strategy(api.STRATEGY_GATHER)
        api.op_exit()
    return rc, knobs, st


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_tuned_solve_bit_identical_and_cached(dt):
    api.set_error_mode(api.ERRORS_RETURN)
    m = M.naca0012(41, 61)
    cache = scratch_dir() + "/tune.txt"
    _, _, ref = session(m, dt, 20)
    rc, knobs, st = session(m, dt, 20, cache)
    assert rc == 0
    for k in ("q", "qold", "res", "adt"):
        assert np.array_equal(st[k], ref[k]), k
    lines = open(cache).read().strip().splitlines()
    assert len(lines) == 1 and lines[0].count("\t") == 2
    rc2, knobs2, st2 = session(m, dt, 20, cache)
    assert rc2 == 1 and knobs2 == knobs  # from the cache, no timing
    for k in ("q", "qold", "res", "adt"):
        assert np.array_equal(st2[k], ref[k]), k


def test_tuning_with_colouring_allowed():
    api.set_error_mode(api.ERRORS_RETURN)
    m = M.naca0012(41, 61)
    _, _, ref = session(m, np.float64, 20)
    rc, _, st = session(m, np.float64, 20, scratch_dir() + "/tune.txt", allow_reorder=1)
    assert rc == 0
    for k in ("q", "qold", "adt"):  # COLOURED, if chosen, reorders the additions only
        assert np.allclose(st[k], ref[k], rtol=1e-12, atol=1e-14), k


def test_autotune_needs_a_chain_first(op2):
    m = M.naca0012(10, 15)
    apps.Airfoil(m, np.float32)
    assert api.lib().op2b_autotune(None, 2, 0) == -1
    assert "run one outer iteration first" in op2.last_error()
    op2.clear_error()
