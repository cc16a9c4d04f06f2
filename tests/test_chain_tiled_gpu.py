"""The tiled res_calc chain (one launch, no wait between CTAs: each CTA
computes the fluxes of its tile of cells into shared memory -- edges between
tiles on both sides -- then folds, updates and runs adt_calc on the tile's
cells, writing q and adt to second buffers; k_chain_tiled) against the
two-launch chain (flux pass, then per-cell pass) it replaces:
  - q, qold, res, adt bit-identical after every iteration, FP32 and FP64, on
    meshes whose sizes are not multiples of the tiles, for CTAs of 1024 and
    512 threads and tile sizes from 64 cells to one tile for the mesh;
  - the rms: within summation order in TREE mode, bit-identical in SEQ mode;
  - captured as a graph: one launch per chain, and a graph holding an odd
    number of chains (which swaps the buffers an odd number of times) gives
    the same fields when launched again and again."""
import hashlib

import numpy as np
import pytest

from conftest import load_golden
from oplus2_matlab_b200 import api, apps
from oplus2_matlab_b200 import mesh as M

pytestmark = pytest.mark.gpu

RK = ("adt_calc", "res_calc", "bres_calc", "update")
DEFAULTS = {"chain_tiled": 0, "tile_threads": 1024, "tile_cells": 0}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def solve(m, dt, niter, knobs, reduction=None):
    lib = api.lib()
    api.op_init([], 0)
    api.set_strategy(api.STRATEGY_GATHER)
    api.set_reduction(reduction if reduction is not None else api.REDUCE_TREE)
    for k, v in knobs.items():
        lib.op2b_set_tuning(k.encode(), v)
    try:
        lib.op2b_tiled_launches(1)
        A = apps.Airfoil(m, dt)
        rms = A.iterate(niter)
        st = {k: v.copy() for k, v in A.fetch().items()}
        assert api.last_error() == "", api.last_error()
        # the tiled chain ran (it is skipped when a run-ahead flux pass has
        # done the next chain's fluxes, so not at every chain)
        assert (lib.op2b_tiled_launches(1) > 0) == bool(knobs.get("chain_tiled", 0))
    finally:
        for k in knobs:
            lib.op2b_set_tuning(k.encode(), DEFAULTS[k])
        api.set_reduction(api.REDUCE_TREE)
        api.op_exit()
    return rms, st


@pytest.mark.parametrize("I,J", [(41, 61), (13, 7), (40, 60)])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_tiled_chain_bit_identical_to_two_launches(I, J, dt):
    api.set_error_mode(api.ERRORS_RETURN)
    m = M.naca0012(I, J)
    rms0, st0 = solve(m, dt, 40, {"chain_tiled": 0})
    for knobs in ({"chain_tiled": 1}, {"chain_tiled": 1, "tile_threads": 512},
                  {"chain_tiled": 1, "tile_cells": 64}, {"chain_tiled": 1, "tile_cells": 333},
                  {"chain_tiled": 1, "tile_cells": 1 << 20},
                  {"chain_tiled": 1, "tile_threads": 512, "tile_cells": 97}):
        rms, st = solve(m, dt, 40, knobs)
        for k in ("q", "qold", "res", "adt"):
            assert np.array_equal(st[k], st0[k]), (knobs, k)
        tol = 5e-6 if dt == np.float32 else 1e-13
        assert np.max(np.abs(rms - rms0) / rms0) < tol, knobs


@pytest.mark.parametrize("case", ["airfoil_40x60_f32", "airfoil_40x60s_f32"])
def test_tiled_chain_seq_rms_matches_reference(case):
    g = load_golden(case)
    api.set_error_mode(api.ERRORS_RETURN)
    m = M.naca0012(g["I"], g["J"], scramble=g["scramble"])
    rms, st = solve(m, np.float32, g["niter"], {"chain_tiled": 1}, reduction=api.REDUCE_SEQ)
    for f, key in (("p_q", "q"), ("p_qold", "qold"), ("p_res", "res"), ("p_adt", "adt")):
        assert sha(st[key]) == g["final"][f]["sha256"], f
    for it, val in g["rms"]:
        assert rms[it - 1] == np.float32(val), (it, rms[it - 1], val)


@pytest.mark.parametrize("case", ["airfoil_40x60_f32", "airfoil_40x60_f64"])
def test_tiled_chain_graph_is_two_launches(op2, case):
    g = load_golden(case)
    m = M.naca0012(g["I"], g["J"])
    dt = np.float32 if g["dtype"] == "f32" else np.float64
    lib = api.lib()
    op2.set_strategy(op2.STRATEGY_GATHER)
    lib.op2b_set_tuning(b"chain_tiled", 1)
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
        lib.op2b_graph_destroy(h)
        for nm in RK[1:] + RK[:-1]:
            A.loop(nm)
        api.sync()
        A.rms[0] = 0
        A.loop("update")
        api.sync()
    finally:
        api.set_gbl_deferred(0)
        lib.op2b_set_tuning(b"chain_tiled", 0)
    assert op2.last_error() == ""
    st = A.fetch()
    for f, key in (("p_q", "q"), ("p_qold", "qold"), ("p_res", "res"), ("p_adt", "adt")):
        assert sha(st[key]) == g["final"][f]["sha256"], f


def test_tiled_chain_graph_with_one_chain_replays():
    """A graph of one chain (res_calc, bres_calc, update, adt_calc) swaps q and
    adt once; the capture ends with a copy back, so every launch starts from
    the buffers the host holds.  Fields after K launches equal K eager runs."""
    api.set_error_mode(api.ERRORS_RETURN)
    m = M.naca0012(40, 60)
    lib = api.lib()
    chain = ("res_calc", "bres_calc", "update", "adt_calc")

    def run(tiled, graph):
        api.op_init([], 0)
        api.set_strategy(api.STRATEGY_GATHER)
        lib.op2b_set_tuning(b"chain_tiled", tiled)
        A = apps.Airfoil(m, np.float32)
        api.set_gbl_deferred(1)
        try:
            for nm in ("save_soln", "adt_calc") + chain:  # plans built before the capture
                A.loop(nm)
            api.sync()
            if graph:
                assert lib.op2b_capture_begin(0) == 1, api.last_error()
                for nm in chain:
                    A.loop(nm)
                h = lib.op2b_capture_end()
                assert h, api.last_error()
                assert lib.op2b_graph_nkernels(h) == (1 if tiled else 2)
                for _ in range(7):
                    assert lib.op2b_graph_launch(h) == 0
                api.sync()
                lib.op2b_graph_destroy(h)
            else:
                for _ in range(7):
                    for nm in chain:
                        A.loop(nm)
                api.sync()
            # an eager chain after the graph sees the graph's results
            for nm in chain:
                A.loop(nm)
            api.sync()
            st = {k: v.copy() for k, v in A.fetch().items()}
            assert api.last_error() == "", api.last_error()
        finally:
            api.set_gbl_deferred(0)
            lib.op2b_set_tuning(b"chain_tiled", 0)
            api.op_exit()
        return st

    ref = run(0, False)
    for tiled, graph in ((1, False), (1, True), (0, True)):
        st = run(tiled, graph)
        for k in ("q", "qold", "res", "adt"):
            assert np.array_equal(st[k], ref[k]), (tiled, graph, k)


@pytest.mark.parametrize("order", ["cm", "rcb"])
def test_tiled_chain_on_renumbered_scrambled_mesh_matches_reference(order):
    """The tiled chain over renumbered sets (its tiles are ranges of the new
    cell order): fields and SEQ rms bit-identical to the reference on the
    scrambled mesh."""
    from oplus2_matlab_b200 import _lib
    g = load_golden("airfoil_40x60s_f32")
    api.set_error_mode(api.ERRORS_RETURN)
    m = M.naca0012(g["I"], g["J"], scramble=g["scramble"])
    lib = api.lib()
    api.op_init([], 0)
    api.set_strategy(api.STRATEGY_GATHER)
    api.set_reduction(api.REDUCE_SEQ)
    lib.op2b_set_tuning(b"chain_tiled", 1)
    try:
        assert _lib.load().op2b_set_renumber(1) == 0
        A = apps.Airfoil(m, np.float32)
        if order == "rcb":
            assert _lib.load().op2b_set_renumber_coords(A.p_x) == 0
        lib.op2b_tiled_launches(1)
        rms = A.iterate(g["niter"])
        st = {k: v.copy() for k, v in A.fetch().items()}
        assert api.last_error() == "", api.last_error()
        assert lib.op2b_tiled_launches(1) > 0
    finally:
        lib.op2b_set_tuning(b"chain_tiled", 0)
        api.set_reduction(api.REDUCE_TREE)
        api.op_exit()
    for f, key in (("p_q", "q"), ("p_qold", "qold"), ("p_res", "res"), ("p_adt", "adt")):
        assert sha(st[key]) == g["final"][f]["sha256"], f
    for it, val in g["rms"]:
        assert rms[it - 1] == np.float32(val), (it, rms[it - 1], val)
