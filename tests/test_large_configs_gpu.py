"""Full-size configurations beyond the default path's own parity test:

  - the device plan builder against the reference's op_plan_core at 720k
    cells (res_calc, adt_calc, bres_calc; part sizes 0, 64, 256) and on the
    2.88M-cell scrambled mesh (part sizes 0, 256): every array equal (SHA-256
    of the reference's arrays, tests/golden/plans_large.json), and the
    device validator, colourings included, finds nothing;
  - COLOURED (the reference's two-level colouring scheme) at 720k FP64 for
    1000 iterations against the reference's sequential build: every printed
    rms and the final fields within 1e-12 relative;
  - renumbering on the 2.88M scrambled mesh: final fields hash to the
    reference's (contributions keep the app's element order);
  - the TREE rms against the exact sum: at every printed iteration the rms
    is recomputed from the update's own inputs (res and adt, read back just
    before the update) -- once as op_seq.h's one-at-a-time float sum, which
    must reproduce the reference's printed value bit for bit, and once
    exactly (float64).  The GPU's TREE rms must be no farther from the exact
    value than op_seq.h's own sum is.

Goldens: tests/golden/make_golden.py --large --large-plans (reference
binaries built from its sources by oracle/Makefile).
"""
import hashlib
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from oplus2_matlab_b200 import _lib, api, apps
from oplus2_matlab_b200 import mesh as M

pytestmark = [pytest.mark.gpu, pytest.mark.large]

INDS = {"res_calc": [0, 0, 1, 1, 2, 2, 3, 3], "adt_calc": [0, 0, 0, 0, -1, -1],
        "bres_calc": [0, 0, 1, 2, 3, -1]}
MESHES = {"400x600": (400, 600, False), "800x1200s": (800, 1200, True)}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def need(case):
    if not os.path.exists(os.path.join(GOLDEN, case + ".json")):
        pytest.fail("golden fixture %s missing (tests/golden/make_golden.py --large)" % case)
    return load_golden(case)


_mesh_cache = {}


def mesh(tag):
    if tag not in _mesh_cache:
        I, J, scr = MESHES[tag]
        _mesh_cache[tag] = M.naca0012(I, J, scramble=scr)
    return _mesh_cache[tag]


def large_plans():
    p = os.path.join(GOLDEN, "plans_large.json")
    return load_golden("plans_large") if os.path.exists(p) else []


@pytest.mark.parametrize("tag", list(MESHES))
def test_device_plans_equal_reference_full_size(op2, tag):
    plans = [g for g in large_plans() if g["mesh"] == tag]
    assert plans, "tests/golden/plans_large.json missing (make_golden.py --large-plans)"
    m = mesh(tag)
    A = apps.Airfoil(m, np.float32)
    for g in plans:
        s, args = A.loops[g["loop"]]
        inds = INDS[g["loop"]]
        p = op2.op_plan_core(g["loop"], s, g["part_size"], args, inds)
        assert p, op2.last_error()
        got = op2.plan_arrays(p, args, inds)
        assert (got["nblocks"], got["ncolors"], got["nshared"]) == \
            (g["nblocks"], g["ncolors"], g["nshared"]), g["case"]
        for key, rec in g["arrays"].items():
            assert got[key].size == rec["n"], (g["case"], key)
            assert sha(got[key]) == rec["sha256"], (g["case"], key)
        # the byte models: summed exactly here, in float one term at a time
        # by the reference (common/op_lib_core.c:989-1056), so they differ
        # by at most that sum's rounding, (number of terms) x 2^-24 relative
        ninds = max(inds) + 1
        terms = got["nblocks"] * (len(args) + 3 * ninds) + 2 * int(np.sum(got["ind_sizes"]))
        for key in ("transfer", "transfer2"):
            assert abs(got[key] - g[key]) <= terms * 2.0 ** -24 * g[key], (g["case"], key)
        assert op2.op_plan_validate(g["loop"], s, g["part_size"], args, inds) == 0, g["case"]


def test_coloured_720k_fp64_against_reference(op2):
    g = need("airfoil_400x600_f64")
    m = mesh("400x600")
    op2.set_strategy(op2.STRATEGY_COLOURED)
    op2.set_reduction(op2.REDUCE_TREE)
    A = apps.Airfoil(m, np.float64)
    rms = A.iterate(g["niter"])
    st = A.fetch()
    assert op2.last_error() == ""
    for it, val in g["rms"]:
        assert abs(float(rms[it - 1]) - val) <= 1e-12 * val, (it, float(rms[it - 1]), val)
    for f, key in (("p_q", "q"), ("p_qold", "qold"), ("p_adt", "adt")):
        ref = g["final"][f]
        got = st[key].ravel()
        assert abs(float(got.sum()) - ref["sum"]) <= 1e-12 * abs(ref["sum"]), f
        first = np.array(ref["first"])  # relative to the field's scale (some are ~1e-16)
        assert np.all(np.abs(got[:8] - first) <= 1e-12 * np.abs(first).max()), f


def test_renumbered_scrambled_2880k_matches_reference(op2):
    g = need("airfoil_800x1200s_f32")
    m = mesh("800x1200s")
    op2.set_strategy(op2.STRATEGY_GATHER)
    op2.set_reduction(op2.REDUCE_TREE)
    assert _lib.load().op2b_set_renumber(1) == 0
    A = apps.Airfoil(m, np.float32)
    rms = A.iterate(g["niter"])
    st = A.fetch()
    assert op2.last_error() == ""
    for f, key in (("p_q", "q"), ("p_qold", "qold"), ("p_res", "res"), ("p_adt", "adt")):
        assert sha(st[key]) == g["final"][f]["sha256"], f
    ref = np.array([v for _, v in g["rms"]])
    got = np.array([rms[it - 1] for it, _ in g["rms"]], np.float64)
    assert np.max(np.abs(got - ref) / ref) < 5e-4


def rms_errors(case):
    """Per printed iteration: the default path's TREE rms, op_seq.h's serial
    float rms recomputed from the update's inputs, and the exact rms."""
    g = need(case)
    m = mesh("%dx%d%s" % (g["I"], g["J"], "s" if g["scramble"] else ""))
    f32 = np.float32
    api.set_strategy(api.STRATEGY_GATHER)
    api.set_reduction(api.REDUCE_TREE)
    A = apps.Airfoil(m, f32)           # the default, fused path
    tree = A.iterate(g["niter"])
    qa = A.fetch()["q"].copy()
    B = apps.Airfoil(m, f32)           # the same solve, read back at printed iterations
    printed = {it for it, _ in g["rms"]}
    nc = f32(m.ncell)
    rows = []
    for it in range(1, g["niter"] + 1):
        B.loop("save_soln")
        for k in range(2):
            for nm in ("adt_calc", "res_calc", "bres_calc"):
                B.loop(nm)
            if k == 1 and it in printed:
                api.op_fetch_data(B.p_res)
                api.op_fetch_data(B.p_adt)
                # airfoil/update.h:1-12, in float32 as the reference computes it
                adti = f32(1.0) / B.adt[:, 0]
                d = adti[:, None] * B.res
                sq = (d * d).ravel()
                serial = np.cumsum(sq, dtype=f32)[-1]          # op_seq.h's order
                seq_rms = np.sqrt(f32(serial) / nc)
                exact = math.sqrt(math.fsum(sq.astype(np.float64)) / m.ncell)
                rows.append((it, float(tree[it - 1]), float(seq_rms), exact))
            B.rms[0] = 0
            B.loop("update")
    qb = B.fetch()["q"]
    assert api.last_error() == ""
    assert np.array_equal(qa, qb)  # both solves moved the same fields
    return g, m, rows


@pytest.mark.parametrize("case", ["airfoil_400x600_f32", "airfoil_800x1200s_f32"])
def test_tree_rms_no_farther_from_exact_than_op_seq(op2, case):
    g, m, rows = rms_errors(case)
    golden = dict((it, v) for it, v in g["rms"])
    u = 2.0 ** -24
    bound = math.sqrt(4 * m.ncell) * u   # sqrt(N) u, N = 4 squares per cell
    tree_err, seq_err = [], []
    for it, tree, seq, exact in rows:
        # the recomputed serial sum is the reference's printed value, bit for bit
        assert np.float32(seq) == np.float32(golden[it]), (it, seq, golden[it])
        tree_err.append(abs(tree - exact) / exact)
        seq_err.append(abs(seq - exact) / exact)
    tree_err, seq_err = np.array(tree_err), np.array(seq_err)
    print("\n%s: rel. error from the exact rms over %d printed iterations: TREE max %.3e mean "
          "%.3e; op_seq.h max %.3e mean %.3e; sqrt(N)u %.3e"
          % (case, len(rows), tree_err.max(), tree_err.mean(), seq_err.max(), seq_err.mean(), bound))
    assert tree_err.max() <= bound
    assert tree_err.max() <= seq_err.max()
    assert tree_err.mean() <= seq_err.mean()
