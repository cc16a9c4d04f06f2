"""The CPU oracle pinned against the reference's own outputs (tests/golden/,
made by tests/golden/make_golden.py from the reference's seq build)."""
import hashlib

import numpy as np
import pytest

import oracle_lib as O
from conftest import load_golden
from oplus2_matlab_b200 import mesh as M


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def mesh_sha(m):
    h = hashlib.sha256()
    for a in (m.cell, m.edge, m.ecell, m.bedge, m.becell, m.bound, m.x64, m.x32):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("case", ["airfoil_40x60_f32", "airfoil_40x60_f64", "airfoil_40x60s_f32"])
def test_oracle_airfoil_matches_reference(case):
    g = load_golden(case)
    m = M.naca0012(g["I"], g["J"], scramble=g["scramble"])
    assert mesh_sha(m) == g["mesh_sha256"], "mesh generator drifted from the golden mesh"
    dt = np.float32 if g["dtype"] == "f32" else np.float64
    rms, st = O.airfoil(m, dt, g["niter"])
    for it, val in g["rms"]:
        assert rms[it - 1] == dt(val), (it, rms[it - 1], val)
    for f, key in (("p_q", "q"), ("p_qold", "qold"), ("p_res", "res"), ("p_adt", "adt")):
        assert sha(st[key]) == g["final"][f]["sha256"], f


@pytest.mark.parametrize("case", ["jac1_nn6", "jac2_nn6", "jac1_nn64", "jac2_nn64"])
def test_oracle_jac_matches_reference(case):
    g = load_golden(case)
    jm = M.jac(g["NN"], g["variant"])
    hist, u = O.jac(jm, g["variant"], g["niter"])
    for (um, us), (gm, grms) in zip(hist, g["u_max_rms"]):
        assert np.float32(um) == np.float32(gm)
        assert np.float32(np.sqrt(np.float32(us) / np.float32(jm.nnode))) == np.float32(grms)
    assert sha(u) == g["u_sha256"]


def test_jac1_known_answer():
    # jac1 at NN=6 after 2 iterations: exactly representable u field
    g = load_golden("jac1_nn6")
    u = np.array(g["u"], np.float32).reshape(5, 5)
    assert u[0].tolist() == [0.625, 0.4375, 0.375, 0.4375, 0.625]
    assert u[2, 2] == 0.0
    assert g["u_max_rms"][-1][0] == 0.625


def _airfoil_specs(m, real=4):
    R, INC = 0, 3
    e2n, e2c, b2n, b2c, c2n = m.edge, m.ecell, m.bedge, m.becell.reshape(-1, 1), m.cell
    return {
        "res_calc": O.LoopSpec(m.nedge, [(e2n, 2, 0, m.nnode, 2 * real, R), (e2n, 2, 1, m.nnode, 2 * real, R),
                                         (e2c, 2, 0, m.ncell, 4 * real, R), (e2c, 2, 1, m.ncell, 4 * real, R),
                                         (e2c, 2, 0, m.ncell, real, R), (e2c, 2, 1, m.ncell, real, R),
                                         (e2c, 2, 0, m.ncell, 4 * real, INC), (e2c, 2, 1, m.ncell, 4 * real, INC)],
                               [0, 0, 1, 1, 2, 2, 3, 3]),
        "adt_calc": O.LoopSpec(m.ncell, [(c2n, 4, 0, m.nnode, 2 * real, R), (c2n, 4, 1, m.nnode, 2 * real, R),
                                         (c2n, 4, 2, m.nnode, 2 * real, R), (c2n, 4, 3, m.nnode, 2 * real, R),
                                         (None, 0, -1, m.ncell, 4 * real, R), (None, 0, -1, m.ncell, real, 1)],
                               [0, 0, 0, 0, -1, -1]),
        "bres_calc": O.LoopSpec(m.nbedge, [(b2n, 2, 0, m.nnode, 2 * real, R), (b2n, 2, 1, m.nnode, 2 * real, R),
                                           (b2c, 1, 0, m.ncell, 4 * real, R), (b2c, 1, 0, m.ncell, real, R),
                                           (b2c, 1, 0, m.ncell, 4 * real, INC), (None, 0, -1, m.nbedge, 4, R)],
                                [0, 0, 1, 2, 3, -1]),
    }


def test_oracle_plans_match_reference():
    plans = load_golden("plans")
    meshes = {"40x60": M.naca0012(40, 60), "40x60s": M.naca0012(40, 60, scramble=True)}
    specs = {k: _airfoil_specs(m) for k, m in meshes.items()}
    jm = M.jac(64, 1)
    specs["jac1_nn64"] = {"res": O.LoopSpec(jm.nedge, [(None, 0, -1, jm.nedge, 4, 0),
                                                       (jm.pp, 2, 1, jm.nnode, 4, 0),
                                                       (jm.pp, 2, 0, jm.nnode, 4, 3)], [-1, 0, 1])}
    assert len(plans) >= 10
    for g in plans:
        if "mesh_sha256" in g:
            assert mesh_sha(meshes[g["mesh"]]) == g["mesh_sha256"]
        spec = specs[g["mesh"]][g["loop"]]
        p, checks, colours = O.plan_core(spec, g["part_size"])
        try:
            assert (p["nblocks"], p["ncolors"], p["nshared"]) == (g["nblocks"], g["ncolors"], g["nshared"]), g["case"]
            for key, rec in g["arrays"].items():
                assert sha(p[key]) == rec["sha256"], (g["case"], key)
            # the reference accumulates its byte models in float
            assert abs(p["transfer"] - g["transfer"]) <= 1e-6 * g["transfer"]
            assert abs(p["transfer2"] - g["transfer2"]) <= 1e-6 * g["transfer2"]
            assert checks == 0 and colours == 0, g["case"]
        finally:
            O.plan_free(p)


def test_plan_checker_detects_planted_colouring_error():
    """Plant a colouring conflict in an oracle plan (CPU only) and check the
    colour validator sees it -- the validator the device checker mirrors."""
    import ctypes as C
    m = M.naca0012(40, 60)
    spec = _airfoil_specs(m)["res_calc"]
    p, checks, colours = O.plan_core(spec, 0)
    try:
        assert colours == 0
        plan = p["_plan"]
        thr = np.ctypeslib.as_array(C.cast(plan.thrcol, C.POINTER(C.c_int)), shape=(m.nedge,))
        # edges 0 and 1 share cell 0 (both are edges of cell (0,0)) in block 0
        shared = set(m.ecell[0]) & set(m.ecell[1])
        assert shared
        thr[1] = thr[0]
        mp, dims, idxs, tos, ds, acc, ii = spec.c_arrays()
        bad = O.load().op2o_plan_check_colours(C.byref(plan), mp, dims, idxs, tos, acc, ii)
        assert bad > 0
    finally:
        O.plan_free(p)
