"""The device-built execution plan against the reference's op_plan_core:
bit-exact arrays (goldens from the reference itself, and the CPU oracle on
further meshes and part sizes), zero colouring violations."""
import hashlib

import numpy as np
import pytest

import oracle_lib as O
from conftest import load_golden
from oplus2_matlab_b200 import apps
from oplus2_matlab_b200 import mesh as M

pytestmark = pytest.mark.gpu

INDS = {"res_calc": [0, 0, 1, 1, 2, 2, 3, 3], "adt_calc": [0, 0, 0, 0, -1, -1],
        "bres_calc": [0, 0, 1, 2, 3, -1]}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_device_plans_equal_reference_goldens(op2):
    plans = [g for g in load_golden("plans") if g["loop"] in INDS]
    meshes = {"40x60": M.naca0012(40, 60), "40x60s": M.naca0012(40, 60, scramble=True)}
    apps_ = {k: apps.Airfoil(m, np.float32) for k, m in meshes.items()}
    for g in plans:
        A = apps_[g["mesh"]]
        s, args = A.loops[g["loop"]]
        inds = INDS[g["loop"]]
        p = op2.op_plan_core(g["loop"], s, g["part_size"], args, inds)
        assert p, op2.last_error()
        got = op2.plan_arrays(p, args, inds)
        assert (got["nblocks"], got["ncolors"], got["nshared"]) == (g["nblocks"], g["ncolors"], g["nshared"])
        for key, rec in g["arrays"].items():
            assert sha(got[key]) == rec["sha256"], (g["case"], key)
        assert abs(got["transfer"] - g["transfer"]) <= 1e-6 * g["transfer"]
        assert abs(got["transfer2"] - g["transfer2"]) <= 1e-6 * g["transfer2"]
        assert op2.op_plan_validate(g["loop"], s, g["part_size"], args, inds) == 0


def test_device_plan_jac_res_equals_reference(op2):
    from oplus2_matlab_b200 import apps as A_
    for g in [g for g in load_golden("plans") if g["loop"] == "res"]:
        J = A_.Jac(M.jac(64, 1), 1)
        inds = [-1, 0, 1, -1]
        p = op2.op_plan_core("res", J.edges, g["part_size"], J.res_args, inds)
        got = op2.plan_arrays(p, J.res_args, inds)
        assert (got["nblocks"], got["ncolors"], got["nshared"]) == (g["nblocks"], g["ncolors"], g["nshared"])
        for key, rec in g["arrays"].items():
            assert sha(got[key]) == rec["sha256"], (g["case"], key)
        assert op2.op_plan_validate("res", J.edges, g["part_size"], J.res_args, inds) == 0
        op2.op_exit()
        op2.op_init([], 0)


@pytest.mark.parametrize("I,J,scramble,part", [(100, 150, False, 0), (100, 150, True, 0),
                                               (100, 150, True, 128), (60, 90, False, 1024)])
def test_device_plans_equal_oracle(op2, I, J, scramble, part):
    m = M.naca0012(I, J, scramble=scramble)
    A = apps.Airfoil(m, np.float32)
    R, INC = 0, 3
    specs = {
        "res_calc": O.LoopSpec(m.nedge, [(m.edge, 2, 0, m.nnode, 8, R), (m.edge, 2, 1, m.nnode, 8, R),
                                         (m.ecell, 2, 0, m.ncell, 16, R), (m.ecell, 2, 1, m.ncell, 16, R),
                                         (m.ecell, 2, 0, m.ncell, 4, R), (m.ecell, 2, 1, m.ncell, 4, R),
                                         (m.ecell, 2, 0, m.ncell, 16, INC), (m.ecell, 2, 1, m.ncell, 16, INC)],
                               INDS["res_calc"]),
        "bres_calc": O.LoopSpec(m.nbedge, [(m.bedge, 2, 0, m.nnode, 8, R), (m.bedge, 2, 1, m.nnode, 8, R),
                                           (m.becell.reshape(-1, 1), 1, 0, m.ncell, 16, R),
                                           (m.becell.reshape(-1, 1), 1, 0, m.ncell, 4, R),
                                           (m.becell.reshape(-1, 1), 1, 0, m.ncell, 16, INC),
                                           (None, 0, -1, m.nbedge, 4, R)], INDS["bres_calc"]),
    }
    for loop, spec in specs.items():
        s, args = A.loops[loop]
        p = op2.op_plan_core(loop, s, part, args, INDS[loop])
        assert p, op2.last_error()
        got = op2.plan_arrays(p, args, INDS[loop])
        ref, checks, colours = O.plan_core(spec, part)
        try:
            assert checks == 0 and colours == 0
            for key in [k for k in ref if not k.startswith("_") and isinstance(ref[k], np.ndarray)]:
                assert np.array_equal(got[key], ref[key]), (loop, key)
            for key in ("nblocks", "ncolors", "nshared"):
                assert got[key] == ref[key], (loop, key)
        finally:
            O.plan_free(ref)
        assert op2.op_plan_validate(loop, s, part, args, INDS[loop]) == 0
