"""Renumbering for locality (op2b_set_renumber).

The orders (computed on the GPU) are permutations, and on a scrambled mesh
they bring the two cells of an edge, and an edge and its cells, close
together again.
Recursive coordinate bisection (op2b_set_renumber_coords) is checked
against a restatement here, order for order.
On the device: with renumbering on (either order), the scrambled airfoil's final fields are
still bit-identical to the reference's sequential build (contributions keep
the app's element order) and come back from op_fetch_data in the app's
order; the TREE rms stays within its summation tolerance; jac is unchanged.
"""
import ctypes as C
import hashlib
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from conftest import load_golden
from oplus2_matlab_b200 import _lib, apps
from oplus2_matlab_b200 import mesh as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rcb_order(xyz):
    """Recursive coordinate bisection as op2b_set_renumber_coords defines it
    (the checker for the device order): each segment is halved at
    mid = len // 2 along the axis of its largest extent (last minus first
    coordinate in that axis' order, in float; ties: the lower axis), the
    halves keep every axis' order, down to single elements; coordinates are
    compared rounded to float, -0 before +0, ties by element number."""
    c = np.ascontiguousarray(np.asarray(xyz).astype(np.float32))
    if c.ndim == 1:
        c = c[:, None]
    n, dim = c.shape
    u = c.view(np.uint32)
    key = np.where(u & np.uint32(0x80000000), ~u, u | np.uint32(0x80000000))
    idx = np.arange(n)
    lists = [np.lexsort((idx, key[:, a])) for a in range(dim)]
    upper = np.zeros(n, bool)
    out = []

    def walk(ls):
        k = len(ls[0])
        if k < 2:
            out.extend(ls[0].tolist())
            return
        best, ax = None, 0
        for a in range(dim):
            e = c[ls[a][-1], a] - c[ls[a][0], a]
            if a == 0 or e > best:
                best, ax = e, a
        upper[ls[ax][: k // 2]] = False
        upper[ls[ax][k // 2:]] = True
        lo = [l[~upper[l]] for l in ls]
        hi = [l[upper[l]] for l in ls]
        walk(lo)
        walk(hi)

    if n:
        walk(lists)
    return np.array(out, np.int64)


def test_rcb_checker_known_answer():
    # 4 x 2 points numbered row by row: x is the longer extent, then each
    # half is 2 x 2 (tie: x first), then each column is split in y
    xy = np.array([(x, y) for y in range(2) for x in range(4)], np.float64)
    assert rcb_order(xy).tolist() == [0, 4, 1, 5, 2, 6, 3, 7]
    # three collinear points and a duplicate: ties by element number
    assert rcb_order(np.array([[2.0], [0.0], [2.0], [-0.0]])).tolist() == [3, 1, 0, 2]
    p = rcb_order(np.random.default_rng(5).normal(size=(1000, 3)))
    assert np.array_equal(np.sort(p), np.arange(1000))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.gpu
def test_orders_are_permutations_that_restore_locality():
    code = textwrap.dedent("""
        import sys, ctypes as C, numpy as np
        sys.path.insert(0, %r)
        from oplus2_matlab_b200 import api, _lib, mesh as M
        L = _lib.load()
        m = M.naca0012(40, 60, scramble=True)
        nodes = api.op_decl_set(m.nnode, "nodes"); edges = api.op_decl_set(m.nedge, "edges")
        bedges = api.op_decl_set(m.nbedge, "bedges"); cells = api.op_decl_set(m.ncell, "cells")
        api.op_decl_map(edges, nodes, 2, m.edge, "pedge")
        api.op_decl_map(edges, cells, 2, m.ecell, "pecell")
        api.op_decl_map(bedges, nodes, 2, m.bedge, "pbedge")
        api.op_decl_map(bedges, cells, 1, m.becell, "pbecell")
        api.op_decl_map(cells, nodes, 4, m.cell, "pcell")
        P = {}
        for name, s, n in (("nodes", nodes, m.nnode), ("edges", edges, m.nedge),
                           ("bedges", bedges, m.nbedge), ("cells", cells, m.ncell)):
            p = np.zeros(n, np.int32)
            assert L.op2b_renumber_order(s, p.ctypes.data_as(C.POINTER(C.c_int))) == 1
            assert np.array_equal(np.sort(p), np.arange(n)), name
            P[name] = p
        Qc = np.argsort(P["cells"]); Qn = np.argsort(P["nodes"])
        # spread of an edge's two cells, and of consecutive edges' cells
        before = np.abs(m.ecell[:, 0] - m.ecell[:, 1]).mean()
        after = np.abs(Qc[m.ecell[:, 0]] - Qc[m.ecell[:, 1]]).mean()
        e_new = m.ecell[P["edges"]]
        jump_before = np.abs(np.diff(m.ecell[:, 0])).mean()
        jump_after = np.abs(np.diff(Qc[e_new[:, 0]])).mean()
        print(before, after, jump_before, jump_after)
        assert after < before / 20 and jump_after < jump_before / 20
        nodes_after = np.abs(Qn[m.cell[P["cells"]][:, 0]] - np.arange(m.ncell)).mean()
        assert nodes_after < m.nnode / 20
    """ % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_rcb_order_matches_checker_and_restores_locality(op2, dtype):
    L = _lib.load()
    m = M.naca0012(40, 60, scramble=True)
    A = apps.Airfoil(m, dtype)
    assert L.op2b_set_renumber_coords(A.p_x) == 0
    P = {}
    for name, s, n in (("nodes", A.nodes, m.nnode), ("edges", A.edges, m.nedge),
                       ("bedges", A.bedges, m.nbedge), ("cells", A.cells, m.ncell)):
        p = np.zeros(n, np.int32)
        assert L.op2b_renumber_order(s, p.ctypes.data_as(C.POINTER(C.c_int))) == 1
        assert np.array_equal(np.sort(p), np.arange(n)), name
        P[name] = p
    assert op2.last_error() == ""
    assert np.array_equal(P["nodes"], rcb_order(A.x))
    Qc = np.argsort(P["cells"])
    before = np.abs(m.ecell[:, 0] - m.ecell[:, 1]).mean()
    after = np.abs(Qc[m.ecell[:, 0]] - Qc[m.ecell[:, 1]]).mean()
    assert after < before / 20


@pytest.mark.gpu
def test_rcb_rejects_bad_coordinates(op2):
    L = _lib.load()
    op2.set_error_mode(op2.ERRORS_RETURN)
    m = M.naca0012(40, 60)
    A = apps.Airfoil(m, np.float32)
    assert L.op2b_set_renumber_coords(A.p_bound) == -1  # int components
    assert L.op2b_set_renumber_coords(A.p_q) == -1      # four components
    assert "coordinates for bisection" in op2.last_error()
    op2.clear_error()


@pytest.mark.gpu
@pytest.mark.parametrize("case,order", [("airfoil_40x60s_f32", "cm"), ("airfoil_40x60_f32", "cm"),
                                        ("airfoil_40x60s_f32", "rcb")])
def test_renumbered_airfoil_fields_bit_identical(op2, case, order):
    g = load_golden(case)
    m = M.naca0012(g["I"], g["J"], scramble=g["scramble"])
    op2.set_strategy(op2.STRATEGY_GATHER)
    op2.set_reduction(op2.REDUCE_TREE)
    assert _lib.load().op2b_set_renumber(1) == 0
    A = apps.Airfoil(m, np.float32)
    if order == "rcb":
        assert _lib.load().op2b_set_renumber_coords(A.p_x) == 0
    rms = A.iterate(g["niter"])
    st = A.fetch()
    assert op2.last_error() == ""
    for f, key in (("p_q", "q"), ("p_qold", "qold"), ("p_res", "res"), ("p_adt", "adt")):
        assert sha(st[key]) == g["final"][f]["sha256"], f
    ref = np.array([v for _, v in g["rms"]])
    assert np.max(np.abs(rms - ref) / ref) < 5e-5


@pytest.mark.gpu
def test_renumbered_jac1_matches_reference(op2):
    g = load_golden("jac1_nn64")
    op2.set_strategy(op2.STRATEGY_GATHER)
    op2.set_reduction(op2.REDUCE_TREE)
    assert _lib.load().op2b_set_renumber(1) == 0
    jm = M.jac(g["NN"], g["variant"])
    J = apps.Jac(jm, g["variant"])
    J.iterate(g["niter"])
    u = J.fetch()
    assert op2.last_error() == ""
    assert sha(u) == g["u_sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("order", ["cm", "rcb"])
def test_renumbered_seq_rms_bit_identical_to_reference(op2, order):
    """With the sets renumbered, REDUCE_SEQ still adds update's del^2 in the
    app's cell order (the device buffer is read through the renumbering), so
    every printed rms of the scrambled mesh equals the reference's bit for
    bit, as the fields do."""
    g = load_golden("airfoil_40x60s_f32")
    m = M.naca0012(g["I"], g["J"], scramble=g["scramble"])
    op2.set_strategy(op2.STRATEGY_GATHER)
    op2.set_reduction(op2.REDUCE_SEQ)
    assert _lib.load().op2b_set_renumber(1) == 0
    A = apps.Airfoil(m, np.float32)
    if order == "rcb":
        assert _lib.load().op2b_set_renumber_coords(A.p_x) == 0
    rms = A.iterate(g["niter"])
    st = A.fetch()
    assert op2.last_error() == ""
    for it, val in g["rms"]:
        assert rms[it - 1] == np.float32(val), (it, rms[it - 1], val)
    for f, key in (("p_q", "q"), ("p_qold", "qold"), ("p_res", "res"), ("p_adt", "adt")):
        assert sha(st[key]) == g["final"][f]["sha256"], f
