"""Mesh inputs: the NACA0012 generator (restating airfoil/naca0012.m), its
text format, the seeded renumbering, and the jac grid.  CPU only."""
import os

import numpy as np
import pytest

from conftest import scratch_dir

from oplus2_matlab_b200 import mesh as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("I,J", [(40, 60), (400, 600), (7, 5)])
def test_counts_follow_naca0012_formulae(I, J):
    m = M.naca0012(I, J)
    assert m.nnode == (3 * I + 1) * (J + 1)
    assert m.ncell == 3 * I * J
    assert m.nedge == (3 * I - 1) * J + 3 * I * (J - 1) + I
    assert m.nbedge == I + 3 * I + 2 * J
    assert (m.bound == 1).sum() == I and (m.bound == 2).sum() == 3 * I + 2 * J


def test_maps_in_range_and_each_interior_edge_joins_two_cells():
    m = M.naca0012(40, 60)
    for a, n in ((m.cell, m.nnode), (m.edge, m.nnode), (m.ecell, m.ncell), (m.bedge, m.nnode),
                 (m.becell, m.ncell)):
        assert a.min() >= 0 and a.max() < n
    assert np.all(m.ecell[:, 0] != m.ecell[:, 1])
    # every cell has 4 faces: interior edges count twice, boundary edges once
    deg = np.bincount(m.ecell.ravel(), minlength=m.ncell) + np.bincount(m.becell, minlength=m.ncell)
    assert np.all(deg == 4)


def test_grid_file_round_trip():
    m = M.naca0012(12, 9)
    d = scratch_dir()
    p = os.path.join(d, "new_grid.dat")
    M.write_grid(m, p)
    r = M.read_grid(p)
    os.remove(p)
    for k in ("cell", "edge", "ecell", "bedge", "becell", "bound", "x64", "x32"):
        assert np.array_equal(getattr(m, k), getattr(r, k)), k


def test_scramble_is_a_consistent_renumbering():
    a, b = M.naca0012(20, 30), M.naca0012(20, 30, scramble=True)
    assert not np.array_equal(a.edge, b.edge)
    # same multiset of coordinates, edge geometry and boundary flags
    assert np.array_equal(np.sort(a.x64.view(np.complex128).ravel()), np.sort(b.x64.view(np.complex128).ravel()))
    ga = np.sort(np.sort(a.x64[a.edge].reshape(-1, 4), axis=0), axis=0)
    gb = np.sort(np.sort(b.x64[b.edge].reshape(-1, 4), axis=0), axis=0)
    assert np.array_equal(ga, gb)
    assert np.array_equal(np.sort(a.bound), np.sort(b.bound))
    # deterministic in the seed
    c = M.naca0012(20, 30, scramble=True)
    assert np.array_equal(b.edge, c.edge) and np.array_equal(b.x32, c.x32)


def test_jac_grid():
    j = M.jac(6, 1)
    assert (j.nnode, j.nedge) == (25, 105)
    assert j.pp[0].tolist() == [0, 0] and j.A[0] == -1.0
    # 4*(NN-1) boundary contacts of 0.25 each
    assert abs(float(j.r.sum()) - 0.25 * 4 * 5) < 1e-6
    j2 = M.jac(6, 2)
    assert j2.A.shape == (105, 3) and np.array_equal(j2.A[:, 0].astype(np.float32), j.A)


# ---------------------------------------------------------- mesh files ----

def _read(fn, *paths):
    import ctypes as C
    from oplus2_matlab_b200 import _lib
    L = _lib.load()
    s = _lib.op2b_mesh()
    rc = getattr(L, fn)(*[p.encode() for p in paths], C.byref(s))
    if rc != 0:
        return rc, None
    try:
        return 0, M._take(s)
    finally:
        L.op2b_mesh_free(C.byref(s))


def _same(a, b):
    for k in ("cell", "edge", "ecell", "bedge", "becell", "bound", "x64", "x32"):
        assert np.array_equal(a[k], getattr(b, k) if not isinstance(b, dict) else b[k]), k


def test_text_binary_and_cached_reads_agree(tmp_path):
    import ctypes as C
    import os
    from oplus2_matlab_b200 import _lib
    m = M.naca0012(40, 60)
    txt, binp, cache = str(tmp_path / "g.dat"), str(tmp_path / "g.bin"), str(tmp_path / "g.cache")
    M.write_grid(m, txt)
    rc, t = _read("op2b_mesh_read", txt)
    assert rc == 0
    _same(t, m)  # the fast text reader gives the generator's values bit for bit
    s, keep = M.as_struct(m)
    assert _lib.load().op2b_mesh_write_bin(C.byref(s), binp.encode()) == 0
    rc, b = _read("op2b_mesh_read_bin", binp)
    assert rc == 0
    _same(b, m)
    rc, c1 = _read("op2b_mesh_read_cached", txt, cache)  # parses, writes the cache
    assert rc == 0 and os.path.exists(cache)
    _same(c1, m)
    stamp = os.stat(cache).st_mtime_ns
    rc, c2 = _read("op2b_mesh_read_cached", txt, cache)  # reads the cache
    assert rc == 0 and os.stat(cache).st_mtime_ns == stamp
    _same(c2, m)


def test_damaged_or_stale_cache_is_not_used(tmp_path):
    import os
    m = M.naca0012(20, 30)
    txt, cache = str(tmp_path / "g.dat"), str(tmp_path / "g.cache")
    M.write_grid(m, txt)
    assert _read("op2b_mesh_read_cached", txt, cache)[0] == 0
    with open(cache, "r+b") as f:  # flip one payload byte
        f.seek(os.path.getsize(cache) - 5)
        b = f.read(1)
        f.seek(-1, 1)
        f.write(bytes([b[0] ^ 0xFF]))
    assert _read("op2b_mesh_read_bin", cache)[0] == 2
    rc, c = _read("op2b_mesh_read_cached", txt, cache)  # falls back to the text, rewrites
    assert rc == 0
    _same(c, m)
    assert _read("op2b_mesh_read_bin", cache)[0] == 0
    m2 = M.naca0012(21, 30)  # a new text file: the old cache is stale
    M.write_grid(m2, txt)
    rc, c = _read("op2b_mesh_read_cached", txt, cache)
    assert rc == 0 and c["ncell"] == m2.ncell
