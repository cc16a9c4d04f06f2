"""Mesh inputs of the airfoil and jac apps, as numpy arrays.

The generators are C++ in libop2b200.so (csrc/meshgen.cpp): the NACA0012
C-mesh of airfoil/naca0012.m with an optional seeded renumbering, and the jac
Jacobi grid of jac1/jac.cpp.  This module only wraps them.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib

SEED = 20261203  # the fixed 64-bit seed of the randomised configurations


@dataclass
class AirfoilMesh:
    I: int
    J: int
    nnode: int
    ncell: int
    nedge: int
    nbedge: int
    cell: np.ndarray    # [ncell, 4]  pcell
    edge: np.ndarray    # [nedge, 2]  pedge
    ecell: np.ndarray   # [nedge, 2]  pecell
    bedge: np.ndarray   # [nbedge, 2] pbedge
    becell: np.ndarray  # [nbedge]    pbecell
    bound: np.ndarray   # [nbedge]    1 wall, 2 far field
    x64: np.ndarray     # [nnode, 2]  coordinates as read with %lf
    x32: np.ndarray     # [nnode, 2]  coordinates as read with %f

    def x(self, dtype):
        return self.x64 if np.dtype(dtype) == np.float64 else self.x32


def _take(m):
    def arr(ptr, shape, dt):
        n = int(np.prod(shape))
        return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt).reshape(shape).copy()
    return dict(
        nnode=m.nnode, ncell=m.ncell, nedge=m.nedge, nbedge=m.nbedge,
        cell=arr(m.cell, (m.ncell, 4), np.int32), edge=arr(m.edge, (m.nedge, 2), np.int32),
        ecell=arr(m.ecell, (m.nedge, 2), np.int32), bedge=arr(m.bedge, (m.nbedge, 2), np.int32),
        becell=arr(m.becell, (m.nbedge,), np.int32), bound=arr(m.bound, (m.nbedge,), np.int32),
        x64=arr(m.x64, (m.nnode, 2), np.float64), x32=arr(m.x32, (m.nnode, 2), np.float32))


def naca0012(I, J, scramble=False, seed=SEED):
    """The (3I x J)-cell mesh of airfoil/naca0012.m; I=400, J=600 gives the
    720k-cell mesh, I=40, J=60 the 7.2k one."""
    lib = _lib.load()
    m = _lib.op2b_mesh()
    rc = lib.op2b_mesh_naca0012(int(I), int(J), 1 if scramble else 0, C.c_uint64(seed), C.byref(m))
    if rc != 0:
        raise ValueError("mesh generation failed (I=%d, J=%d): rc %d" % (I, J, rc))
    try:
        return AirfoilMesh(I=I, J=J, **_take(m))
    finally:
        lib.op2b_mesh_free(C.byref(m))


def as_struct(mesh):
    """An op2b_mesh view of an AirfoilMesh's arrays; returns (struct, keep),
    where `keep` must outlive every use of the struct."""
    m = _lib.op2b_mesh()
    keep = []

    def ptr(a, ct, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(ct))
    m.nnode, m.ncell, m.nedge, m.nbedge = mesh.nnode, mesh.ncell, mesh.nedge, mesh.nbedge
    m.cell = ptr(mesh.cell, C.c_int, np.int32)
    m.edge = ptr(mesh.edge, C.c_int, np.int32)
    m.ecell = ptr(mesh.ecell, C.c_int, np.int32)
    m.bedge = ptr(mesh.bedge, C.c_int, np.int32)
    m.becell = ptr(mesh.becell, C.c_int, np.int32)
    m.bound = ptr(mesh.bound, C.c_int, np.int32)
    m.x64 = ptr(mesh.x64, C.c_double, np.float64)
    m.x32 = ptr(mesh.x32, C.c_float, np.float32)
    return m, keep


def write_grid(mesh, path):
    """Write new_grid.dat (naca0012.m:328-351) for the reference apps."""
    lib = _lib.load()
    m, keep = as_struct(mesh)
    if lib.op2b_mesh_write(C.byref(m), str(path).encode()) != 0:
        raise IOError("cannot write %s" % path)


def cells_to_IJ(cells):
    """I, J of a 2:1 (3I : J = 2 : 1) C-mesh with about `cells` cells."""
    J = max(4, int(round((cells / 2.0) ** 0.5)))
    I = max(2, int(round(2.0 * J / 3.0)))
    return I, J


@dataclass
class JacMesh:
    NN: int
    nnode: int
    nedge: int
    pp: np.ndarray   # [nedge, 2] edge -> node
    A: np.ndarray    # jac1: [nedge] float32; jac2: [nedge, 3] float64
    r: np.ndarray    # jac1: [nnode] float32; jac2: [nnode, 2] float32


def jac(NN, variant=1):
    lib = _lib.load()
    nn, ne = C.c_int(), C.c_int()
    if lib.op2b_jac_sizes(int(NN), C.byref(nn), C.byref(ne)) != 0:
        raise ValueError("NN must be >= 3")
    nnode, nedge = nn.value, ne.value
    pp = np.zeros((nedge, 2), np.int32)
    if variant == 1:
        A = np.zeros(nedge, np.float32)
        r = np.zeros(nnode, np.float32)
        rc = lib.op2b_mesh_jac1(int(NN), pp.ctypes.data, A.ctypes.data, r.ctypes.data)
    else:
        A = np.zeros((nedge, 3), np.float64)
        r = np.zeros((nnode, 2), np.float32)
        rc = lib.op2b_mesh_jac2(int(NN), pp.ctypes.data, A.ctypes.data, r.ctypes.data)
    if rc != nedge:
        raise RuntimeError("jac mesh generation failed")
    return JacMesh(NN=NN, nnode=nnode, nedge=nedge, pp=pp, A=A, r=r)


def read_grid(path, cache=None):
    """Read new_grid.dat (airfoil/airfoil.cpp:80-129); with `cache`, through a
    binary cache of the same file (op2b_mesh_read_cached)."""
    lib = _lib.load()
    m = _lib.op2b_mesh()
    if cache:
        rc = lib.op2b_mesh_read_cached(str(path).encode(), str(cache).encode(), C.byref(m))
    else:
        rc = lib.op2b_mesh_read(str(path).encode(), C.byref(m))
    if rc != 0:
        raise IOError("cannot read %s (rc %d)" % (path, rc))
    try:
        return AirfoilMesh(I=0, J=0, **_take(m))
    finally:
        lib.op2b_mesh_free(C.byref(m))
