"""ctypes bindings of the CPU oracle (oracle/op2_oracle.c) for the tests.

Test infrastructure only: the checker the device results are compared with.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_build", "liboracle.so")

_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile"), "port"],
                           check=True)
        _lib = C.CDLL(LIB)
        _lib.op2o_plan_check_colours.restype = C.c_long
    return _lib


def P(a):
    return a.ctypes.data_as(C.c_void_p)


class OPlan(C.Structure):
    _fields_ = [(n, C.c_int) for n in "set_size nargs ninds bsize nblocks ncolors nshared".split()] + \
               [(n, C.c_void_p) for n in
                "nthrcol thrcol offset nelems ind_offs ind_sizes nindirect ind_maps loc_maps ncolblk blkmap".split()] + \
               [("transfer", C.c_double), ("transfer2", C.c_double)]


class LoopSpec:
    """A loop signature for the plan oracle: per arg (map array or None, map
    dim, idx, target-set size, dat bytes per element, access, ind)."""

    def __init__(self, set_size, args, inds):
        self.set_size = set_size
        self.args = args
        self.inds = list(inds)

    def c_arrays(self):
        n = len(self.args)
        self._maps = [None if a[0] is None else np.ascontiguousarray(a[0], np.int32) for a in self.args]
        mp = (C.c_void_p * n)(*[None if m is None else m.ctypes.data for m in self._maps])
        dims = (C.c_int * n)(*[a[1] for a in self.args])
        idxs = (C.c_int * n)(*[a[2] for a in self.args])
        tos = (C.c_int * n)(*[a[3] for a in self.args])
        ds = (C.c_int * n)(*[a[4] for a in self.args])
        acc = (C.c_int * n)(*[a[5] for a in self.args])
        ii = (C.c_int * n)(*self.inds)
        return mp, dims, idxs, tos, ds, acc, ii


def plan_core(spec, part_size, cache_line=128):
    """Run the restated op_plan_core; returns (dict of numpy arrays, checks)."""
    L = load()
    mp, dims, idxs, tos, ds, acc, ii = spec.c_arrays()
    ninds = max(spec.inds) + 1 if max(spec.inds) >= 0 else 0
    p = OPlan()
    rc = L.op2o_plan_core(spec.set_size, part_size, len(spec.args), mp, dims, idxs, tos, ds, acc,
                          ninds, ii, cache_line, C.byref(p))
    assert rc == 0

    def arr(ptr, n, ct=C.c_int, dt=np.int32):
        if n == 0:
            return np.zeros(0, dt)
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(n,)).astype(dt).copy()

    out = dict(nblocks=p.nblocks, ncolors=p.ncolors, nshared=p.nshared, bsize=p.bsize,
               transfer=p.transfer, transfer2=p.transfer2,
               nthrcol=arr(p.nthrcol, p.nblocks), thrcol=arr(p.thrcol, p.set_size),
               offset=arr(p.offset, p.nblocks), nelems=arr(p.nelems, p.nblocks),
               blkmap=arr(p.blkmap, p.nblocks), ncolblk=arr(p.ncolblk, p.ncolors),
               ind_offs=arr(p.ind_offs, p.nblocks * ninds), ind_sizes=arr(p.ind_sizes, p.nblocks * ninds),
               nindirect=arr(p.nindirect, ninds))
    im = C.cast(p.ind_maps, C.POINTER(C.c_void_p))
    lm = C.cast(p.loc_maps, C.POINTER(C.c_void_p))
    for m in range(ninds):
        out["ind_maps%d" % m] = arr(im[m], int(out["nindirect"][m]))
    for a in range(len(spec.args)):
        if spec.inds[a] >= 0:
            out["loc_maps%d" % a] = arr(lm[a], p.set_size, C.c_short, np.int16)
    checks = L.op2o_plan_check(C.byref(p), mp, dims, idxs, tos, ii)
    colours = L.op2o_plan_check_colours(C.byref(p), mp, dims, idxs, tos, acc, ii)
    out["_plan"] = p  # caller frees with plan_free
    return out, checks, colours


def plan_free(out):
    load().op2o_plan_free(C.byref(out["_plan"]))


def airfoil_consts(dtype):
    t = np.float32 if np.dtype(dtype) == np.float32 else np.float64
    K = np.zeros(10, t)
    getattr(load(), "op2o_airfoil_consts_" + ("f32" if t == np.float32 else "f64"))(P(K))
    return K


def airfoil(mesh, dtype, niter, state=None):
    """niter outer iterations of the app on `mesh`; returns (rms history,
    dict of final q, qold, adt, res)."""
    L = load()
    t = np.dtype(dtype).type
    suf = "f32" if t == np.float32 else "f64"
    K = airfoil_consts(t)
    x = np.ascontiguousarray(mesh.x(t))
    nc = mesh.ncell
    if state is None:
        q = np.tile(K[6:10], nc).astype(t)
        qold, adt, res = np.zeros(4 * nc, t), np.zeros(nc, t), np.zeros(4 * nc, t)
    else:
        q, qold, adt, res = (np.ascontiguousarray(state[k], t).ravel().copy() for k in ("q", "qold", "adt", "res"))
    rms = np.zeros(max(niter, 1), t)
    getattr(L, "op2o_airfoil_" + suf)(nc, mesh.nedge, mesh.nbedge, P(mesh.cell), P(mesh.edge),
                                     P(mesh.ecell), P(mesh.bedge), P(mesh.becell), P(mesh.bound),
                                     P(x), P(q), P(qold), P(adt), P(res), P(K), niter, P(rms))
    return rms[:niter], dict(q=q.reshape(nc, 4), qold=qold.reshape(nc, 4), adt=adt.reshape(nc, 1),
                             res=res.reshape(nc, 4))


def airfoil_loop(name, mesh, dtype, state):
    """One call of one airfoil loop on copies of `state`; returns the new state."""
    L = load()
    t = np.dtype(dtype).type
    suf = "f32" if t == np.float32 else "f64"
    K = airfoil_consts(t)
    x = np.ascontiguousarray(mesh.x(t))
    s = {k: np.ascontiguousarray(v, t).copy() for k, v in state.items()}
    if name == "save_soln":
        getattr(L, "op2o_save_soln_" + suf)(mesh.ncell, P(s["q"]), P(s["qold"]))
    elif name == "adt_calc":
        getattr(L, "op2o_adt_calc_" + suf)(mesh.ncell, P(mesh.cell), P(x), P(s["q"]), P(s["adt"]), P(K))
    elif name == "res_calc":
        getattr(L, "op2o_res_calc_" + suf)(mesh.nedge, P(mesh.edge), P(mesh.ecell), P(x), P(s["q"]),
                                           P(s["adt"]), P(s["res"]), P(K))
    elif name == "bres_calc":
        getattr(L, "op2o_bres_calc_" + suf)(mesh.nbedge, P(mesh.bedge), P(mesh.becell), P(x), P(s["q"]),
                                            P(s["adt"]), P(s["res"]), P(mesh.bound), P(K))
    elif name == "update":
        rms = np.zeros(1, t)
        getattr(L, "op2o_update_" + suf)(mesh.ncell, P(s["qold"]), P(s["q"]), P(s["res"]), P(s["adt"]), P(rms))
        s["rms"] = rms
    return s


def jac(jm, variant, niter):
    """jac1/jac.cpp's loop on the oracle: returns ([(u_max, u_sum)], u)."""
    L = load()
    nn = jm.nnode
    if variant == 1:
        u, du = np.zeros(nn, np.float32), np.zeros(nn, np.float32)
    else:
        u, du = np.zeros(2 * nn, np.float32), np.zeros(3 * nn, np.float32)
    A = np.ascontiguousarray(jm.A).ravel()
    r = np.ascontiguousarray(jm.r).ravel()
    hist = []
    us, um = C.c_float(0), C.c_float(0)
    for _ in range(niter):
        if variant == 1:
            L.op2o_jac1_res(jm.nedge, P(jm.pp), P(A), P(u), P(du), C.c_float(1.0))
        else:
            L.op2o_jac2_res(jm.nedge, P(jm.pp), P(A), P(u), P(du), C.c_float(1.0))
        us.value, um.value = 0.0, 0.0
        f = L.op2o_jac1_update if variant == 1 else L.op2o_jac2_update
        f(nn, P(r), P(du), P(u), C.byref(us), C.byref(um), C.c_float(1.0))
        hist.append((um.value, us.value))
    return hist, u
