"""Many airfoil solves on one GPU (include/op2b_group.h), and the plain
single-solve path they are compared with.

Group wraps the C-ABI engine: every loop of the outer iteration runs as one
launch over all active solves, each solve's rms history and stopping test
stay on the device.  plain_solve runs one solve through the OP2 C API
(libop2b200_apps.so: op_decl_* from host arrays, op_par_loop_* with the rms
returned to the host after every update, op_fetch_data), as a generated app
main does.

draw_instances() is the seeded instance stream of the batched and served
workloads: cell counts log-uniform in [cmin, cmax] with the mesh aspect
3I:J = 2:1 (J = round(sqrt(C/2)), I = round(2J/3)), Mach uniform in
[0.3, 0.7], alpha uniform in [-2, 6] degrees, all from one splitmix64 stream.
"""
import ctypes as C
import math
import os

import numpy as np

from . import _lib
from . import mesh as M

APPS_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libop2b200_apps.so")


class AppTiming(C.Structure):
    _fields_ = [("t_declare", C.c_double), ("t_iterate", C.c_double), ("t_fetch", C.c_double),
                ("t_total", C.c_double), ("h2d_bytes", C.c_longlong), ("d2h_bytes", C.c_longlong)]


_apps = None


def apps_lib():
    global _apps
    if _apps is None:
        _lib.load()
        a = C.CDLL(APPS_LIB)
        a.op2b_airfoil_app_flow.argtypes = [C.POINTER(_lib.op2b_mesh), C.c_int, C.c_int,
                                            C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                            C.c_int, C.POINTER(AppTiming)]
        a.op2b_airfoil_app_flow.restype = C.c_int
        _apps = a
    return _apps


def flow_qinf(mach, alpha_deg, dtype=np.float32):
    """(qinf[4], (gam, gm1, cfl, eps)) of a flow condition, in dtype."""
    dt = np.dtype(dtype)
    q = np.zeros(4, dt)
    c = np.zeros(4, dt)
    _lib.load().op2b_flow_qinf(float(mach), float(alpha_deg), 1 if dt == np.float64 else 0,
                               q.ctypes.data, c.ctypes.data)
    return q, c


def plain_solve(mesh, mach, alpha_deg, niter, dtype=np.float32, strategy=1, q_out=None):
    """One solve through the OP2 C API; returns (q, rms history, AppTiming).
    q_out: an (ncell, 4) array of dtype to hold q (e.g. in pinned memory);
    default a new one."""
    dt = np.dtype(dtype)
    qinf, _ = flow_qinf(mach, alpha_deg, dt)
    if q_out is None:
        q = np.ascontiguousarray(np.tile(qinf, (mesh.ncell, 1)))
    else:
        q = q_out
        q[...] = qinf
    rms = np.zeros(niter, np.float64)
    m, keep = M.as_struct(mesh)
    t = AppTiming()
    rc = apps_lib().op2b_airfoil_app_flow(C.byref(m), 1 if dt == np.float64 else 0, int(niter),
                                          float(mach), float(alpha_deg), q.ctypes.data,
                                          rms.ctypes.data, int(strategy), C.byref(t))
    del keep
    if rc != 0:
        raise RuntimeError("plain solve failed: %s" % _lib.load().op2b_last_error().decode())
    return q, rms, t


def mesh_dims(cells):
    """(I, J) of the 3I x J C-mesh closest to `cells` cells at aspect 2:1."""
    J = max(4, int(round(math.sqrt(cells / 2.0))))
    I = max(2, int(round(2.0 * J / 3.0)))
    return I, J


def draw_instances(n, seed=M.SEED, cmin=20000, cmax=720000):
    """n seeded (I, J, mach, alpha_deg) draws of the batched/served workloads."""
    lib = _lib.load()
    state = C.c_uint64(seed)

    def uniform():
        return (lib.op2b_splitmix64(C.byref(state)) >> 11) * (1.0 / 9007199254740992.0)
    out = []
    for _ in range(n):
        cells = math.exp(math.log(cmin) + uniform() * (math.log(cmax) - math.log(cmin)))
        I, J = mesh_dims(cells)
        mach = 0.3 + 0.4 * uniform()
        alpha = -2.0 + 8.0 * uniform()
        out.append((I, J, mach, alpha))
    return out


class Group:
    """A set of airfoil solves iterated together (op2b_group_*)."""

    def __init__(self, dtype=np.float32):
        self.lib = _lib.load()
        self.dtype = np.dtype(dtype)
        self.h = self.lib.op2b_group_create(1 if self.dtype == np.float64 else 0)
        if not self.h:
            raise RuntimeError(self._err("op2b_group_create"))
        self.ncell = {}

    def _err(self, what):
        return "%s failed: %s" % (what, self.lib.op2b_last_error().decode())

    def _check(self, rc, what):
        if rc is None or rc < 0:
            raise RuntimeError(self._err(what))
        return rc

    def close(self):
        if self.h:
            self.lib.op2b_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, mesh, mach, alpha_deg, max_iter, rel_tol=0.0):
        m, keep = M.as_struct(mesh)
        sid = self.lib.op2b_group_add(self.h, C.byref(m), float(mach), float(alpha_deg),
                                      int(max_iter), float(rel_tol))
        del keep
        self._check(sid, "op2b_group_add")
        self.ncell[sid] = mesh.ncell
        return sid

    def run(self, niter):
        return self._check(self.lib.op2b_group_run(self.h, int(niter)), "op2b_group_run")

    def poll(self, max_ids=4096):
        ids = (C.c_int * max_ids)()
        n = self._check(self.lib.op2b_group_poll(self.h, ids, max_ids), "op2b_group_poll")
        return [ids[i] for i in range(n)]

    def sync(self):
        self._check(self.lib.op2b_group_sync(self.h), "op2b_group_sync")

    def iterations(self, sid):
        return self._check(self.lib.op2b_group_iterations(self.h, sid), "op2b_group_iterations")

    def history(self, sid, max_n=1 << 20):
        n = self.iterations(sid)
        out = np.zeros(max(n, 1), np.float64)
        got = self._check(self.lib.op2b_group_history(self.h, sid,
                                                      out.ctypes.data_as(C.POINTER(C.c_double)),
                                                      min(n, max_n)), "op2b_group_history")
        return out[:got]

    def fetch_q(self, sid, out=None):
        q = np.zeros((self.ncell[sid], 4), self.dtype) if out is None else out
        self._check(self.lib.op2b_group_fetch_q(self.h, sid, q.ctypes.data), "op2b_group_fetch_q")
        return q

    def fetch_q_async(self, sid, out):
        """q of a solve poll() has reported stopped, copied while the others
        iterate; `out` (pinned for an overlapped copy) is valid after sync()."""
        self._check(self.lib.op2b_group_fetch_q_async(self.h, sid, out.ctypes.data),
                    "op2b_group_fetch_q_async")
        return out

    def remove(self, sid):
        self._check(self.lib.op2b_group_remove(self.h, sid), "op2b_group_remove")

    def solve_bytes(self, mesh, max_iter):
        return self.lib.op2b_group_solve_bytes(self.h, mesh.nnode, mesh.ncell, mesh.nedge,
                                               mesh.nbedge, int(max_iter))

    def device_bytes(self):
        return self.lib.op2b_group_device_bytes(self.h)

    def active(self):
        return self.lib.op2b_group_active(self.h)

    @property
    def edge_tile(self):
        return self.lib.op2b_group_edge_tile(self.h)

    @edge_tile.setter
    def edge_tile(self, e):
        self._check(self.lib.op2b_group_set_edge_tile(self.h, int(e)), "op2b_group_set_edge_tile")

    def set_streams(self, n):
        self._check(self.lib.op2b_group_set_streams(self.h, int(n)), "op2b_group_set_streams")

    def set_tiled(self, on=True):
        """One launch per update over all solves, flux values in shared
        memory (op2b_group_set_tiled); fields unchanged."""
        self._check(self.lib.op2b_group_set_tiled(self.h, 1 if on else 0), "op2b_group_set_tiled")

    def set_block_bytes(self, nbytes):
        self._check(self.lib.op2b_group_set_block_bytes(self.h, int(nbytes)),
                    "op2b_group_set_block_bytes")

    def autotune(self, iters=5):
        return self._check(self.lib.op2b_group_autotune(self.h, int(iters)), "op2b_group_autotune")

    def autotune_run(self, iters=1):
        """Tune on real iterations (they count); returns the iterations run."""
        return self._check(self.lib.op2b_group_autotune_run(self.h, int(iters)),
                           "op2b_group_autotune_run")
