"""Continuous-batching solve server over one GPU's group engine: a thin
driver of the C++ server (include/op2b_serve.h, csrc/serve.cpp).

Requests (mesh + flow condition + stopping rule) arrive at any time.  The
server keeps every admitted solve's state resident in HBM (op2b_group),
admits queued requests (first-come first-served, or least work first) while
the group's device bytes plus the request's stay under the memory budget
(and, optionally, while fewer than max_active solves run), and advances all
admitted solves together: each `step` enqueues a few outer iterations of
every active solve as one launch per loop, admits newly arrived requests
while those run on the GPU (their uploads and list builds go on the group's
admission stream), then waits, retires the solves that stopped (rms
tolerance or iteration cap) and frees their memory, making room for the
queue.  A solve's results do not depend on what it was batched with
(include/op2b_group.h), so a request's answer is the same alone or in the mix.

The admission, retirement and latency bookkeeping run in C++; this module
keeps the Python objects (Request) and, for a stand-in group written in
Python (the host tests), hands the C++ server a table of callbacks.

shard_by_cells splits a list of instances over ranks (GPUs) by greedy
balance of cell counts: instances are independent, so N GPUs need no
collective, only the gather of results.
"""
import ctypes as C

import numpy as np

from . import _lib
from . import group as G
from . import mesh as M


def shard_by_cells(cells, world):
    """Indices of `cells` per rank: largest first, each to the rank with the
    fewest cells so far (ties to the lower rank); deterministic."""
    order = sorted(range(len(cells)), key=lambda i: (-cells[i], i))
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += cells[i]
    return [sorted(o) for o in out]


class Request:
    __slots__ = ("rid", "mesh", "mach", "alpha", "max_iter", "rel_tol", "arrival", "admitted",
                 "finished", "sid", "iterations", "rms", "q")

    def __init__(self, rid, mesh, mach, alpha, max_iter, rel_tol, arrival):
        self.rid, self.mesh, self.mach, self.alpha = rid, mesh, mach, alpha
        self.max_iter, self.rel_tol, self.arrival = max_iter, rel_tol, arrival
        self.admitted = self.finished = None
        self.sid = None
        self.iterations = 0
        self.rms = None
        self.q = None


class Server:
    """Admit, iterate and retire solves on one GPU (op2b_server_*)."""

    def __init__(self, dtype=np.float32, budget_bytes=150 * 10**9, iters_per_step=10,
                 keep_q=False, clock=None, max_active=0, policy="fifo", group=None):
        """max_active > 0 caps the solves iterated together (0: memory budget
        only); policy "fifo" admits in arrival order, "shortest" admits the
        queued request with the least work (cells x iteration cap) first.
        group: the solve group to drive (default: a new G.Group of dtype);
        an object with the Group methods (add, run, poll, history, fetch_q,
        remove, solve_bytes, device_bytes) is driven through callbacks.
        clock: a callable giving the time in seconds (default: the C++
        server's steady clock, op2b_server_now)."""
        if policy not in ("fifo", "shortest"):
            raise ValueError("policy must be 'fifo' or 'shortest'")
        self.lib = _lib.load()
        self.dtype = np.dtype(dtype)
        self.group = group if group is not None else G.Group(dtype)
        self.keep_q = keep_q
        self.reqs = {}      # rid -> Request, until finished
        self._keep = {}     # rid -> the mesh struct and its arrays, until admitted
        self.active = {}    # sid -> Request
        self.done = []
        self.steps = 0
        ops = _lib.op2b_group_ops()
        if isinstance(self.group, G.Group):
            if self.lib.op2b_group_ops_fill(self.group.h, C.byref(ops)) != 0:
                raise RuntimeError("op2b_group_ops_fill failed")
        else:
            self._callbacks(ops)
        if clock is not None:
            self._now = _lib.NOW_FN(lambda ctx: float(clock()))
            ops.now = self._now
        self._ops = ops
        self.h = self.lib.op2b_server_create(C.byref(ops), int(budget_bytes), int(iters_per_step),
                                             int(max_active), 1 if policy == "shortest" else 0,
                                             1 if keep_q else 0, self.dtype.itemsize)
        if not self.h:
            raise RuntimeError("op2b_server_create: %s" % self.lib.op2b_last_error().decode())

    def _callbacks(self, ops):
        """The table of a group written in Python (a stand-in)."""
        g = self.group
        self._qs = {}

        def add(ctx, rid, m, mach, alpha, max_iter, rel_tol):
            return int(g.add(self.reqs[rid].mesh, mach, alpha, max_iter, rel_tol))

        def poll(ctx, ids, mx):
            got = list(g.poll())[:mx]
            for i, v in enumerate(got):
                ids[i] = v
            return len(got)

        def history(ctx, sid, out, mx):
            h = np.asarray(g.history(sid), np.float64)
            for i in range(min(mx, h.size)):
                out[i] = h[i]
            return int(h.size)

        def fetch_q(ctx, sid, q):
            self._qs[sid] = g.fetch_q(sid)
            return 0

        def remove(ctx, sid):
            g.remove(sid)
            return 0
        self._cb = [_lib.ADD_FN(add), _lib.RUN_FN(lambda ctx, n: int(g.run(n))),
                    _lib.POLL_FN(poll), _lib.HISTORY_FN(history), _lib.FETCHQ_FN(fetch_q),
                    _lib.REMOVE_FN(remove),
                    _lib.SOLVE_BYTES_FN(lambda ctx, rid, m, it:
                                        int(g.solve_bytes(self.reqs[rid].mesh, it))),
                    _lib.DEVICE_BYTES_FN(lambda ctx: int(g.device_bytes()))]
        (ops.add, ops.run, ops.poll, ops.history, ops.fetch_q, ops.remove, ops.solve_bytes,
         ops.device_bytes) = self._cb

    def now(self):
        return float(self.lib.op2b_server_now(self.h))

    def submit(self, req):
        if isinstance(req.mesh, M.AirfoilMesh):
            m, keep = M.as_struct(req.mesh)
        else:  # sizes only (a stand-in group never reads the arrays)
            m, keep = _lib.op2b_mesh(), []
            m.ncell = int(req.mesh.ncell)
            for k in ("nnode", "nedge", "nbedge"):
                setattr(m, k, int(getattr(req.mesh, k, 0)))
        self.reqs[req.rid] = req
        self._keep[req.rid] = (m, keep)
        rc = self.lib.op2b_server_submit(self.h, int(req.rid), C.byref(m), float(req.mach),
                                         float(req.alpha), int(req.max_iter), float(req.rel_tol),
                                         float(req.arrival))
        if rc != 0:
            raise ValueError("op2b_server_submit rejected request %r" % (req.rid,))

    def _sync_active(self):
        n = self.lib.op2b_server_active(self.h, None, None, 0)
        rids = (C.c_longlong * max(1, n))()
        sids = (C.c_int * max(1, n))()
        self.lib.op2b_server_active(self.h, rids, sids, n)
        self.active = {}
        for i in range(n):
            r = self.reqs[rids[i]]
            r.sid = sids[i]
            self._keep.pop(r.rid, None)  # admitted: the group has its own copy
            self.active[sids[i]] = r

    def step(self):
        """One round: admit, run k iterations, retire; returns the requests
        finished in this round."""
        if self.lib.op2b_server_step(self.h) < 0:
            raise RuntimeError("op2b_server_step: %s" % self.lib.op2b_last_error().decode())
        self._sync_active()
        out = []
        while True:
            buf = (_lib.op2b_served * 64)()
            n = self.lib.op2b_server_done(self.h, buf, 64)
            for i in range(n):
                rec = buf[i]
                r = self.reqs.pop(rec.rid)
                self._keep.pop(rec.rid, None)
                r.sid, r.iterations = rec.sid, rec.iterations
                r.admitted, r.finished = rec.admitted, rec.finished
                r.rms = np.zeros(max(1, rec.iterations), np.float64)
                got = self.lib.op2b_server_history(self.h, rec.rid,
                                                   r.rms.ctypes.data_as(C.POINTER(C.c_double)),
                                                   rec.iterations)
                r.rms = r.rms[:max(0, got)]
                if self.keep_q:
                    if isinstance(self.group, G.Group):
                        q = np.zeros((r.mesh.ncell, 4), self.dtype)
                        self.lib.op2b_server_q(self.h, rec.rid, q.ctypes.data)
                        r.q = q
                    else:
                        r.q = self._qs.pop(rec.sid, None)
                self.lib.op2b_server_release(self.h, rec.rid)
                out.append(r)
            if n < 64:
                break
        self.done.extend(out)
        self.steps += 1
        return out

    @property
    def peak_active(self):
        return int(self.lib.op2b_server_peak_active(self.h))

    @property
    def queued(self):
        return int(self.lib.op2b_server_queued(self.h))

    def idle(self):
        return bool(self.lib.op2b_server_idle(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.op2b_server_destroy(self.h)
            self.h = None
        if self.group is not None and hasattr(self.group, "close"):
            self.group.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def latency_stats(reqs):
    lat = np.array([r.finished - r.arrival for r in reqs], np.float64)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}
