"""Continuous-batching solve server over one GPU's group engine.

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

shard_by_cells splits a list of instances over ranks (GPUs) by greedy
balance of cell counts: instances are independent, so N GPUs need no
collective, only the gather of results.
"""
import time
from collections import deque

import numpy as np

from . import group as G


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
    """Admit, iterate and retire solves on one GPU."""

    def __init__(self, dtype=np.float32, budget_bytes=150 * 10**9, iters_per_step=10,
                 keep_q=False, clock=time.perf_counter, max_active=0, policy="fifo",
                 group=None):
        """max_active > 0 caps the solves iterated together (0: memory budget
        only); policy "fifo" admits in arrival order, "shortest" admits the
        queued request with the least work (cells x iteration cap) first.
        group: the solve group to drive (default: a new G.Group of dtype)."""
        if policy not in ("fifo", "shortest"):
            raise ValueError("policy must be 'fifo' or 'shortest'")
        self.group = group if group is not None else G.Group(dtype)
        self._unsorted = False
        self.budget = int(budget_bytes)
        self.k = int(iters_per_step)
        self.keep_q = keep_q
        self.clock = clock
        self.max_active = int(max_active)
        self.policy = policy
        self.queue = deque()
        self.active = {}  # sid -> Request
        self.done = []
        self.peak_active = 0
        self.steps = 0

    def submit(self, req):
        self.queue.append(req)
        self._unsorted = True

    def _admit(self, now):
        g = self.group
        if self.policy == "shortest" and self._unsorted and len(self.queue) > 1:
            self.queue = deque(sorted(self.queue, key=lambda q: (q.mesh.ncell * q.max_iter,
                                                                 q.arrival)))
        self._unsorted = False
        while self.queue:
            if self.max_active and len(self.active) >= self.max_active:
                break
            r = self.queue[0]
            need = g.solve_bytes(r.mesh, r.max_iter)
            if self.active and g.device_bytes() + need > self.budget:
                break  # the head of the queue waits for memory
            self.queue.popleft()
            r.sid = g.add(r.mesh, r.mach, r.alpha, r.max_iter, r.rel_tol)
            r.admitted = now
            self.active[r.sid] = r
        self.peak_active = max(self.peak_active, len(self.active))

    def step(self):
        """One round: admit, run k iterations, retire; returns the requests
        finished in this round."""
        now = self.clock()
        if not self.active:
            self._admit(now)
        if not self.active:
            return []
        self.group.run(self.k)
        # admissions overlap the iterations just enqueued
        self._admit(self.clock())
        finished = self.group.poll()
        t = self.clock()
        out = []
        for sid in finished:
            r = self.active.pop(sid, None)
            if r is None:
                continue
            r.finished = t
            r.rms = self.group.history(sid)
            r.iterations = len(r.rms)
            if self.keep_q:
                r.q = self.group.fetch_q(sid)
            self.group.remove(sid)
            out.append(r)
        self.done.extend(out)
        self.steps += 1
        return out

    def idle(self):
        return not self.active and not self.queue

    def close(self):
        self.group.close()


def latency_stats(reqs):
    lat = np.array([r.finished - r.arrival for r in reqs], np.float64)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}
