"""The server's admission logic on the host, driven against a stand-in
group: arrival order or least work first, the memory budget, the cap on
solves iterated together, retirement and the latency record.  The group
engine itself is tested on the GPU (tests/test_group.py, tests/test_serve.py)."""
from types import SimpleNamespace

import numpy as np

from oplus2_matlab_b200 import serve as S


class StandInGroup:
    """Solves that each stop after their iteration cap; device bytes are
    cells x 100."""

    def __init__(self):
        self.solves, self.order = {}, []

    def add(self, mesh, mach, alpha, max_iter, rel_tol=0.0):
        sid = len(self.order)
        self.solves[sid] = {"cells": mesh.ncell, "left": max_iter, "done": 0}
        self.order.append(sid)
        return sid

    def run(self, niter):
        for s in self.solves.values():
            step = min(niter, s["left"])
            s["left"] -= step
            s["done"] += step
        return len(self.solves)

    def poll(self):
        return [sid for sid, s in self.solves.items() if s["left"] == 0]

    def history(self, sid):
        return np.ones(self.solves[sid]["done"])

    def fetch_q(self, sid):
        return None

    def remove(self, sid):
        del self.solves[sid]

    def solve_bytes(self, mesh, max_iter):
        return mesh.ncell * 100

    def device_bytes(self):
        return sum(s["cells"] * 100 for s in self.solves.values())

    def close(self):
        pass


def request(rid, cells, iters, arrival=0.0):
    return S.Request(rid, SimpleNamespace(ncell=cells), 0.5, 0.0, iters, 0.0, arrival)


def test_fifo_admits_in_arrival_order_under_the_budget():
    clock = iter(range(1000)).__next__
    srv = S.Server(budget_bytes=250, iters_per_step=5, clock=clock, group=StandInGroup())
    reqs = [request(i, 1, 10) for i in range(5)]
    for r in reqs:
        srv.submit(r)
    srv.step()
    assert sorted(r.rid for r in srv.active.values()) == [0, 1]  # 2 x 100 bytes fit in 250
    while not srv.idle():
        srv.step()
    assert sorted(r.rid for r in srv.done) == [0, 1, 2, 3, 4]
    assert all(r.iterations == 10 for r in srv.done)
    by_admission = sorted(srv.done, key=lambda r: (r.admitted, r.sid))
    assert [r.rid for r in by_admission] == [0, 1, 2, 3, 4]


def test_cap_and_shortest_first():
    g = StandInGroup()
    srv = S.Server(budget_bytes=10**9, iters_per_step=1, group=g, max_active=2,
                   policy="shortest", clock=iter(range(1000)).__next__)
    work = {0: (3, 40), 1: (1, 10), 2: (2, 10), 3: (1, 5)}  # rid: (cells, iterations)
    for rid, (c, n) in work.items():
        srv.submit(request(rid, c, n))
    srv.step()
    assert len(srv.active) == 2
    # least cells x iterations first: rid 3 (5), then rid 1 (10)
    assert [g.order.index(r.sid) for r in srv.active.values()] == [0, 1]
    assert sorted(r.rid for r in srv.active.values()) == [1, 3]
    while not srv.idle():
        srv.step()
        assert len(srv.active) <= 2
    assert srv.peak_active == 2
    by_admission = [r.rid for r in sorted(srv.done, key=lambda r: (r.admitted, r.sid))]
    assert by_admission[:2] == [1, 3] or by_admission[:2] == [3, 1]
    assert set(by_admission) == {0, 1, 2, 3}


def test_latency_stats():
    reqs = [SimpleNamespace(arrival=0.0, finished=float(t)) for t in range(1, 101)]
    st = S.latency_stats(reqs)
    assert abs(st["p50_s"] - 50.5) < 1e-9 and abs(st["p99_s"] - 99.01) < 1e-9
    assert st["max_s"] == 100.0


def test_server_latency_record_matches_latency_stats():
    """The C++ server's own latency record (op2b_server_latency) against the
    same numbers computed from the finished requests."""
    import ctypes as C
    t = iter(range(0, 10000, 3)).__next__
    srv = S.Server(budget_bytes=350, iters_per_step=4, clock=t, group=StandInGroup())
    for i in range(7):
        srv.submit(request(i, 1 + i % 3, 6 + 2 * i, arrival=float(i)))
    while not srv.idle():
        srv.step()
    vals = [C.c_double() for _ in range(4)]
    assert srv.lib.op2b_server_latency(srv.h, *[C.byref(v) for v in vals]) == 0
    st = S.latency_stats(srv.done)
    for got, key in zip(vals, ("p50_s", "p99_s", "mean_s", "max_s")):
        assert abs(got.value - st[key]) < 1e-12, key
    assert srv.queued == 0 and not srv.active
    srv.close()
