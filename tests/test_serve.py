"""The continuous-batching server (oplus2_matlab_b200/serve.py) and the
sharding of independent instances over ranks.

Sharding is host logic: checked here directly and with two gloo ranks on
the CPU, each taking its share and the union gathered.  The server runs on
the GPU: a request stream under a budget that forces queuing must finish
every request, and each answer must be bit-identical to the same request
solved alone.
"""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from oplus2_matlab_b200 import group as G
from oplus2_matlab_b200 import mesh as M
from oplus2_matlab_b200 import serve as S


def test_shard_by_cells_is_a_balanced_partition():
    cells = [720000, 20000, 350000, 90000, 90000, 500000, 31000, 64000]
    for world in (1, 2, 3, 8):
        parts = S.shard_by_cells(cells, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cells)))
        loads = [sum(cells[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(cells)
    assert S.shard_by_cells(cells, 2) == S.shard_by_cells(list(cells), 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    inst = G.draw_instances(64, cmin=20000, cmax=720000)
    cells = [3 * I * J for I, J, _, _ in inst]
    mine = S.shard_by_cells(cells, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, (mine, sum(cells[i] for i in mine)))
    if rank == 0:
        out.put(got)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_cover_every_instance_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    ids = sorted(i for mine, _ in got for i in mine)
    assert ids == list(range(64))
    loads = [c for _, c in got]
    assert abs(loads[0] - loads[1]) <= 720000


@pytest.mark.gpu
def test_served_answers_equal_alone_answers(op2):
    specs = [((20, 30), 0.40, 0.0, 30), ((30, 45), 0.60, 2.0, 25), ((20, 30), 0.55, -1.0, 40),
             ((40, 60), 0.35, 4.0, 20), ((30, 45), 0.50, 1.0, 35)]
    meshes = {ij: M.naca0012(*ij) for ij, _, _, _ in specs}
    one = G.Group()
    per_solve = max(one.solve_bytes(m, 40) for m in meshes.values())
    one.close()
    srv = S.Server(budget_bytes=int(2.5 * per_solve), iters_per_step=4, keep_q=True,
                   clock=lambda: 0.0)
    for k, (ij, mach, alpha, n) in enumerate(specs):
        srv.submit(S.Request(k, meshes[ij], mach, alpha, n, 0.0, 0.0))
    while not srv.idle():
        srv.step()
    assert srv.peak_active < len(specs)  # the budget made requests queue
    assert sorted(r.rid for r in srv.done) == list(range(len(specs)))
    for r in srv.done:
        ij, mach, alpha, n = specs[r.rid]
        g = G.Group()
        sid = g.add(meshes[ij], mach, alpha, n)
        g.run(n)
        assert r.iterations == n
        assert r.q.tobytes() == g.fetch_q(sid).tobytes()
        assert r.rms.tobytes() == g.history(sid).tobytes()
        g.close()
    srv.close()


@pytest.mark.gpu
def test_concurrency_cap_and_shortest_first_policy(op2):
    sizes = [(40, 60), (20, 30), (30, 45), (20, 30)]
    meshes = {ij: M.naca0012(*ij) for ij in sizes}
    srv = S.Server(iters_per_step=5, clock=lambda: 0.0, max_active=1, policy="shortest")
    for k, ij in enumerate(sizes):
        srv.submit(S.Request(k, meshes[ij], 0.5, 0.0, 10, 0.0, 0.0))
    while not srv.idle():
        srv.step()
    assert srv.peak_active == 1
    # one at a time, least work first (ties in arrival order)
    assert [r.rid for r in srv.done] == [1, 3, 2, 0]
    srv.close()
