"""The bench's multi-rank plumbing (one process per GPU under torchrun):
ranks meet at barriers and every timing is the maximum over ranks.  Run here
as two gloo ranks on host tensors (OP2B_DIST_BACKEND=gloo), through the same
Dist class bench.py uses with NCCL."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank), OP2B_DIST_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    d.barrier()
    m = d.max(1.5 + rank)  # each rank's "time"
    out.put((rank, d.world, m))
    d.close()


def test_two_gloo_ranks_take_the_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert got == [(0, 2, 2.5), (1, 2, 2.5)]
