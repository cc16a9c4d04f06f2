"""The grouped (batched / served) airfoil engine, include/op2b_group.h.

Against the plain path: every solve's flow field q must equal, bit for bit,
the plain op_par_loop solve of the same mesh and flow condition (same device
arithmetic, same contribution order); the rms history, summed in a different
order, within the tree-reduction tolerance of the plain tests.  Against
itself: a solve's q and rms history must be bit-identical alone and in any
mix, whenever it joins, and whatever launch shape the autotuner picks.
"""
import numpy as np
import pytest

from oplus2_matlab_b200 import group as G
from oplus2_matlab_b200 import mesh as M
from oplus2_matlab_b200.apps import airfoil_consts

RMS_RTOL = 5e-5  # FP32 tree-order rms tolerance of the plain tests at 7.2k cells

MESHES = {}


def mesh(I, J):
    if (I, J) not in MESHES:
        MESHES[(I, J)] = M.naca0012(I, J)
    return MESHES[(I, J)]


# ------------------------------------------------------------------ CPU ----

def test_flow_qinf_is_the_reference_free_stream():
    for dt in (np.float32, np.float64):
        q, c = G.flow_qinf(0.4, 0.0, dt)
        ref = airfoil_consts(dt)
        assert q.tobytes() == np.asarray(ref["qinf"], dt).tobytes()
        assert c.tobytes() == np.asarray([ref["gam"], ref["gm1"], ref["cfl"], ref["eps"]],
                                         dt).tobytes()


def test_flow_qinf_turns_the_velocity_by_alpha():
    q0, _ = G.flow_qinf(0.5, 0.0, np.float64)
    q, _ = G.flow_qinf(0.5, 4.0, np.float64)
    a = np.float32(4.0) * np.arctan(1.0) / 45.0
    assert q[0] == q0[0] and q[3] == q0[3]
    assert np.hypot(q[1], q[2]) == pytest.approx(q0[1], rel=1e-15)
    assert np.arctan2(q[2], q[1]) == pytest.approx(a, rel=1e-12)


def test_instance_draw_is_seeded_and_in_range():
    a = G.draw_instances(64)
    b = G.draw_instances(64)
    assert a == b
    assert a != G.draw_instances(64, seed=1)
    for I, J, mach, alpha in a:
        cells = 3 * I * J
        assert 17000 < cells < 760000
        assert 0.3 <= mach <= 0.7 and -2.0 <= alpha <= 6.0
    assert G.mesh_dims(720000) == (400, 600)


# ------------------------------------------------------------------ GPU ----

CASES = [((20, 30), 0.40, 0.0), ((30, 45), 0.55, 3.5), ((40, 60), 0.35, -1.5)]


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_group_matches_plain_solves(op2, dtype):
    niter = 25
    g = G.Group(dtype)
    ids = [g.add(mesh(*ij), mach, alpha, niter) for ij, mach, alpha in CASES]
    g.run(niter)
    g.sync()
    for sid, (ij, mach, alpha) in zip(ids, CASES):
        qp, rp, _ = G.plain_solve(mesh(*ij), mach, alpha, niter, dtype)
        assert g.iterations(sid) == niter
        qg = g.fetch_q(sid)
        assert qg.tobytes() == qp.astype(dtype).tobytes(), (ij, mach, alpha)
        rtol = RMS_RTOL if dtype == np.float32 else 1e-12
        np.testing.assert_allclose(g.history(sid), rp, rtol=rtol)
    g.close()


@pytest.mark.gpu
def test_solve_alone_equals_solve_in_mix(op2):
    niter = 20
    alone = G.Group()
    a = alone.add(mesh(30, 45), 0.6, 2.0, niter)
    alone.run(niter)
    qa, ha = alone.fetch_q(a), alone.history(a)
    alone.close()

    mix = G.Group()
    mix.add(mesh(40, 60), 0.45, -1.0, niter)
    b = mix.add(mesh(30, 45), 0.6, 2.0, niter)
    mix.add(mesh(20, 30), 0.35, 5.0, 7)  # stops early, inside the run
    mix.run(niter)
    assert mix.fetch_q(b).tobytes() == qa.tobytes()
    assert mix.history(b).tobytes() == ha.tobytes()
    mix.close()


@pytest.mark.gpu
def test_late_join_and_extra_runs_do_not_change_a_solve(op2):
    niter = 15
    ref = G.Group()
    r = ref.add(mesh(20, 30), 0.5, 1.0, niter)
    ref.run(niter)
    qr, hr = ref.fetch_q(r), ref.history(r)
    ref.close()

    g = G.Group()
    g.add(mesh(40, 60), 0.4, 0.0, 100)
    g.run(6)
    late = g.add(mesh(20, 30), 0.5, 1.0, niter)  # joins at the next run
    g.run(niter + 5)  # 5 more than it needs: a stopped solve stays as it was
    assert g.iterations(late) == niter
    assert g.fetch_q(late).tobytes() == qr.tobytes()
    assert g.history(late).tobytes() == hr.tobytes()
    g.close()


@pytest.mark.gpu
def test_relative_tolerance_stops_at_the_first_qualifying_iteration(op2):
    g = G.Group()
    tol = 0.7
    sid = g.add(mesh(20, 30), 0.5, 0.0, 200, rel_tol=tol)
    g.run(200)
    h = g.history(sid)
    n = g.iterations(sid)
    assert n == len(h)
    expect = next((k for k in range(2, 201) if k == 200 or h[k - 1] < tol * h[0]), None)
    # the rule is applied in the solve's real type
    assert n == expect
    assert n < 200
    g.close()


@pytest.mark.gpu
def test_poll_reports_each_stopped_solve_once_and_remove_frees(op2):
    g = G.Group()
    short = g.add(mesh(20, 30), 0.4, 0.0, 3)
    long_ = g.add(mesh(20, 30), 0.4, 0.0, 50)
    g.run(5)
    assert g.poll() == [short]
    assert g.poll() == []
    before = g.device_bytes()
    g.remove(short)
    assert g.device_bytes() < before
    assert g.run(2) == 1  # only the long solve is launched
    g.run(45)
    assert g.poll() == [long_]
    assert g.iterations(long_) == 50
    g.close()


@pytest.mark.gpu
def test_autotune_keeps_state_and_results(op2):
    niter = 12
    a = G.Group()
    ia = a.add(mesh(40, 60), 0.45, 2.0, niter)
    a.run(niter)
    qa = a.fetch_q(ia)
    a.close()

    b = G.Group()
    ib = b.add(mesh(40, 60), 0.45, 2.0, niter)
    best = b.autotune(iters=3)
    assert best in (512, 1024, 2048, 4096, 8192) and b.edge_tile == best
    assert b.iterations(ib) == 0
    b.run(niter)
    assert b.fetch_q(ib).tobytes() == qa.tobytes()
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("block_bytes,streams", [(1 << 20, 2), (1 << 19, 3), (-1, 4)])
def test_blocks_on_several_streams_give_the_same_solves(op2, block_bytes, streams):
    """Blocks of solves dealt to several streams of the captured iteration
    (their passes overlap) leave every solve bit-identical, including one
    that stops early inside the run."""
    niter = 15
    specs = [((40, 60), 0.45, -1.0, niter), ((30, 45), 0.6, 2.0, niter),
             ((20, 30), 0.35, 5.0, 7), ((30, 45), 0.5, 0.0, niter), ((20, 30), 0.7, 3.0, niter)]
    ref = G.Group()
    ids = [ref.add(mesh(*ij), m, a, n) for ij, m, a, n in specs]
    ref.run(niter)
    want = [(ref.fetch_q(i).tobytes(), ref.history(i).tobytes()) for i in ids]
    ref.close()
    g = G.Group()
    g.set_block_bytes(block_bytes)
    g.set_streams(streams)
    ids = [g.add(mesh(*ij), m, a, n) for ij, m, a, n in specs]
    g.run(niter)
    got = [(g.fetch_q(i).tobytes(), g.history(i).tobytes()) for i in ids]
    g.close()
    assert got == want


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("block_bytes,streams", [(-1, 1), (1 << 20, 2)])
def test_tiled_group_fields_equal_two_launch_group(op2, dtype, block_bytes, streams):
    """The tiled chain (one launch per update over all solves, fluxes in
    shared memory, q and adt double-buffered) gives every solve the q of the
    two-launch form bit for bit, on meshes of several tiles (edges between
    tiles computed twice) and with a solve that stops early; the rms agrees
    to summation order and stops the same solve at the same iteration."""
    niter = 12
    specs = [((100, 150), 0.45, -1.0, niter), ((40, 60), 0.6, 2.0, niter),
             ((20, 30), 0.35, 5.0, 5), ((120, 90), 0.5, 0.0, niter)]
    ref = G.Group(dtype)
    ids = [ref.add(mesh(*ij), m, a, n) for ij, m, a, n in specs]
    ref.run(niter)
    want = [(ref.fetch_q(i).tobytes(), ref.history(i)) for i in ids]
    ref.close()
    g = G.Group(dtype)
    g.set_tiled(True)
    g.set_block_bytes(block_bytes)
    g.set_streams(streams)
    ids = [g.add(mesh(*ij), m, a, n) for ij, m, a, n in specs]
    g.run(niter)
    assert g.lib.op2b_group_tiled(g.h) == 1
    for i, (wq, wh) in zip(ids, want):
        assert g.fetch_q(i).tobytes() == wq
        h = g.history(i)
        assert len(h) == len(wh)
        rtol = RMS_RTOL if dtype == np.float32 else 1e-12
        np.testing.assert_allclose(h, wh, rtol=rtol)
    g.close()


@pytest.mark.gpu
def test_tiled_group_solve_alone_equals_in_mix_and_late_switch(op2):
    """Tiled: a solve alone equals the same solve in a mix (q and rms), and
    switching a running group to the tiled chain between runs keeps q."""
    niter = 10
    alone = G.Group()
    alone.set_tiled(True)
    a = alone.add(mesh(100, 150), 0.6, 2.0, niter)
    alone.run(niter)
    qa, ha = alone.fetch_q(a), alone.history(a)
    alone.close()
    mix = G.Group()
    mix.set_tiled(True)
    mix.add(mesh(40, 60), 0.45, -1.0, niter)
    b = mix.add(mesh(100, 150), 0.6, 2.0, niter)
    mix.add(mesh(20, 30), 0.35, 5.0, 4)
    mix.run(niter)
    assert mix.fetch_q(b).tobytes() == qa.tobytes()
    assert mix.history(b).tobytes() == ha.tobytes()
    mix.close()
    ref = G.Group()
    r = ref.add(mesh(100, 150), 0.6, 2.0, niter)
    ref.run(niter)
    qr = ref.fetch_q(r)
    ref.close()
    sw = G.Group()
    c = sw.add(mesh(100, 150), 0.6, 2.0, niter)
    sw.run(4)
    sw.set_tiled(True)  # joined solves get their tile lists at the next run
    sw.run(niter - 4)
    assert sw.fetch_q(c).tobytes() == qr.tobytes()
    sw.close()


@pytest.mark.gpu
def test_autotune_on_real_iterations_counts_them(op2):
    """op2b_group_autotune_run times each launch shape on real iterations of
    the active solves: after it and the remaining iterations, every solve
    (one of them stopping during the trials) is bit-identical, q and rms
    history, to an untuned run of the same length."""
    niter = 30
    specs = [((40, 60), 0.45, -1.0, niter), ((30, 45), 0.6, 2.0, niter),
             ((20, 30), 0.35, 5.0, 5)]
    ref = G.Group()
    ids = [ref.add(mesh(*ij), m, a, n) for ij, m, a, n in specs]
    ref.run(niter)
    want = [(ref.fetch_q(i).tobytes(), ref.history(i).tobytes()) for i in ids]
    ref.close()
    g = G.Group()
    ids = [g.add(mesh(*ij), m, a, n) for ij, m, a, n in specs]
    ran = g.autotune_run(2)
    assert ran == 22  # 11 launch shapes x 2 iterations
    g.run(niter - ran)
    got = [(g.fetch_q(i).tobytes(), g.history(i).tobytes()) for i in ids]
    g.close()
    assert got == want


@pytest.mark.gpu
def test_lazy_retire_and_async_fetch_keep_results(op2):
    """Stopped solves stay in the captured iteration until a quarter of its
    cells have stopped (their CTAs return at once), and their q can be
    copied out while the others iterate: every solve ends bit-identical to
    the same solves run with a rebuild at every stop and synchronous
    fetches."""
    niter = 24
    specs = [((40, 60), 0.45, -1.0, niter), ((30, 45), 0.6, 2.0, 6),
             ((20, 30), 0.35, 5.0, 9), ((40, 60), 0.5, 0.0, 15), ((30, 45), 0.7, 3.0, niter)]

    def run(lazy):
        from oplus2_matlab_b200 import api
        api.lib().op2b_set_tuning(b"group_lazy_retire", 1 if lazy else 0)
        try:
            g = G.Group()
            ids = [g.add(mesh(*ij), m, a, n) for ij, m, a, n in specs]
            out = {}
            stopped = 0
            while stopped < len(ids):
                g.run(4)
                done = g.poll()
                stopped += len(done)
                for sid in done:
                    buf = np.zeros((g.ncell[sid], 4), np.float32)
                    out[sid] = g.fetch_q_async(sid, buf) if lazy else g.fetch_q(sid, buf)
            g.sync()
            res = [(out[i].tobytes(), g.history(i).tobytes(), g.iterations(i)) for i in ids]
            g.close()
            return res
        finally:
            api.lib().op2b_set_tuning(b"group_lazy_retire", 1)

    assert run(True) == run(False)
