"""op_checkpoint: save, then restart with fast-forward (doc/dev.tex:1080-1087).

A run saves a checkpoint after iteration 8 and goes on to 16.  A restarted
run with the same checkpoint file fast-forwards -- its first 8 iterations'
loop calls return the saved rms values without running -- restores every
dataset at the checkpoint and runs iterations 9-16.  Its rms history and
final fields must be bit-identical to the first run's, and to a run without
checkpointing.
"""
import os

import numpy as np
import pytest

from conftest import scratch_dir
from oplus2_matlab_b200 import _lib, api, apps
from oplus2_matlab_b200 import mesh as M

pytestmark = pytest.mark.gpu


def run(op2, m, niter, path=None, at=None, renumber=False):
    lib = _lib.load()
    op2.set_strategy(op2.STRATEGY_GATHER)
    op2.set_reduction(op2.REDUCE_TREE)
    if renumber:
        lib.op2b_set_renumber(1)
    resumed = lib.op2b_checkpoint_file(path.encode()) if path else 0
    A = apps.Airfoil(m, np.float32)
    hist, codes = [], []
    for it in range(1, niter + 1):
        hist.append(A.iteration())
        if path and it == at:
            codes.append(lib.op_checkpoint())
    st = A.fetch()
    assert op2.last_error() == ""
    return resumed, codes, np.array(hist), {k: v.copy() for k, v in st.items()}


@pytest.mark.parametrize("renumber", [False, True])
def test_fast_forward_restart_is_bit_identical(op2, renumber):
    m = M.naca0012(30, 45)
    path = os.path.join(scratch_dir(), "airfoil.ckpt")
    r1, c1, h1, s1 = run(op2, m, 16, path, at=8, renumber=renumber)
    assert (r1, c1) == (0, [1]) and os.path.exists(path)
    api.op_exit()
    api.op_init([], 0)
    r2, c2, h2, s2 = run(op2, m, 16, path, at=8, renumber=renumber)
    assert (r2, c2) == (1, [2])  # resumed at the checkpoint
    assert h2.tobytes() == h1.tobytes()
    for k in ("q", "qold", "res", "adt"):
        assert s2[k].tobytes() == s1[k].tobytes(), k
    api.op_exit()
    api.op_init([], 0)
    _, _, h3, s3 = run(op2, m, 16, renumber=renumber)
    assert h3.tobytes() == h1.tobytes()
    assert s3["q"].tobytes() == s1["q"].tobytes()


def test_mismatched_restart_is_an_error(op2):
    m = M.naca0012(20, 30)
    path = os.path.join(scratch_dir(), "airfoil.ckpt")
    run(op2, m, 6, path, at=3)
    api.op_exit()
    api.op_init([], 0)
    lib = _lib.load()
    assert lib.op2b_checkpoint_file(path.encode()) == 1
    A = apps.Airfoil(m, np.float32)
    for _ in range(4):  # passes the saved checkpoint without calling op_checkpoint
        A.iteration()
    assert "op_checkpoint error" in op2.last_error()
    op2.clear_error()
