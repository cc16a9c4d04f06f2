"""op2b_update_noalloc: the airfoil update for callers that cannot allocate
device memory (their allocator owns the GPU, or a cudaMalloc would stall
them).  Called through the C ABI on arrays this test owns, it must match the
library's normal update entry point (op_par_loop_update) -- q and res bit
for bit, the rms within the FP32 tolerance the other tests use -- on two
calls in a row, since both calls share the library's fixed scratch array.
This file sorts last so a stop-at-first-failure run has done everything else.
The argument checks run on the host before anything touches the GPU, so
they are tested without one.
"""
import ctypes as C

import numpy as np
import pytest

from oplus2_matlab_b200 import _lib, apps
from oplus2_matlab_b200 import mesh as M


def _cudart():
    for name in ("libcudart.so.12", "libcudart.so"):
        try:
            rt = C.CDLL(name)
            break
        except OSError:
            continue
    rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    rt.cudaFree.argtypes = [C.c_void_p]
    rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    return rt


H2D, D2H = 1, 2


def test_update_noalloc_rejects_misaligned_pointers_before_launch():
    """qold, q and res are 16-byte vectors in the kernel; a misaligned
    pointer would fault on the device, so it is refused on the host (-3),
    as are null pointers and sizes beyond the fixed scratch (-1).  The
    pointers below are never dereferenced: every case returns first."""
    lib = _lib.load()
    ok16, ok4 = 0x10000, 0x20000
    assert lib.op2b_update_noalloc(64, ok16 + 4, ok16, ok16, ok4, ok4, None) == -3  # qold
    assert lib.op2b_update_noalloc(64, ok16, ok16 + 8, ok16, ok4, ok4, None) == -3  # q
    assert lib.op2b_update_noalloc(64, ok16, ok16, ok16 + 12, ok4, ok4, None) == -3  # res
    assert lib.op2b_update_noalloc(64, ok16, ok16, ok16, ok4 + 2, ok4, None) == -3  # adt
    assert lib.op2b_update_noalloc(64, ok16, ok16, ok16, ok4, ok4 + 1, None) == -3  # rms
    assert lib.op2b_update_noalloc(64, None, ok16, ok16, ok4, ok4, None) == -3
    assert lib.op2b_update_noalloc(4096 * 1024 + 1, ok16, ok16, ok16, ok4, ok4, None) == -1
    assert lib.op2b_update_noalloc(-1, ok16, ok16, ok16, ok4, ok4, None) == -1
    assert lib.op2b_update_noalloc(0, None, None, None, None, None, None) == 0


@pytest.mark.gpu
def test_update_noalloc_matches_op_par_loop_update(op2):
    m = M.naca0012(100, 150)  # 45,000 cells
    n = m.ncell
    rng = np.random.default_rng(20261203)
    state = {"q": np.zeros((n, 4), np.float32),
             "qold": rng.uniform(0.5, 2.0, (n, 4)).astype(np.float32),
             "res": rng.normal(0.0, 1e-3, (n, 4)).astype(np.float32),
             "adt": rng.uniform(1.0, 50.0, (n, 1)).astype(np.float32)}

    # the library's own entry point, through op_par_loop_update
    A = apps.Airfoil(m, np.float32, state=state)
    A.rms[0] = 0
    A.loop("update")
    got = A.fetch()
    q_ref, res_ref, rms_ref = got["q"].copy(), got["res"].copy(), float(A.rms[0])
    assert op2.last_error() == ""
    assert np.all(res_ref == 0) and rms_ref > 0

    lib = _lib.load()
    rt = _cudart()
    bufs = {}
    for k, nbytes in (("qold", 16 * n), ("q", 16 * n), ("res", 16 * n), ("adt", 4 * n), ("rms", 4)):
        p = C.c_void_p()
        assert rt.cudaMalloc(C.byref(p), nbytes) == 0
        bufs[k] = p
    try:
        for call in range(2):  # two calls in a row share the fixed scratch
            for k in ("qold", "res", "adt"):
                a = np.ascontiguousarray(state[k])
                assert rt.cudaMemcpy(bufs[k], a.ctypes.data, a.nbytes, H2D) == 0
            zero = np.zeros(1, np.float32)
            assert rt.cudaMemcpy(bufs["rms"], zero.ctypes.data, 4, H2D) == 0
            rc = lib.op2b_update_noalloc(n, bufs["qold"], bufs["q"], bufs["res"], bufs["adt"],
                                         bufs["rms"], None)
            assert rc == 0, rc
            assert rt.cudaDeviceSynchronize() == 0
            q = np.empty((n, 4), np.float32)
            res = np.empty((n, 4), np.float32)
            rms = np.empty(1, np.float32)
            assert rt.cudaMemcpy(q.ctypes.data, bufs["q"], q.nbytes, D2H) == 0
            assert rt.cudaMemcpy(res.ctypes.data, bufs["res"], res.nbytes, D2H) == 0
            assert rt.cudaMemcpy(rms.ctypes.data, bufs["rms"], 4, D2H) == 0
            assert np.array_equal(q, q_ref), call
            assert np.array_equal(res, res_ref), call
            # both are fixed-shape tree sums of the same 180,000 squares
            assert abs(float(rms[0]) - rms_ref) <= 1e-5 * rms_ref, (call, float(rms[0]), rms_ref)

        # beyond the scratch's capacity: rejected, nothing launched
        assert lib.op2b_update_noalloc(4096 * 1024 + 1, bufs["qold"], bufs["q"], bufs["res"],
                                       bufs["adt"], bufs["rms"], None) == -1
        assert rt.cudaDeviceSynchronize() == 0
    finally:
        for p in bufs.values():
            rt.cudaFree(p)
