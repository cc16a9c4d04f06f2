"""op_decl_dat of a large pageable array holding only zero bytes clears the
device buffer instead of copying (op2b_h2d_bytes counts what was copied):
the dataset reads back as the array, a single nonzero byte anywhere (here
the very last one) makes it a copy, and the airfoil fields are unchanged
whether the scan is on or off."""
import numpy as np
import pytest

from oplus2_matlab_b200 import api, apps
from oplus2_matlab_b200 import mesh as M

pytestmark = pytest.mark.gpu

N = 1 << 19  # cells of 4 floats: 8 MiB, above the 1 MiB threshold


def declare(arr):
    lib = api.lib()
    api.set_error_mode(api.ERRORS_RETURN)
    api.op_init([], 0)
    s = api.op_decl_set(arr.shape[0], "cells")
    lib.op2b_h2d_bytes(1)
    d = api.op_decl_dat(s, 4, "float", arr, "d")
    copied = lib.op2b_h2d_bytes(1)
    arr[...] = 7.0  # op_fetch_data writes the device values into the declared array
    api.op_fetch_data(d)
    got = arr.copy()
    err = api.last_error()
    api.op_exit()
    assert err == "", err
    return copied, got


def test_zero_array_is_cleared_not_copied():
    a = np.zeros((N, 4), np.float32)
    copied, got = declare(a)
    assert copied == 0
    assert not np.any(got.view(np.uint32))  # +0.0 everywhere


def test_one_nonzero_byte_makes_a_copy():
    a = np.zeros((N, 4), np.float32)
    a.view(np.uint8).reshape(-1)[-1] = 1  # the last byte
    want = a.copy()
    copied, got = declare(a)
    assert copied == a.nbytes
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_negative_zero_is_copied():
    a = np.zeros((N, 4), np.float32)
    a[N // 2, 1] = -0.0  # not zero bytes
    want = a.copy()
    copied, got = declare(a)
    assert copied == a.nbytes
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_airfoil_fields_same_with_scan_off():
    """A mesh whose qold, adt and res arrays are above the threshold."""
    m = M.naca0012(400, 600)
    lib = api.lib()
    out = []
    for scan in (1, 0):
        api.set_error_mode(api.ERRORS_RETURN)
        api.op_init([], 0)
        api.set_strategy(api.STRATEGY_GATHER)
        lib.op2b_set_tuning(b"decl_zero_scan", scan)
        try:
            lib.op2b_h2d_bytes(1)
            A = apps.Airfoil(m, np.float32)
            copied = lib.op2b_h2d_bytes(1)
            A.iterate(3)
            out.append(({k: v.copy() for k, v in A.fetch().items()}, copied))
            assert api.last_error() == ""
        finally:
            lib.op2b_set_tuning(b"decl_zero_scan", 1)
            api.op_exit()
    (a, ca), (b, cb) = out
    for k in ("q", "qold", "res", "adt"):
        assert np.array_equal(a[k], b[k]), k
    # qold (16 B/cell), adt (4) and res (16) were cleared, not copied
    assert cb - ca == 36 * m.ncell
