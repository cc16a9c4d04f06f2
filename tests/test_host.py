"""Host-side API semantics that need no GPU: declaration and argument errors
print the reference's messages and exit with its codes
(common/op_lib_core.c:94-305), or return in RETURN mode.  Exiting cases run
in a subprocess."""
import os
import subprocess
import sys
import textwrap

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_py(code):
    full = "import sys; sys.path.insert(0, %r)\n" % ROOT + textwrap.dedent(code)
    r = subprocess.run([sys.executable, "-c", full], capture_output=True, text=True, timeout=120)
    return r.returncode, r.stdout + r.stderr


def test_zero_size_set_exits_like_reference():
    rc, out = run_py("""
        from oplus2_matlab_b200 import api
        api.op_decl_set(0, "empty")
        print("not reached")
    """)
    assert rc == 255
    assert "op_decl_set error -- negative/zero size for set: empty" in out
    assert "not reached" not in out


def test_bad_map_entry_exits_with_element_and_dimension():
    rc, out = run_py("""
        import numpy as np
        from oplus2_matlab_b200 import api
        a = api.op_decl_set(4, "a"); b = api.op_decl_set(3, "b")
        api.op_decl_map(a, b, 2, np.array([0, 1, 2, 0, 1, 3, 0, 0], np.int32), "m")
    """)
    assert rc == 255
    assert "op_decl_map error -- invalid data for map m" in out
    assert "element = 2, dimension = 1, map = 3" in out


def test_errors_return_in_return_mode():
    from oplus2_matlab_b200 import api
    old = api.set_error_mode(api.ERRORS_RETURN)
    try:
        api.clear_error()
        assert api.op_decl_set(-1, "neg") is None
        assert "negative/zero size" in api.last_error()
        api.clear_error()
        assert api.last_error() == ""
    finally:
        api.set_error_mode(old)


def _arg_check(arg_code):
    return run_py("""
        import ctypes as C, numpy as np
        from oplus2_matlab_b200 import api, _lib
        L = api.lib()
        cells = api.op_decl_set(3, "cells"); nodes = api.op_decl_set(4, "nodes")
        buf = np.zeros(16, np.float32)
        d = L.op_decl_dat_core(nodes, 2, b"float", 4, buf.ctypes.data, b"p_x")
        m = L.op_decl_map(cells, nodes, 2, np.array([0,1,1,2,2,3], np.int32).ctypes.data, b"pm")
        n = C.c_int(0)
        %s
        L.op_arg_check(cells, 1, arg, C.byref(n), b"loop")
        print("ninds", n.value)
    """ % arg_code)


def test_arg_check_accepts_valid_indirect_arg():
    rc, out = _arg_check('arg = L.op_arg_dat(d, 1, m, 2, b"float", api.OP_READ)')
    assert rc == 0 and "ninds 1" in out


def test_arg_check_rejects_type_dim_index_and_set_mismatch():
    cases = {
        'arg = L.op_arg_dat(d, 1, m, 2, b"double", api.OP_READ)': "dataset type does not match declared type",
        'arg = L.op_arg_dat(d, 1, m, 3, b"float", api.OP_READ)': "dataset dim does not match declared dim",
        'arg = L.op_arg_dat(d, 2, m, 2, b"float", api.OP_READ)': "invalid index",
        'arg = L.op_arg_dat(d, -1, None, 2, b"float", api.OP_READ)': "dataset set does not match loop set",
        'arg = L.op_arg_gbl_core(None, 1, b"float", api.OP_INC)': "NULL pointer for global data",
    }
    for code, msg in cases.items():
        rc, out = _arg_check(code)
        assert rc == 1, (code, out)
        assert 'error: arg 1 in kernel "loop"' in out and msg in out, (code, out)


def test_gbl_type_error_is_reported():
    rc, out = _arg_check('arg = api.op_arg_gbl(np.zeros(1, np.float64), 1, "float", api.OP_INC)')
    assert rc == 1 and "datatype does not match declared type" in out


def test_decl_dat_type_check():
    from oplus2_matlab_b200 import api
    import pytest
    s = api.op_decl_set(2, "s")
    with pytest.raises(TypeError):
        api.op_decl_dat(s, 1, "float", np.zeros(2, np.float64), "bad")
