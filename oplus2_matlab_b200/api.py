"""Python mirror of the OP2 user API (include/op_lib.h), over the C ABI.

Names, argument order and meaning follow the reference's C API
(common/op_lib.h:101-190; doc/user.tex:269-430) so that a loop written here
reads like the reference apps:

    nodes = op_decl_set(nnode, "nodes")
    pedge = op_decl_map(edges, nodes, 2, edge, "pedge")
    p_x   = op_decl_dat(nodes, 2, "float", x, "p_x")
    op_decl_const("gam", 1, "float", gam)
    op_par_loop("res_calc", edges,
                op_arg_dat(p_x, 0, pedge, 2, "float", OP_READ), ...)

numpy arrays handed to op_decl_map / op_decl_dat / op_arg_gbl are borrowed
by the library exactly as in C (the pointer is stored), so this module keeps
them alive until op_exit.  op_fetch_data writes the device copy back into the
array given to op_decl_dat and returns it.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import (OP_INC, OP_MAX, OP_MIN, OP_READ, OP_RW, OP_WRITE, op_arg,  # noqa: F401
                   REDUCE_SEQ, REDUCE_TREE, STRATEGY_AUTO, STRATEGY_COLOURED, STRATEGY_GATHER,
                   ERRORS_EXIT, ERRORS_RETURN)

OP_ID = None
OP_GBL = None

_TYPES = {"float": np.float32, "double": np.float64, "int": np.int32, "uint": np.uint32,
          "ll": np.int64, "ull": np.uint64, "bool": np.bool_}

# objects the C side holds pointers to (names, arrays); released by op_exit
_keep = []


def _b(s):
    b = s.encode() if isinstance(s, str) else s
    _keep.append(b)
    return b


def lib():
    return _lib.load()


def op_init(argv=(), diags=0):
    """op_init(argc, argv, diags) (common/op_lib.cu:128-143)."""
    arr = (C.c_char_p * (len(argv) + 1))(*([_b("op2b")] + [_b(a) for a in argv]))
    _keep.append(arr)
    lib().op_init(len(argv) + 1, arr, diags)


def op_exit():
    lib().op_exit()
    del _keep[:]


def op_decl_set(size, name):
    s = lib().op_decl_set(int(size), _b(name))
    return s if s else None


def op_decl_map(from_set, to_set, dim, imap, name):
    imap = np.ascontiguousarray(imap, dtype=np.int32)
    _keep.append(imap)
    m = lib().op_decl_map(from_set, to_set, int(dim), imap.ctypes.data, _b(name))
    return m if m else None


def op_decl_dat(set_, dim, type_, data, name):
    """op_decl_dat<T> (common/op_lib.h:160-167): type-checked, then
    op_decl_dat_char (device copy).  `data` must be a C-contiguous numpy
    array of the declared type; it is borrowed, not copied."""
    want = _TYPES.get(type_)
    if want is None or not isinstance(data, np.ndarray) or data.dtype != want:
        print('incorrect type specified for dataset "%s" ' % name)
        raise TypeError("incorrect type specified for dataset \"%s\"" % name)
    if not data.flags["C_CONTIGUOUS"]:
        raise ValueError("dataset arrays must be C-contiguous")
    _keep.append(data)
    d = lib().op_decl_dat_char(set_, int(dim), _b(type_), data.itemsize, data.ctypes.data, _b(name))
    return d if d else None


def op_decl_const(name, dim, type_, values):
    """op_decl_const2<T>(name, dim, type, data) (common/op_lib.h:169-175)."""
    arr = np.ascontiguousarray(np.atleast_1d(values), dtype=_TYPES[type_])
    if arr.size < dim:
        raise ValueError("constant %s needs %d values" % (name, dim))
    lib().op_decl_const_char(int(dim), _b(type_), arr.itemsize, arr.ctypes.data, _b(name))


def op_arg_dat(dat, idx, map_, dim, type_, acc):
    return lib().op_arg_dat(dat, int(idx), map_, int(dim), _b(type_), int(acc))


def op_arg_gbl(data, dim, type_, acc):
    """op_arg_gbl<T> (common/op_lib.h:184-190).  `data` is a numpy array of
    the given type; reductions write their result into it."""
    want = _TYPES.get(type_)
    ok = isinstance(data, np.ndarray) and data.dtype == want and data.flags["C_CONTIGUOUS"]
    _keep.append(data)
    return lib().op_arg_gbl_core(data.ctypes.data, int(dim), _b(type_ if ok else "error"), int(acc))


def op_par_loop(name, set_, *args):
    """Generic op_par_loop: dispatches by name and argument signature to the
    device loops (op2b_par_loop)."""
    arr = (op_arg * len(args))(*args)
    lib().op2b_par_loop(_b(name), set_, len(args), arr)


def op_fetch_data(dat):
    """Copy the device data back into the array given to op_decl_dat and
    return that array (common/op_lib.cu:116-121)."""
    lib().op_fetch_data(dat)
    d = dat.contents
    n = d.set.contents.size
    t = _TYPES[d.type.decode()]
    buf = (C.c_char * (n * d.size)).from_address(d.data)
    return np.frombuffer(buf, dtype=t).reshape(n, d.dim)


def op_diagnostic_output():
    lib().op_diagnostic_output()


def op_timing_output():
    lib().op_timing_output()


def _plan_args(args, inds):
    a = (op_arg * len(args))(*args)
    i = (C.c_int * len(inds))(*inds)
    ninds = (max(inds) + 1) if len(inds) and max(inds) >= 0 else 0
    return a, i, ninds


def op_plan_core(name, set_, part_size, args, inds):
    """The plan of a loop with every array in host memory (op_lib_core.c:627)."""
    a, i, ninds = _plan_args(args, inds)
    return lib().op_plan_core(_b(name), set_, int(part_size), len(args), a, ninds, i)


def op_plan_validate(name, set_, part_size, args, inds):
    """Number of plan / colouring violations found on the device (0 = valid)."""
    a, i, ninds = _plan_args(args, inds)
    return lib().op2b_plan_validate(_b(name), set_, int(part_size), len(args), a, ninds, i)


def plan_arrays(p, args, inds):
    """numpy copies of an op_plan_core plan's arrays."""
    P = p.contents
    ninds = P.ninds
    n = P.set.contents.size

    def arr(ptr, k, dt=np.int32):
        return np.ctypeslib.as_array(ptr, shape=(k,)).astype(dt).copy() if k else np.zeros(0, dt)

    out = {
        "nblocks": P.nblocks, "ncolors": P.ncolors, "nshared": P.nshared,
        "transfer": P.transfer, "transfer2": P.transfer2,
        "nthrcol": arr(P.nthrcol, P.nblocks), "thrcol": arr(P.thrcol, n),
        "offset": arr(P.offset, P.nblocks), "nelems": arr(P.nelems, P.nblocks),
        "blkmap": arr(P.blkmap, P.nblocks), "ncolblk": arr(P.ncolblk, P.ncolors),
        "ind_offs": arr(P.ind_offs, P.nblocks * ninds),
        "ind_sizes": arr(P.ind_sizes, P.nblocks * ninds),
        "nindirect": arr(P.nindirect, ninds),
    }
    for m in range(ninds):
        out["ind_maps%d" % m] = arr(P.ind_maps[m], out["nindirect"][m])
    for a in range(len(args)):
        if inds[a] >= 0:
            out["loc_maps%d" % a] = arr(P.loc_maps[a], n, np.int16)
    return out


# ---- extensions (include/op2b.h) ----

def set_strategy(s):
    return lib().op2b_set_strategy(int(s))


def set_reduction(m):
    return lib().op2b_set_reduction(int(m))


def set_error_mode(m):
    return lib().op2b_set_error_mode(int(m))


def last_error():
    return lib().op2b_last_error().decode()


def clear_error():
    lib().op2b_clear_error()


def set_gbl_deferred(on):
    return lib().op2b_set_gbl_deferred(1 if on else 0)


def sync():
    return lib().op2b_sync()


def get_stream():
    return lib().op2b_get_stream()


def set_stream(ptr):
    lib().op2b_set_stream(ptr)


def loop_time(name):
    c = C.c_int(0)
    t = lib().op2b_loop_time(_b(name), C.byref(c))
    return t, c.value


def set_timing(on):
    return lib().op2b_set_timing(1 if on else 0)


def global_int(name):
    return _lib.global_int(name).value
