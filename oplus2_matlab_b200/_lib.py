"""ctypes view of libop2b200.so: the C types of include/op_lib_core.h and the
prototypes of include/op_lib.h, include/op2b.h and include/op2b_mesh.h.

The library must have been built (python -m oplus2_matlab_b200.build); there
is no fallback implementation, so a missing library is an ImportError.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libop2b200.so")

# op_access / op_arg_type (op_lib_core.h:67-69)
OP_READ, OP_WRITE, OP_RW, OP_INC, OP_MIN, OP_MAX = range(6)
OP_ARG_GBL, OP_ARG_DAT = range(2)
# op2b.h
STRATEGY_AUTO, STRATEGY_GATHER, STRATEGY_COLOURED = 0, 1, 2
REDUCE_TREE, REDUCE_SEQ = 0, 1
ERRORS_EXIT, ERRORS_RETURN = 0, 1


class op_set_core(C.Structure):
    _fields_ = [("index", C.c_int), ("size", C.c_int), ("name", C.c_char_p)]


op_set = C.POINTER(op_set_core)


class op_map_core(C.Structure):
    _fields_ = [("index", C.c_int), ("from_", op_set), ("to", op_set), ("dim", C.c_int),
                ("map", C.POINTER(C.c_int)), ("name", C.c_char_p)]


op_map = C.POINTER(op_map_core)


class op_dat_core(C.Structure):
    _fields_ = [("index", C.c_int), ("set", op_set), ("dim", C.c_int), ("size", C.c_int),
                ("data", C.c_void_p), ("data_d", C.c_void_p), ("type", C.c_char_p),
                ("name", C.c_char_p)]


op_dat = C.POINTER(op_dat_core)


class op_arg(C.Structure):
    _fields_ = [("index", C.c_int), ("dat", op_dat), ("map", op_map), ("dim", C.c_int),
                ("idx", C.c_int), ("size", C.c_int), ("data", C.c_void_p),
                ("data_d", C.c_void_p), ("type", C.c_char_p), ("acc", C.c_int),
                ("argtype", C.c_int)]


class op_plan(C.Structure):
    _fields_ = [("name", C.c_char_p), ("set", op_set), ("nargs", C.c_int), ("ninds", C.c_int),
                ("part_size", C.c_int), ("maps", C.POINTER(op_map)), ("dats", C.POINTER(op_dat)),
                ("idxs", C.POINTER(C.c_int)), ("accs", C.POINTER(C.c_int)),
                ("nthrcol", C.POINTER(C.c_int)), ("thrcol", C.POINTER(C.c_int)),
                ("offset", C.POINTER(C.c_int)), ("ind_maps", C.POINTER(C.POINTER(C.c_int))),
                ("ind_offs", C.POINTER(C.c_int)), ("ind_sizes", C.POINTER(C.c_int)),
                ("nindirect", C.POINTER(C.c_int)),
                ("loc_maps", C.POINTER(C.POINTER(C.c_short))), ("nblocks", C.c_int),
                ("nelems", C.POINTER(C.c_int)), ("ncolors", C.c_int),
                ("ncolblk", C.POINTER(C.c_int)), ("blkmap", C.POINTER(C.c_int)),
                ("nshared", C.c_int), ("transfer", C.c_float), ("transfer2", C.c_float),
                ("count", C.c_int)]


class op_kernel(C.Structure):
    _fields_ = [("name", C.c_char_p), ("count", C.c_int), ("time", C.c_float),
                ("transfer", C.c_float), ("transfer2", C.c_float)]


class op2b_mesh(C.Structure):
    _fields_ = [("nnode", C.c_int), ("ncell", C.c_int), ("nedge", C.c_int), ("nbedge", C.c_int)] + \
               [(n, C.POINTER(C.c_int)) for n in ("cell", "edge", "ecell", "bedge", "becell", "bound")] + \
               [("x64", C.POINTER(C.c_double)), ("x32", C.POINTER(C.c_float))]


_P = C.c_void_p

_PMESH = C.POINTER(op2b_mesh)
# include/op2b_serve.h: the group table the server drives, and its records
ADD_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_longlong, _PMESH, C.c_double, C.c_double, C.c_int,
                     C.c_double)
RUN_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int)
POLL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_int), C.c_int)
HISTORY_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_int)
FETCHQ_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p)
REMOVE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int)
SOLVE_BYTES_FN = C.CFUNCTYPE(C.c_longlong, C.c_void_p, C.c_longlong, _PMESH, C.c_int)
DEVICE_BYTES_FN = C.CFUNCTYPE(C.c_longlong, C.c_void_p)
NOW_FN = C.CFUNCTYPE(C.c_double, C.c_void_p)


class op2b_group_ops(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("add", ADD_FN), ("run", RUN_FN), ("poll", POLL_FN),
                ("history", HISTORY_FN), ("fetch_q", FETCHQ_FN), ("remove", REMOVE_FN),
                ("solve_bytes", SOLVE_BYTES_FN), ("device_bytes", DEVICE_BYTES_FN),
                ("now", NOW_FN)]


class op2b_served(C.Structure):
    _fields_ = [("rid", C.c_longlong), ("sid", C.c_int), ("iterations", C.c_int),
                ("arrival", C.c_double), ("admitted", C.c_double), ("finished", C.c_double)]

# (name, restype, argtypes) of every exported entry point
PROTOTYPES = [
    # op_lib_core.h
    ("op_init_core", None, [C.c_int, C.POINTER(C.c_char_p), C.c_int]),
    ("op_decl_set", op_set, [C.c_int, C.c_char_p]),
    ("op_decl_map", op_map, [op_set, op_set, C.c_int, _P, C.c_char_p]),
    ("op_decl_dat_core", op_dat, [op_set, C.c_int, C.c_char_p, C.c_int, _P, C.c_char_p]),
    ("op_arg_check", None, [op_set, C.c_int, op_arg, C.POINTER(C.c_int), C.c_char_p]),
    ("op_arg_dat", op_arg, [op_dat, C.c_int, op_map, C.c_int, C.c_char_p, C.c_int]),
    ("op_arg_gbl_core", op_arg, [_P, C.c_int, C.c_char_p, C.c_int]),
    ("op_diagnostic_output", None, []),
    ("op_timing_output", None, []),
    ("op_plan_core", C.POINTER(op_plan),
     [C.c_char_p, op_set, C.c_int, C.c_int, C.POINTER(op_arg), C.c_int, C.POINTER(C.c_int)]),
    ("op_timers", None, [C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("op_timing_realloc", None, [C.c_int]),
    ("op_exit_core", None, []),
    # op_lib.h
    ("op_init", None, [C.c_int, C.POINTER(C.c_char_p), C.c_int]),
    ("op_decl_dat_char", op_dat, [op_set, C.c_int, C.c_char_p, C.c_int, _P, C.c_char_p]),
    ("op_decl_const_char", None, [C.c_int, C.c_char_p, C.c_int, _P, C.c_char_p]),
    ("op_fetch_data", None, [op_dat]),
    ("op_plan_get", C.POINTER(op_plan),
     [C.c_char_p, op_set, C.c_int, C.c_int, C.POINTER(op_arg), C.c_int, C.POINTER(C.c_int)]),
    ("op_exit", None, []),
    ("op_par_loop_save_soln", None, [C.c_char_p, op_set] + [op_arg] * 2),
    ("op_par_loop_adt_calc", None, [C.c_char_p, op_set] + [op_arg] * 6),
    ("op_par_loop_res_calc", None, [C.c_char_p, op_set] + [op_arg] * 8),
    ("op_par_loop_bres_calc", None, [C.c_char_p, op_set] + [op_arg] * 6),
    ("op_par_loop_update", None, [C.c_char_p, op_set] + [op_arg] * 5),
    ("op_par_loop_res", None, [C.c_char_p, op_set] + [op_arg] * 4),
    ("op2b_par_loop", None, [C.c_char_p, op_set, C.c_int, C.POINTER(op_arg)]),
    # op2b.h
    ("op2b_set_strategy", C.c_int, [C.c_int]),
    ("op2b_set_reduction", C.c_int, [C.c_int]),
    ("op2b_set_error_mode", C.c_int, [C.c_int]),
    ("op2b_last_error", C.c_char_p, []),
    ("op2b_clear_error", None, []),
    ("op2b_get_stream", _P, []),
    ("op2b_set_stream", None, [_P]),
    ("op2b_sync", C.c_int, []),
    ("op2b_set_gbl_deferred", C.c_int, [C.c_int]),
    ("op2b_loop_time", C.c_double, [C.c_char_p, C.POINTER(C.c_int)]),
    ("op2b_set_timing", C.c_int, [C.c_int]),
    ("op2b_plan_validate", C.c_long,
     [C.c_char_p, op_set, C.c_int, C.c_int, C.POINTER(op_arg), C.c_int, C.POINTER(C.c_int)]),
    ("op2b_version", C.c_char_p, []),
    ("op2b_l2_flush", C.c_int, []),
    ("op2b_wait_timeouts", C.c_uint, [C.c_int]),
    ("op2b_tiled_launches", C.c_ulonglong, [C.c_int]),
    ("op2b_res_skips", C.c_ulonglong, [C.c_int]),
    ("op2b_h2d_bytes", C.c_ulonglong, [C.c_int]),
    ("op2b_layout_ab", C.c_int, [C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P, C.c_float,
                                 C.c_float, C.c_int, C.POINTER(C.c_double),
                                 C.POINTER(C.c_double)]),
    ("op2b_set_tuning", C.c_int, [C.c_char_p, C.c_int]),
    ("op2b_get_tuning", C.c_int, [C.c_char_p, C.c_int]),
    ("op2b_autotune", C.c_int, [C.c_char_p, C.c_int, C.c_int]),
    ("op2b_update_noalloc", C.c_int, [C.c_int, _P, _P, _P, _P, _P, _P]),
    ("op2b_set_renumber", C.c_int, [C.c_int]),
    ("op2b_checkpoint_file", C.c_int, [C.c_char_p]),
    ("op_checkpoint", C.c_int, []),
    ("op2b_renumber_order", C.c_int, [op_set, C.POINTER(C.c_int)]),
    ("op2b_set_renumber_coords", C.c_int, [op_dat]),
    # op2b_serve.h
    ("op2b_group_ops_fill", C.c_int, [_P, C.POINTER(op2b_group_ops)]),
    ("op2b_server_create", _P, [C.POINTER(op2b_group_ops), C.c_longlong, C.c_int, C.c_int,
                                C.c_int, C.c_int, C.c_int]),
    ("op2b_server_destroy", None, [_P]),
    ("op2b_server_submit", C.c_int, [_P, C.c_longlong, _PMESH, C.c_double, C.c_double, C.c_int,
                                     C.c_double, C.c_double]),
    ("op2b_server_step", C.c_int, [_P]),
    ("op2b_server_done", C.c_int, [_P, C.POINTER(op2b_served), C.c_int]),
    ("op2b_server_history", C.c_int, [_P, C.c_longlong, C.POINTER(C.c_double), C.c_int]),
    ("op2b_server_q", C.c_int, [_P, C.c_longlong, _P]),
    ("op2b_server_release", None, [_P, C.c_longlong]),
    ("op2b_server_active", C.c_int, [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_int), C.c_int]),
    ("op2b_server_queued", C.c_int, [_P]),
    ("op2b_server_peak_active", C.c_int, [_P]),
    ("op2b_server_idle", C.c_int, [_P]),
    ("op2b_server_now", C.c_double, [_P]),
    ("op2b_server_latency", C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("op2b_renumber_seconds", C.c_double, []),
    ("op2b_decl_const_named", None, [C.c_int, C.c_char_p, C.c_int, _P, C.c_char_p]),
    ("op2b_capture_begin", C.c_int, [C.c_int]),
    ("op2b_capture_end", _P, []),
    ("op2b_graph_launch", C.c_int, [_P]),
    ("op2b_graph_nloops", C.c_int, [_P]),
    ("op2b_graph_nkernels", C.c_int, [_P]),
    ("op2b_graph_loop_name", C.c_char_p, [_P, C.c_int]),
    ("op2b_graph_loop_times", C.c_int, [_P, C.POINTER(C.c_double), C.c_int]),
    ("op2b_graph_destroy", None, [_P]),
    # op2b_mesh.h
    ("op2b_mesh_naca0012", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(op2b_mesh)]),
    ("op2b_mesh_free", None, [C.POINTER(op2b_mesh)]),
    ("op2b_mesh_write", C.c_int, [C.POINTER(op2b_mesh), C.c_char_p]),
    ("op2b_mesh_read", C.c_int, [C.c_char_p, C.POINTER(op2b_mesh)]),
    ("op2b_mesh_write_bin", C.c_int, [C.POINTER(op2b_mesh), C.c_char_p]),
    ("op2b_mesh_read_bin", C.c_int, [C.c_char_p, C.POINTER(op2b_mesh)]),
    ("op2b_mesh_read_cached", C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(op2b_mesh)]),
    ("op2b_jac_sizes", C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("op2b_mesh_jac1", C.c_int, [C.c_int, _P, _P, _P]),
    ("op2b_mesh_jac2", C.c_int, [C.c_int, _P, _P, _P]),
    ("op2b_splitmix64", C.c_uint64, [C.POINTER(C.c_uint64)]),
    # op2b_group.h
    ("op2b_flow_qinf", C.c_int, [C.c_double, C.c_double, C.c_int, _P, _P]),
    ("op2b_group_create", _P, [C.c_int]),
    ("op2b_group_destroy", None, [_P]),
    ("op2b_group_add", C.c_int, [_P, C.POINTER(op2b_mesh), C.c_double, C.c_double, C.c_int,
                                 C.c_double]),
    ("op2b_group_run", C.c_int, [_P, C.c_int]),
    ("op2b_group_poll", C.c_int, [_P, C.POINTER(C.c_int), C.c_int]),
    ("op2b_group_sync", C.c_int, [_P]),
    ("op2b_group_iterations", C.c_int, [_P, C.c_int]),
    ("op2b_group_history", C.c_int, [_P, C.c_int, C.POINTER(C.c_double), C.c_int]),
    ("op2b_group_fetch_q", C.c_int, [_P, C.c_int, _P]),
    ("op2b_group_fetch_q_async", C.c_int, [_P, C.c_int, _P]),
    ("op2b_group_remove", C.c_int, [_P, C.c_int]),
    ("op2b_group_solve_bytes", C.c_longlong, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("op2b_group_device_bytes", C.c_longlong, [_P]),
    ("op2b_group_active", C.c_int, [_P]),
    ("op2b_group_set_edge_tile", C.c_int, [_P, C.c_int]),
    ("op2b_group_set_block_bytes", C.c_int, [_P, C.c_longlong]),
    ("op2b_group_set_streams", C.c_int, [_P, C.c_int]),
    ("op2b_group_set_tiled", C.c_int, [_P, C.c_int]),
    ("op2b_group_tiled", C.c_int, [_P]),
    ("op2b_group_edge_tile", C.c_int, [_P]),
    ("op2b_group_autotune", C.c_int, [_P, C.c_int]),
    ("op2b_group_autotune_run", C.c_int, [_P, C.c_int]),
]

# data symbols of op_lib.h
GLOBALS = ["OP_diags", "OP_part_size", "OP_block_size", "OP_set_index", "OP_map_index",
           "OP_dat_index", "OP_plan_index", "OP_kern_max"]

_lib = None


def load():
    """Load libop2b200.so once and attach the prototypes.  Raises ImportError
    when the library has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libop2b200.so is not built (%s); run "
                          "`python -m oplus2_matlab_b200.build`" % LIB_PATH)
    lib = C.CDLL(LIB_PATH, mode=C.RTLD_GLOBAL)
    for name, res, args in PROTOTYPES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def global_int(name):
    return C.c_int.in_dll(load(), name)
