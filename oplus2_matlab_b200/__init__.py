"""oplus2_matlab_b200 -- B200-native OP2 op_par_loop execution path.

The product is libop2b200.so (csrc/, built by `python -m
oplus2_matlab_b200.build`): the reference's OP2 C API (include/op_lib.h) with
device data management, a device-built execution plan and hand-written
sm_100a loop kernels.  This package holds its ctypes bindings (api), the mesh
generators (mesh) and the reference apps' mains restated over the API (apps).
"""
from . import _lib  # noqa: F401
from ._lib import load  # noqa: F401

__all__ = ["api", "apps", "mesh", "load"]
