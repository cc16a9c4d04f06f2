"""The C ABI of libop2b200.so: every entry point the public headers declare is
exported with C linkage, and the struct layouts are the reference's
(common/op_lib_core.h:75-158).  CPU only: nothing here launches a kernel."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import scratch_dir

from oplus2_matlab_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
HEADERS = ["op_lib_core.h", "op_lib.h", "op2b.h", "op2b_mesh.h", "op2b_group.h"]


def declared_functions(header):
    text = open(os.path.join(INCLUDE, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    # templates (C++ only, header-defined) are not exported
    text = re.sub(r"template\s*<[^>]*>\s*[^{;]*\{.*?\n\}", "", text, flags=re.S)
    text = re.sub(r"inline[^;{]*\{[^}]*\}", "", text)
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(op\w+)\s*\(", text, flags=re.M):
        names.add(m.group(1))
    return sorted(names)


def exported_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


@pytest.mark.parametrize("header", HEADERS)
def test_every_declared_function_is_exported_unmangled(header):
    syms = exported_symbols()
    names = declared_functions(header)
    assert names, header
    missing = [n for n in names if n not in syms]
    assert not missing, "declared in %s but not exported with C linkage: %s" % (header, missing)


def test_library_loads_and_binds_all_prototypes():
    lib = _lib.load()
    for name, _, _ in _lib.PROTOTYPES:
        assert getattr(lib, name) is not None
    for g in _lib.GLOBALS:
        _lib.global_int(g)
    assert b"sm_100a" in lib.op2b_version()


def test_struct_layouts_match_reference():
    # LP64 layout of the reference structs (common/op_lib_core.h:75-158),
    # as gcc lays them out from the reference header
    assert C.sizeof(_lib.op_set_core) == 16
    assert C.sizeof(_lib.op_map_core) == 48 and _lib.op_map_core.map.offset == 32
    assert C.sizeof(_lib.op_dat_core) == 56 and _lib.op_dat_core.data_d.offset == 32
    assert C.sizeof(_lib.op_arg) == 72
    assert [_lib.op_arg.dat.offset, _lib.op_arg.map.offset, _lib.op_arg.dim.offset,
            _lib.op_arg.data.offset, _lib.op_arg.type.offset, _lib.op_arg.acc.offset,
            _lib.op_arg.argtype.offset] == [8, 16, 24, 40, 56, 64, 68]
    assert C.sizeof(_lib.op_plan) == 184 and _lib.op_plan.count.offset == 180
    assert C.sizeof(_lib.op_kernel) == 24


def test_header_layout_compiles_identically():
    """Compile a probe against include/op_lib_core.h and compare sizeof /
    offsetof with the ctypes mirror used by the tests."""
    src = r"""
#include <stddef.h>
#include <stdio.h>
#include "op_lib_core.h"
int main(void){ printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(op_set_core), sizeof(op_map_core),
  sizeof(op_dat_core), sizeof(op_arg), sizeof(op_plan), sizeof(op_kernel), offsetof(op_plan, count));
  return 0; }
"""
    d = scratch_dir()
    c, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
    open(c, "w").write(src)
    subprocess.run(["gcc", "-I", INCLUDE, c, "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert [int(v) for v in out] == [16, 48, 56, 72, 184, 24, 180]
    os.remove(c)
    os.remove(exe)


def test_app_declarations_inherit_c_linkage():
    """An app that includes op_lib.h and then declares a loop itself (as
    airfoil/airfoil_op.cpp:64-99 does) must reference the unmangled symbol."""
    src = r"""
#include "op_lib.h"
void op_par_loop_save_soln(char const *, op_set, op_arg, op_arg);
int main(){ op_par_loop_save_soln("save_soln", 0, op_arg(), op_arg()); return 0; }
"""
    d = scratch_dir()
    cpp, obj = os.path.join(d, "app.cpp"), os.path.join(d, "app.o")
    open(cpp, "w").write(src)
    subprocess.run(["g++", "-c", "-I", INCLUDE, cpp, "-o", obj], check=True)
    und = subprocess.run(["nm", "-u", obj], capture_output=True, text=True, check=True).stdout
    assert "op_par_loop_save_soln" in und.split()
    os.remove(cpp)
    os.remove(obj)
