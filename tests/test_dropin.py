"""Drop-in: the reference's unchanged app mains linked against this library.

oracle/Makefile (target `dropin`) compiles, exactly as the reference ships
them, against include/ and libop2b200.so (no generated CUDA stubs):
  - the generated mains airfoil/airfoil_op.cpp, jac1/jac_op.cpp,
    jac2/jac_op.cpp (op_par_loop_<name> entry points), and
  - the un-generated mains airfoil/airfoil.cpp, jac1/jac.cpp, jac2/jac.cpp
    (the template op_par_loop of op_seq.h, here include/op_seq.h).  Here: every
OP2 symbol those binaries import must come from the library, and on the GPU
their printed results must match the reference's own sequential build
(the goldens made from it): airfoil's rms every 100 iterations (printed
"%10.5e", summed in tree order on the GPU), jac's u max/rms per iteration
and the final u field (printed "%7.4f").
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import load_golden, scratch_dir
from oplus2_matlab_b200 import _lib
from oplus2_matlab_b200 import mesh as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")
APPS = ["airfoil_op", "jac1_op", "jac2_op", "airfoil_seqapi", "jac1_seqapi", "jac2_seqapi"]


def binary(name):
    path = os.path.join(DROPIN, name)
    if not os.path.exists(path):
        pytest.skip("drop-in binaries not built (make -f oracle/Makefile dropin)")
    return path


def dynsyms(path, flag):
    out = subprocess.run(["nm", "-D", flag, path], capture_output=True, text=True,
                         check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if l.strip()}


@pytest.mark.parametrize("app", APPS)
def test_dropin_imports_every_op2_symbol_from_the_library(app):
    path = binary(app)
    need = {s for s in dynsyms(path, "--undefined-only") if s.startswith(("op_", "OP_"))}
    assert "op_init" in need
    assert "op_par_loop_update" in need or "op2b_par_loop" in dynsyms(path, "--undefined-only")
    need |= {s for s in dynsyms(path, "--undefined-only") if s.startswith("op2b_")}
    have = dynsyms(_lib.LIB_PATH, "--defined-only")
    assert need <= have, sorted(need - have)
    ldd = subprocess.run(["ldd", path], capture_output=True, text=True).stdout
    assert "libop2b200.so" in ldd and "not found" not in ldd.split("libop2b200.so")[1].split("\n")[0]


def run(path, cwd):
    r = subprocess.run([path], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("app", ["airfoil_op", "airfoil_seqapi"])
def test_dropin_airfoil_matches_reference_rms(app):
    path = binary(app)
    gold = load_golden("airfoil_40x60_f32")
    d = scratch_dir()
    M.write_grid(M.naca0012(40, 60), os.path.join(d, "new_grid.dat"))
    out = run(path, d)
    rows = [(int(a), float(b)) for a, b in re.findall(r"^\s*(\d+)\s+([0-9.]+e[-+]\d+)\s*$", out,
                                                     flags=re.M)]
    assert [it for it, _ in rows] == list(range(100, 1001, 100))
    ref = np.array([r for _, r in gold["rms"]])
    for it, v in rows:
        # 6 printed digits; tree-order float sum (<= 5e-5 relative at 7.2k cells)
        assert v == pytest.approx(ref[it - 1], rel=1e-4), it


@pytest.mark.gpu
@pytest.mark.parametrize("app,case", [("jac1_op", "jac1_nn6"), ("jac2_op", "jac2_nn6"),
                                      ("jac1_seqapi", "jac1_nn6"), ("jac2_seqapi", "jac2_nn6")])
def test_dropin_jac_matches_reference(app, case):
    path = binary(app)
    gold = load_golden(case)
    out = run(path, scratch_dir())
    got = [(float(a), float(b)) for a, b in re.findall(r"u max/rms = (\S+) (\S+)", out)]
    assert len(got) == gold["niter"]
    for (umax, urms), (gmax, grms) in zip(got, gold["u_max_rms"]):
        assert umax == pytest.approx(gmax, abs=1.5e-6)
        assert urms == pytest.approx(grms, abs=1.5e-6)
    NN = gold["NN"]
    field = out.split("Results after")[1].split("\n")
    lines = [l for l in field if re.match(r"^\s*-?\d+\.\d{4}", l)][:NN - 1]
    # jac2 keeps u[2] per node and prints component 0 (jac2/jac_op.cpp:222)
    u = np.array(gold["u"], np.float32).reshape(NN - 1, NN - 1, -1)[:, :, 0]
    want = ["".join(" %7.4f" % u[j - 1, i - 1] for i in range(1, NN)) for j in range(NN - 1, 0, -1)]
    assert [l.rstrip() for l in lines] == [w.rstrip() for w in want]
