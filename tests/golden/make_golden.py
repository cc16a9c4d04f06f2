"""Generate the golden fixtures of tests/golden/ by running the REFERENCE.

    python tests/golden/make_golden.py            # small cases (about a minute)
    python tests/golden/make_golden.py --large    # adds the 720k / 2.9M / NN=512 runs

The reference ships no golden vectors (its test/ directory is stale and does
not build), so the fixtures are outputs of the reference's own sequential
build, compiled from its sources by oracle/Makefile into oracle/_ref/:
  - airfoil_seq_f32 / _f64  : rms history (printed %.17e, exact) and SHA-256
                              of the final q, qold, res, adt
  - jac1_seq / jac2_seq     : u max / rms per iteration, final u
  - plan_dump               : the reference op_plan_core's arrays (SHA-256)
Inputs are the project's mesh generators (oplus2_matlab_b200.mesh), whose
arrays are hashed into every fixture so a test knows it runs the same mesh.
Needs the reference tree (to build oracle/_ref) and libop2b200.so (meshes).
"""
import argparse
import hashlib
import json
import os
import re
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oplus2_matlab_b200 import mesh as M  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
SCRATCH = os.path.join(HERE, "_scratch", "make_golden_%d" % os.getpid())


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def mesh_hash(m):
    h = hashlib.sha256()
    for a in (m.cell, m.edge, m.ecell, m.bedge, m.becell, m.bound, m.x64, m.x32):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def run(binary, cwd, env):
    e = dict(os.environ)
    e.update({k: str(v) for k, v in env.items()})
    r = subprocess.run([os.path.join(REF, binary)], cwd=cwd, env=e, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("%s failed: %s" % (binary, r.stdout[-2000:] + r.stderr[-2000:]))
    return r.stdout


def airfoil_case(name, I, J, scramble, dtype, niter, every):
    m = M.naca0012(I, J, scramble=scramble)
    d = os.path.join(SCRATCH, name)
    shutil.rmtree(d, ignore_errors=True)
    os.makedirs(os.path.join(d, "dump"))
    M.write_grid(m, os.path.join(d, "new_grid.dat"))
    binary = "airfoil_seq_f32" if dtype == "f32" else "airfoil_seq_f64"
    out = run(binary, d, {"OP2REF_NITER": niter, "OP2REF_PRINT": every,
                          "OP2REF_DUMP": os.path.join(d, "dump")})
    hist = [(int(a), float(b)) for a, b in re.findall(r"^\s+(\d+)\s+([-+0-9.eE]+)\s*$", out, re.M)]
    t = np.float32 if dtype == "f32" else np.float64
    fields = {}
    for f in ("p_q", "p_qold", "p_res", "p_adt"):
        a = np.fromfile(os.path.join(d, "dump", f + ".bin"), dtype=t)
        fields[f] = {"sha256": sha(a), "first": a[:8].tolist(), "sum": float(a.astype(np.float64).sum())}
    shutil.rmtree(d, ignore_errors=True)
    return {"case": name, "I": I, "J": J, "scramble": scramble, "seed": M.SEED, "dtype": dtype,
            "niter": niter, "print_every": every, "mesh_sha256": mesh_hash(m),
            "ncell": m.ncell, "nedge": m.nedge, "nnode": m.nnode, "nbedge": m.nbedge,
            "rms": hist, "final": fields}


def jac_case(name, variant, NN, niter):
    d = os.path.join(SCRATCH, name)
    shutil.rmtree(d, ignore_errors=True)
    os.makedirs(os.path.join(d, "dump"))
    out = run("jac%d_seq" % variant, d, {"OP2REF_NN": NN, "OP2REF_NITER": niter,
                                         "OP2REF_DUMP": os.path.join(d, "dump")})
    hist = [(float(a), float(b)) for a, b in
            re.findall(r"u max/rms = ([-+0-9.eE]+) ([-+0-9.eE]+)", out)]
    u = np.fromfile(os.path.join(d, "dump", "p_u.bin"), dtype=np.float32)
    jm = M.jac(NN, variant)
    shutil.rmtree(d, ignore_errors=True)
    rec = {"case": name, "variant": variant, "NN": NN, "niter": niter,
           "mesh_sha256": sha(np.concatenate([jm.pp.ravel().view(np.uint8), jm.A.ravel().view(np.uint8),
                                              jm.r.ravel().view(np.uint8)])),
           "u_max_rms": hist, "u_sha256": sha(u)}
    if u.size <= 64:
        rec["u"] = u.tolist()
    return rec


# loop signatures of airfoil/airfoil_op.cpp and jac1/jac_op.cpp for the
# reference plan builder: (map, idx, dim, bytes per item, acc, ind, dat id)
def plan_specs_airfoil(m, real=4):
    maps = {"pedge": ("edges", "nodes", 2, m.edge), "pecell": ("edges", "cells", 2, m.ecell),
            "pbedge": ("bedges", "nodes", 2, m.bedge), "pbecell": ("bedges", "cells", 1, m.becell),
            "pcell": ("cells", "nodes", 4, m.cell)}
    sets = {"nodes": m.nnode, "edges": m.nedge, "bedges": m.nbedge, "cells": m.ncell}
    R, I_, INC = 0, None, 3
    loops = {
        "res_calc": ("edges", [("pedge", 0, 2, real, R, 0, 0), ("pedge", 1, 2, real, R, 0, 0),
                               ("pecell", 0, 4, real, R, 1, 1), ("pecell", 1, 4, real, R, 1, 1),
                               ("pecell", 0, 1, real, R, 2, 2), ("pecell", 1, 1, real, R, 2, 2),
                               ("pecell", 0, 4, real, INC, 3, 3), ("pecell", 1, 4, real, INC, 3, 3)]),
        "adt_calc": ("cells", [("pcell", 0, 2, real, R, 0, 0), ("pcell", 1, 2, real, R, 0, 0),
                               ("pcell", 2, 2, real, R, 0, 0), ("pcell", 3, 2, real, R, 0, 0),
                               (I_, -1, 4, real, R, -1, 1), (I_, -1, 1, real, 1, -1, 2)]),
        "bres_calc": ("bedges", [("pbedge", 0, 2, real, R, 0, 0), ("pbedge", 1, 2, real, R, 0, 0),
                                 ("pbecell", 0, 4, real, R, 1, 1), ("pbecell", 0, 1, real, R, 2, 2),
                                 ("pbecell", 0, 4, real, INC, 3, 3), (I_, -1, 1, 4, R, -1, 4)]),
    }
    return sets, maps, loops


def plan_case(name, loop, sets, maps, loops, part_size, tag):
    d = os.path.join(SCRATCH, "plan_" + tag + "_" + loop)
    shutil.rmtree(d, ignore_errors=True)
    os.makedirs(os.path.join(d, "out"))
    set_names = list(sets)
    map_names = list(maps)
    lset, args = loops[loop]
    lines = ["%s %d %d %d %d %d %d" % (loop, set_names.index(lset), part_size, len(args),
                                       max(a[5] for a in args) + 1, len(sets), len(maps))]
    lines += [str(sets[s]) for s in set_names]
    for mn in map_names:
        f, t, dim, arr = maps[mn]
        p = os.path.join(d, mn + ".i32")
        np.ascontiguousarray(arr, dtype=np.int32).tofile(p)
        lines.append("%d %d %d %s" % (set_names.index(f), set_names.index(t), dim, p))
    for (mn, idx, dim, nbytes, acc, ind, dat) in args:
        lines.append("%d %d %d %d %d %d %d" % (map_names.index(mn) if mn else -1, idx, dim, nbytes,
                                               acc, ind, dat))
    spec = os.path.join(d, "spec.txt")
    open(spec, "w").write("\n".join(lines) + "\n")
    r = subprocess.run([os.path.join(REF, "plan_dump"), spec, os.path.join(d, "out")],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("plan_dump failed: " + r.stdout + r.stderr)
    meta = dict(l.split() for l in open(os.path.join(d, "out", "meta.txt")))
    rec = {"case": name, "loop": loop, "part_size": part_size,
           "nblocks": int(meta["nblocks"]), "ncolors": int(meta["ncolors"]),
           "nshared": int(meta["nshared"]), "transfer": float(meta["transfer"]),
           "transfer2": float(meta["transfer2"]), "arrays": {}}
    for f in sorted(os.listdir(os.path.join(d, "out"))):
        if f.endswith((".i32", ".i16")):
            a = np.fromfile(os.path.join(d, "out", f), dtype=np.int32 if f.endswith("i32") else np.int16)
            rec["arrays"][f[:-4]] = {"sha256": sha(a), "n": int(a.size)}
    shutil.rmtree(d, ignore_errors=True)
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--large", action="store_true")
    ap.add_argument("--only", default="")
    ap.add_argument("--skip-plans", action="store_true")
    ap.add_argument("--large-plans", action="store_true",
                    help="plans_large.json: the reference op_plan_core at 720k (part sizes 0, 64, "
                         "256) and on the 2.88M scrambled mesh (part sizes 0, 256)")
    ap.add_argument("--ref", default=os.environ.get("OP2B_REFERENCE", "/root/reference"),
                    help="the reference tree, from whose sources oracle/_ref is built")
    a = ap.parse_args()
    subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile"), "REF=" + a.ref,
                    "ref"], check=True)
    os.makedirs(SCRATCH, exist_ok=True)
    out = {}
    small = {
        "airfoil_40x60_f32": lambda: airfoil_case("airfoil_40x60_f32", 40, 60, False, "f32", 1000, 1),
        "airfoil_40x60_f64": lambda: airfoil_case("airfoil_40x60_f64", 40, 60, False, "f64", 1000, 1),
        "airfoil_40x60s_f32": lambda: airfoil_case("airfoil_40x60s_f32", 40, 60, True, "f32", 200, 1),
        "jac1_nn6": lambda: jac_case("jac1_nn6", 1, 6, 2),
        "jac2_nn6": lambda: jac_case("jac2_nn6", 2, 6, 2),
        "jac1_nn64": lambda: jac_case("jac1_nn64", 1, 64, 20),
        "jac2_nn64": lambda: jac_case("jac2_nn64", 2, 64, 20),
    }
    large = {
        "airfoil_400x600_f32": lambda: airfoil_case("airfoil_400x600_f32", 400, 600, False, "f32", 1000, 10),
        "airfoil_400x600_f64": lambda: airfoil_case("airfoil_400x600_f64", 400, 600, False, "f64", 1000, 10),
        "airfoil_800x1200s_f32": lambda: airfoil_case("airfoil_800x1200s_f32", 800, 1200, True, "f32", 500, 10),
        "jac1_nn512": lambda: jac_case("jac1_nn512", 1, 512, 100),
    }
    todo = dict(small)
    if a.large:
        todo.update(large)
    for k, f in todo.items():
        if a.only and a.only not in k:
            continue
        print("running", k, flush=True)
        out[k] = f()
        json.dump(out[k], open(os.path.join(HERE, k + ".json"), "w"), indent=1)
    # plans
    if not a.skip_plans and (not a.only or "plan" in a.only):
        plans = []
        for tag, (I, J, scr) in {"40x60": (40, 60, False), "40x60s": (40, 60, True)}.items():
            m = M.naca0012(I, J, scramble=scr)
            sets, maps, loops = plan_specs_airfoil(m)
            for loop in ("res_calc", "adt_calc", "bres_calc"):
                for ps in ((0, 64, 256) if not scr else (0,)):
                    plans.append(dict(plan_case("%s_%s_p%d" % (tag, loop, ps), loop, sets, maps, loops, ps, tag),
                                      mesh=tag, mesh_sha256=mesh_hash(m)))
        for NN in (64,):
            jm = M.jac(NN, 1)
            sets = {"nodes": jm.nnode, "edges": jm.nedge}
            maps = {"ppedge": ("edges", "nodes", 2, jm.pp)}
            loops = {"res": ("edges", [(None, -1, 1, 4, 0, -1, 0), ("ppedge", 1, 1, 4, 0, 0, 1),
                                       ("ppedge", 0, 1, 4, 3, 1, 2)])}
            for ps in (0, 512):
                plans.append(dict(plan_case("jac1_nn%d_res_p%d" % (NN, ps), "res", sets, maps, loops, ps, "jac"),
                                  mesh="jac1_nn%d" % NN))
        json.dump(plans, open(os.path.join(HERE, "plans.json"), "w"), indent=1)
    if a.large_plans:
        plans = []
        for tag, (I, J, scr, parts) in {"400x600": (400, 600, False, (0, 64, 256)),
                                        "800x1200s": (800, 1200, True, (0, 256))}.items():
            m = M.naca0012(I, J, scramble=scr)
            sets, maps, loops = plan_specs_airfoil(m)
            for loop in ("res_calc", "adt_calc", "bres_calc"):
                for ps in parts:
                    print("plan", tag, loop, ps, flush=True)
                    plans.append(dict(plan_case("%s_%s_p%d" % (tag, loop, ps), loop, sets, maps, loops,
                                                ps, tag), mesh=tag, mesh_sha256=mesh_hash(m)))
        json.dump(plans, open(os.path.join(HERE, "plans_large.json"), "w"), indent=1)
    shutil.rmtree(SCRATCH, ignore_errors=True)


if __name__ == "__main__":
    main()
