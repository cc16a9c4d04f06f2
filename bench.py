#!/usr/bin/env python
"""Benchmark: airfoil 720k-cell outer iterations per second on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the reference's airfoil app at the 720k-cell mesh, I=400, J=600,
FP32): one step = one outer iteration = save_soln + 2 x (adt_calc, res_calc,
bres_calc, update with the rms reduction).  Synthetic input: the NACA0012
C-mesh of airfoil/naca0012.m restated in csrc/meshgen.cpp, flow at free
stream (Mach 0.4) -- the reference ships no mesh, so this is its generator.

value   device throughput: W untimed warm-up iterations build the plans, then
        one iteration is captured as a CUDA graph (op2b_capture_*) and K
        launches are timed with CUDA events on the library stream.  The
        captured iteration is the app's, rotated by two loop calls: res_calc,
        bres_calc, update, adt_calc, res_calc, bres_calc, update, then the
        next iteration's save_soln and adt_calc (run once before the first
        launch), so those two fuse with the update before them; every launch
        is still one whole outer iteration's loops.  L2 is
        flushed before every step by an untimed read-only sweep of 3x its
        size (op2b_l2_flush; a memset would leave dirty lines whose
        write-back the next step would pay).
e2e     a complete solve through the C API (libop2b200_apps.so ->
        op_decl_* from host arrays, 1000 iterations with the rms returned to
        the host after every update, op_fetch_data of q), wall-clock timed.
roofline  the launches that run the step's first res_calc (fused with the
        bres_calc, update and adt_calc after it: a flux pass and a per-cell
        pass): their compulsory bytes (every map entry and dataset element
        the fused loops touch once, twice when read and written) over their
        average device time, timed on a graph of those loop calls alone (L2
        flushed before each launch, CUDA events); the per-kernel split comes
        from event pairs in a profiled copy of the step's graph.
cpu_baseline / --impl reference  the reference's own OpenMP build
        (oracle/_ref/airfoil_op_f32, compiled from its sources) on this
        host's cores, timed by its own op_timing_output.  The reference arm
        writes its input with the host-only oracle/_build/gen_grid, so its
        process loads nothing of this repository's GPU library.
batched / served_200_per_s / served_20_per_s  (plain mode, one GPU) the
        batched workload (64 seeded instances x 500 iterations, grouped
        against the same solves back to back through the plain C API) and
        two served streams (200 requests/s shortened to --forms-requests,
        stop at 1e-6 x the first rms or 2000 iterations; and 20 requests/s
        with a 5% stopping test), each with p50/p99 latency, the plain-path
        comparison and a clock record of its own timed region.
With N > 1 (torchrun), every rank runs an independent replica (the path
does not shard: "replicas only") and value = N*K iterations / max rank time.
"""
import argparse
import ctypes as C
import dataclasses
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "720k-cell airfoil iters/s"
UNIT = "iters/s"
I_MESH, J_MESH = 400, 600
MESH_SEED = 20261203  # the seed of the scrambled and randomised configurations
REF_MIN_ITERS = 400   # the reference arm times at least this many iterations


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--strategy", default="gather", choices=["gather", "coloured"])
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-iters", type=int, default=1000)
    ap.add_argument("--admit-chunk", type=int, default=8,
                    help="batched: solves admitted per chunk (uploads overlap the iterations "
                         "of the solves admitted before)")
    ap.add_argument("--admit-ms", type=float, default=10.0,
                    help="batched: device milliseconds of iterations enqueued after each "
                         "admitted chunk (sized from the admitted cells)")
    ap.add_argument("--no-plain", action="store_true",
                    help="batched: skip the plain back-to-back leg (no speed-up, no parity; "
                         "for profiling the group alone)")
    ap.add_argument("--group-tiled", action="store_true",
                    help="batched and served forms: the tiled chain (op2b_group_set_tiled)")
    ap.add_argument("--no-forms", action="store_true",
                    help="plain mode: skip the batched and served measurements that the "
                         "default line carries")
    ap.add_argument("--forms-requests", type=int, default=400,
                    help="plain mode: requests of the served stream at the batched/served "
                         "workload's 200/s rate (the full workload has 10,000)")
    ap.add_argument("--op-arg", action="append", default=[],
                    help="plain mode: an op_init argument, e.g. OP_BLOCK_SIZE=256 or "
                         "OP_PART_SIZE=256 (the reference's run-time launch-shape options; "
                         "COLOURED reads them)")
    ap.add_argument("--tune", action="append", default=[],
                    help="kernel-variant knob key=value (op2b_set_tuning)")
    ap.add_argument("--mesh", default="400x600",
                    help="plain mode: IxJ of the NACA0012 C-mesh (3IJ cells); a trailing 's' "
                         "renumbers cells, nodes, edges and bedges from the seed (scrambled)")
    ap.add_argument("--renumber", nargs="?", const="cm", default=None, choices=["cm", "rcb"],
                    help="plain mode: renumber the sets for locality (op2b_set_renumber): "
                         "cm = Cuthill-McKee (the default), rcb = recursive coordinate "
                         "bisection of the node coordinates (op2b_set_renumber_coords)")
    ap.add_argument("--nn", type=int, default=512, help="jac mode: NN (grid of (NN-1)^2 nodes)")
    ap.add_argument("--jac-variant", type=int, default=1, choices=[1, 2],
                    help="jac mode: jac1 (float, one component) or jac2 (A double[3], u[2])")
    ap.add_argument("--mode", default="plain",
                    choices=["plain", "batched", "served", "jac", "layout"],
                    help="plain: the 720k single-mesh iteration (default); batched: many "
                         "instances per launch; served: a Poisson request stream")
    ap.add_argument("--instances", type=int, default=64, help="batched: instances")
    ap.add_argument("--iters", type=int, default=500, help="batched: iterations per instance")
    ap.add_argument("--requests", type=int, default=10000, help="served: requests")
    ap.add_argument("--rate", type=float, default=200.0, help="served: mean arrivals per second")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="served: HBM budget")
    ap.add_argument("--max-iter", type=int, default=2000, help="served: iteration cap")
    ap.add_argument("--rel-tol", type=float, default=1e-6, help="served: rms tolerance")
    ap.add_argument("--iters-per-step", type=int, default=10,
                    help="served: iterations between completion checks")
    ap.add_argument("--max-active", type=int, default=0,
                    help="served: cap on solves iterated together (0: memory budget only)")
    ap.add_argument("--policy", default="fifo", choices=["fifo", "shortest"],
                    help="served: admission order")
    ap.add_argument("--plain-sample", type=int, default=32,
                    help="served: requests re-solved with the plain path for its rate")
    return ap.parse_args()


# ------------------------------------------------------------- plumbing ----

class Dist:
    """One process per GPU under torchrun; torch.distributed only for the
    barrier and the max over ranks.  OP2B_DIST_BACKEND=gloo runs the same
    plumbing on host tensors (the CPU tests use it)."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = os.environ.get("OP2B_DIST_BACKEND", "nccl")
        self.dist = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            if self.backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=120))
            self.torch, self.dist = torch, dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, v):
        if not self.dist:
            return v
        t = self.torch.tensor([float(v)], device="cuda" if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()


def cudart():
    for name in ("libcudart.so.12", "libcudart.so"):
        try:
            lib = C.CDLL(name)
            break
        except OSError:
            continue
    lib.cudaEventElapsedTime.argtypes = [C.POINTER(C.c_float), C.c_void_p, C.c_void_p]
    lib.cudaEventRecord.argtypes = [C.c_void_p, C.c_void_p]
    lib.cudaMemsetAsync.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_void_p]
    lib.cudaStreamSynchronize.argtypes = [C.c_void_p]
    lib.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    lib.cudaFree.argtypes = [C.c_void_p]
    lib.cudaEventCreate.argtypes = [C.POINTER(C.c_void_p)]
    lib.cudaMallocHost.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    lib.cudaFreeHost.argtypes = [C.c_void_p]
    return lib


class Clocks:
    """nvidia-smi sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False,
                                               dir=ROOT if os.access(ROOT, os.W_OK) else None)
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        self.index = vis.split(",")[device] if vis and vis.split(",")[device].isdigit() else str(device)
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.index, "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.out.flush()
        rows = [l.split(", ") for l in open(self.out.name).read().strip().splitlines() if l.strip()]
        os.unlink(self.out.name)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], None, set()
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].strip() == "Active":
                        reasons.add(nm)
            except (IndexError, ValueError):
                continue
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        v = json.load(open(p))["hbm_gbs"]
        return float(v), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic():
    """dram bytes per res_calc launch from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "res_calc_airfoil_720k.md")
    try:
        m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


def res_calc_bytes(m, s=4):
    """Algorithmic bytes of one res_calc call: pedge + pecell (16 B / edge),
    x of every node, q and adt of every cell read once, res read and written."""
    return 16.0 * m.nedge + 2 * s * m.nnode + 4 * s * m.ncell + s * m.ncell + 8 * s * m.ncell


def bres_calc_bytes(m, s=4):
    """bres_calc: pbedge, pbecell, bound (16 B / bedge) and, per boundary
    edge, x of its nodes, q and adt of its cell and res read and written."""
    return 16.0 * m.nbedge + (2 * s + 4 * s + s + 8 * s) * m.nbedge


def chain_bytes(m, name, s=4):
    """Compulsory bytes of a fused chain of loops named "res_calc+bres_calc
    +update+adt_calc" (or a prefix of it): every map entry and every dataset
    element the chain touches once, twice when it is both read and written.
    res_calc: pedge, pecell, x, q, adt, res (RMW); bres_calc adds pbedge,
    pbecell, bound; update adds qold and q's write; adt_calc adds pcell and
    adt's write."""
    loops = name.split("+")
    b = res_calc_bytes(m, s)
    if "bres_calc" in loops:
        b += 16.0 * m.nbedge
    if "update" in loops:
        b += 8 * s * m.ncell
    if "adt_calc" in loops:
        b += 16.0 * m.ncell + s * m.ncell
    return b


def chain_loop_bytes(m, name, s=4):
    """The chain's loops' compulsory bytes each counted as if the loop ran
    alone (the per-loop definition: bytes moved per loop), summed."""
    loops = name.split("+")
    per = {"res_calc": res_calc_bytes(m, s),
           "bres_calc": 16 * m.nbedge + (2 * s + 4 * s + s + 8 * s) * m.nbedge,
           "update": 17 * s * m.ncell,
           "adt_calc": 16 * m.ncell + 2 * s * m.nnode + 4 * s * m.ncell + s * m.ncell,
           "save_soln": 8 * s * m.ncell}
    return float(sum(per[l] for l in loops if l in per))


def iteration_bytes(m, s=4):
    save = 8 * s * m.ncell
    adt = 16 * m.ncell + 2 * s * m.nnode + 4 * s * m.ncell + s * m.ncell
    res = res_calc_bytes(m, s)
    bres = 16 * m.nbedge + (2 * s + 4 * s + s + 8 * s) * m.nbedge
    update = 17 * s * m.ncell
    return save + 2 * (adt + res + bres + update)


# ------------------------------------------------------------ reference ----

def make_grid(I, J, path, scramble=False):
    """Write the reference apps' input (new_grid.dat) with the host-only
    generator program oracle/_build/gen_grid (the restated naca0012.m), in a
    child process, so the process timing the reference never loads this
    repository's CUDA library.  Returns the set sizes (nnode, ncell, nedge,
    nbedge) or None."""
    gen = os.path.join(ROOT, "oracle", "_build", "gen_grid")
    if not os.path.exists(gen):
        return None
    cmd = [gen, str(I), str(J)] + (["1", str(MESH_SEED)] if scramble else []) + [path]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        return None
    nnode, ncell, nedge, nbedge = (int(v) for v in r.stdout.split())
    return {"nnode": nnode, "ncell": ncell, "nedge": nedge, "nbedge": nbedge}


def run_reference_openmp(I, J, niter, fp64=False, threads=None):
    """The reference's OpenMP airfoil (oracle/_ref/airfoil_op_f32) on this
    host, on the I x J mesh; returns (iters/s from its own op_timing_output,
    seconds, cores, set sizes) or None."""
    binary = os.path.join(ROOT, "oracle", "_ref", "airfoil_op_f64" if fp64 else "airfoil_op_f32")
    if not os.path.exists(binary):
        return None
    d = tempfile.mkdtemp(prefix="op2b_reference_")
    try:
        sizes = make_grid(I, J, os.path.join(d, "new_grid.dat"))
        if sizes is None:
            return None
        cores = threads or os.cpu_count()
        env = dict(os.environ, OMP_NUM_THREADS=str(cores), OMP_PROC_BIND="close",
                   OP2REF_NITER=str(niter), OP2REF_PRINT=str(max(niter, 1)))
        r = subprocess.run([binary], cwd=d, env=env, capture_output=True, text=True, timeout=1800)
        if r.returncode != 0:
            return None
        tot = 0.0
        for line in r.stdout.splitlines():
            f = line.split()
            if len(f) >= 4 and f[0].isdigit() and f[-1] in ("save_soln", "adt_calc", "res_calc",
                                                          "bres_calc", "update"):
                tot += float(f[1])
        return (niter / tot if tot > 0 else None), tot, cores, sizes
    finally:
        shutil.rmtree(d, ignore_errors=True)


def impl_reference(args, dist):
    """--impl reference: rank 0 times the reference's OpenMP airfoil on the
    same 720k mesh (written by the host-only generator; nothing of this
    repository's GPU library is loaded); other ranks exit without work."""
    if dist.rank != 0:
        return
    niter = max(REF_MIN_ITERS, args.steps + args.warmup)
    res = run_reference_openmp(I_MESH, J_MESH, niter, fp64=args.fp64)
    base = {"impl": "reference", "metric": METRIC, "unit": UNIT, "higher_is_better": True,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup}
    if res is None or res[0] is None:
        print(json.dumps(dict(base, unavailable="reference OpenMP build oracle/_ref/airfoil_op_f32 "
                                                "or the grid writer oracle/_build/gen_grid missing or failed")))
        return
    v, secs, cores, sizes = res
    line = dict(base, value=v, ms_per_step=1e3 / v, scaling="weak", vs_baseline=None,
                dtype="f64" if args.fp64 else "f32", data="synthetic",
                config=plain_config(I_MESH, J_MESH, sizes, False),
                reference={"build": "reference airfoil_op (OpenMP), compiled from its sources by "
                                    "oracle/Makefile", "iterations": niter, "seconds": secs,
                           "timing": "sum of the per-loop times of its own op_timing_output"},
                cpu_baseline={"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                              "sample": "%d iterations of the 720k mesh, sum of op_timing_output" % niter},
                e2e={"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    print(json.dumps(line))


# ------------------------------------------------------------------ ours ----

def plain_mesh(args):
    from oplus2_matlab_b200 import mesh as M
    spec = args.mesh.lower()
    scramble = spec.endswith("s")
    I, J = (int(v) for v in spec.rstrip("s").split("x"))
    return M.naca0012(I, J, scramble=scramble)


def plain_config(I, J, sizes, scrambled):
    """The workload keys both arms report for the plain single-mesh solve
    (the reference arm's config holds exactly these)."""
    return {"workload": "airfoil NACA0012 C-mesh I=%d, J=%d%s: %d cells, %d edges, %d nodes, "
                        "%d bedges; one outer iteration (save_soln + 2 x (adt_calc, res_calc, "
                        "bres_calc, update)) per step"
                        % (I, J, ", scrambled numbering" if scrambled else "", sizes["ncell"],
                           sizes["nedge"], sizes["nnode"], sizes["nbedge"]),
            "cells": sizes["ncell"], "edges": sizes["nedge"]}


def mesh_sizes(mesh):
    return {"nnode": mesh.nnode, "ncell": mesh.ncell, "nedge": mesh.nedge, "nbedge": mesh.nbedge}


def impl_ours(args, dist):
    from oplus2_matlab_b200 import api, apps
    from oplus2_matlab_b200 import mesh as M
    lib = api.lib()
    cr = cudart()
    dt = np.float64 if args.fp64 else np.float32
    s = 8 if args.fp64 else 4

    mesh = plain_mesh(args)
    api.set_error_mode(api.ERRORS_RETURN)
    api.op_init(args.op_arg, 0)
    api.set_strategy(api.STRATEGY_GATHER if args.strategy == "gather" else api.STRATEGY_COLOURED)
    api.set_reduction(api.REDUCE_TREE)
    if args.renumber:
        lib.op2b_set_renumber(1)
    for kv in args.tune:
        k, v = kv.split("=")
        lib.op2b_set_tuning(k.encode(), int(v))
    A = apps.Airfoil(mesh, dt)
    if args.renumber == "rcb":
        assert lib.op2b_set_renumber_coords(A.p_x) == 0, api.last_error()
    stream = lib.op2b_get_stream()

    # warm-up: builds the plans, uploads the maps
    for _ in range(max(3, args.warmup)):
        A.iteration()
    api.sync()
    assert api.last_error() == "", api.last_error()
    renumber_s = lib.op2b_renumber_seconds() if args.renumber else None

    # one outer iteration as a CUDA graph: a plain one for the timed steps,
    # and one with event nodes around every loop for the per-loop times.
    # Rotated: the iteration's first save_soln + adt_calc run once here, and
    # each graph ends with the next iteration's, fused with the last update
    A.loop("save_soln")
    A.loop("adt_calc")
    api.sync()
    rotated = ("res_calc", "bres_calc", "update", "adt_calc", "res_calc", "bres_calc", "update",
               "save_soln", "adt_calc")

    def capture(profile):
        assert lib.op2b_capture_begin(profile) == 1, api.last_error()
        for nm in rotated:
            if nm == "update":
                A.rms[0] = 0
            A.loop(nm)
        h = lib.op2b_capture_end()
        assert h, api.last_error()
        return h
    g = capture(0)
    gp = capture(1)
    nkern = lib.op2b_graph_nkernels(g)
    nloops = lib.op2b_graph_nloops(gp)
    names = [lib.op2b_graph_loop_name(gp, i).decode() for i in range(nloops)]

    assert lib.op2b_l2_flush() == 0  # allocates the sweep buffer before timing
    ev = []
    for _ in range(2 * args.steps):
        e = C.c_void_p()
        cr.cudaEventCreate(C.byref(e))
        ev.append(e)

    def timed_steps(graph, nsteps, per_loop=None):
        """nsteps graph launches, L2 flushed (untimed) before each; returns
        the device time of every step in ms."""
        lt = (C.c_double * max(1, nloops))()
        for k in range(nsteps):
            lib.op2b_l2_flush()
            cr.cudaEventRecord(ev[2 * k], stream)
            rc = lib.op2b_graph_launch(graph)
            cr.cudaEventRecord(ev[2 * k + 1], stream)
            assert rc == 0, rc
            if per_loop is not None:
                got = lib.op2b_graph_loop_times(graph, lt, nloops)
                for i in range(got):
                    per_loop.setdefault(names[i], []).append(lt[i])
        cr.cudaStreamSynchronize(stream)
        out = []
        for k in range(nsteps):
            ms = C.c_float()
            cr.cudaEventElapsedTime(C.byref(ms), ev[2 * k], ev[2 * k + 1])
            out.append(ms.value)
        return out

    clocks = Clocks(dist.local)
    dist.barrier()
    cr.cudaStreamSynchronize(stream)
    step_ms = timed_steps(g, args.steps)           # the timed region
    dist.barrier()
    clk = clocks.stop()
    total_s = dist.max(sum(step_ms) * 1e-3)
    value = dist.world * args.steps / total_s
    # per-loop device times from the instrumented graph (same flush, fewer steps)
    loops = {}
    prof_ms = timed_steps(gp, min(args.steps, 50), loops)
    loop_tot = {n: sum(v) for n, v in loops.items()}
    loop_cnt = {n: len(v) for n, v in loops.items()}
    api.sync()  # delivers the last launch's rms
    rms_last = float(np.sqrt(A.rms[0] / dt(mesh.ncell)))

    # res_calc runs fused with the loops that follow it (bres_calc, update,
    # adt_calc: one flux pass, one per-cell pass) unless fusion is off; the
    # roofline is taken over the launches that carry the first res_calc of
    # the step, against the compulsory bytes of the loops they run
    chains = [n for n in names if n.split("+")[0] == "res_calc" and ":" not in n]
    res_key = chains[0]
    profiled_launch_s = loop_tot[res_key] / max(1, loop_cnt[res_key])
    # the chain's own launch time: a graph holding only its loop calls
    # (res_calc, bres_calc, update[, adt_calc] -- the same fused launches as in
    # the step), L2 flushed before each launch, timed like the steps; the
    # profiled graph's event nodes between kernels would block their overlap
    chain_loops = res_key.split("+")

    def capture_fn(fn):
        assert lib.op2b_capture_begin(0) == 1, api.last_error()
        fn()
        h = lib.op2b_capture_end()
        assert h, api.last_error()
        return h

    def chains(n):
        for rep in range(n):
            if rep:
                assert lib.op2b_l2_flush() == 0
            for nm in chain_loops:
                if nm == "update":
                    A.rms[0] = 0
                A.loop(nm)
    nchain = min(args.steps, 50)
    lib.op2b_tiled_launches(1)
    gc = capture_fn(lambda: chains(1))
    chain_method = "graph of the chain's loop calls alone, L2 flushed before each launch"
    if lib.op2b_tiled_launches(1) == 0:
        lib.op2b_graph_launch(gc)
        chain_ms = timed_steps(gc, nchain)
        lib.op2b_graph_destroy(gc)
    else:
        # the tiled chain writes q and adt into second buffers and swaps
        # them: a graph of one chain ends with a copy back, one of two does
        # not.  Two chains with an L2 sweep between them, less a graph of the
        # sweep alone (both launched after an untimed sweep)
        lib.op2b_graph_destroy(gc)
        gc = capture_fn(lambda: chains(2))
        gf = capture_fn(lambda: lib.op2b_l2_flush())
        lib.op2b_graph_launch(gc)
        pair_ms = timed_steps(gc, nchain)
        sweep_ms = timed_steps(gf, nchain)
        lib.op2b_graph_destroy(gc)
        lib.op2b_graph_destroy(gf)
        chain_ms = [(a - float(np.mean(sweep_ms))) / 2 for a in pair_ms]
        chain_method = ("graph of two chains with an L2 sweep between them, less a graph of "
                        "the sweep alone, halved; L2 flushed before each launch")
    res_launch_s = float(np.mean(chain_ms)) * 1e-3
    algo = chain_bytes(mesh, res_key, s)
    peak, peak_kind = measured_peak()
    achieved = algo / res_launch_s / 1e9
    phases = {n.split(":")[1]: 1e6 * loop_tot[n] / max(1, loop_cnt[n])
              for n in names if n.startswith(res_key + ":")}
    per_loop_us = {n: 1e6 * loop_tot[n] / max(1, loop_cnt[n]) for n in names}
    iter_bytes = iteration_bytes(mesh, s)

    lib.op2b_graph_destroy(g)
    lib.op2b_graph_destroy(gp)
    st = A.fetch()
    ok = bool(np.isfinite(st["q"]).all()) and np.isfinite(rms_last) and rms_last > 0
    api.op_exit()

    # end to end: a whole solve through the C API from host arrays
    e2e = None
    if not args.no_e2e:
        # three complete solves; the median is reported (the host is shared)
        runs = [run_e2e(mesh, args.fp64, args.e2e_iters, args.strategy, dist, args.renumber)
                for _ in range(3)]
        runs = [r for r in runs if r]
        if runs:
            runs.sort(key=lambda r: r["value"])
            e2e = dict(runs[len(runs) // 2], all_values=[r["value"] for r in runs])

    cpu = None
    if not args.no_cpu_baseline and dist.rank == 0 and dist.world == 1:
        cpu = cpu_baseline(mesh, args.fp64)

    # the batched and served forms on the same GPU, each with its own clock
    # record: 64 instances x 500 iterations (the batched workload itself);
    # the served workload's stream (200 requests/s, stop at 1e-6 x the
    # first rms or 2000 iterations) shortened to --forms-requests requests;
    # and a stream at a rate the GPU sustains (20/s) whose looser stopping
    # test (5% of the first rms) retires small meshes before the cap
    forms = None
    if not args.no_forms and dist.world == 1 and not args.fp64 and args.mesh == "400x600":
        forms = {"batched": measure_batched(args, dist, 64, 500),
                 "served_200_per_s": measure_served(args, dist, args.forms_requests, 200.0,
                                                    2000, 1e-6),
                 "served_20_per_s": measure_served(args, dist, 200, 20.0, 2000, 0.05)}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.fp64 else "f32",
        "data": "synthetic: NACA0012 C-mesh from the reference's generator, free-stream start",
        "config": dict(plain_config(mesh.I, mesh.J, mesh_sizes(mesh), args.mesh.endswith("s")),
                       strategy=args.strategy, op_init_args=args.op_arg,
                       renumbered=args.renumber or False,
                       renumber_seconds=renumber_s, reduction="tree",
                       l2="flushed before every step (untimed read-only sweep of 3x the 126 MB L2)",
                       timing="CUDA events around each graph launch on the library stream",
                       parallelism="replicas" if dist.world > 1 else "single GPU"),
        "roofline": {"bound": "hbm", "kernel": res_key, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": ncu_traffic(),
                     "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": algo, "avg_launch_us": res_launch_s * 1e6,
                     "timing": "%s, CUDA events, mean of %d launches" % (chain_method, nchain),
                     "profiled_graph_us": profiled_launch_s * 1e6,
                     "kernels_us": phases,
                     # the per-loop definition (each loop's compulsory bytes as
                     # if it ran alone, summed over the chain's loops) over
                     # the same launch time
                     "per_loop_bytes_per_launch": chain_loop_bytes(mesh, res_key, s),
                     "frac_per_loop_bytes": chain_loop_bytes(mesh, res_key, s) / res_launch_s
                                            / 1e9 / peak},
        "iteration_roofline": {"algorithmic_bytes": iter_bytes,
                               "achieved_gbs": iter_bytes * value / dist.world / 1e9,
                               "frac": iter_bytes * value / dist.world / 1e9 / peak},
        "per_loop_us": per_loop_us,
        "instrumented_ms_per_step": float(np.mean(prof_ms)),
        "gpu_launches": nkern * args.steps,
        "kernels_per_step": nkern,
        "rms_last": rms_last, "finite": ok,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    if forms:
        b = forms["batched"]
        line["batched"] = {"metric": b["metric"], "value": b["value"], "unit": b["unit"],
                           "plain_back_to_back_solves_per_s":
                               b["plain_back_to_back"]["solves_per_s"],
                           "speedup_vs_plain": b["speedup_vs_plain"],
                           "parity": b["parity_rank0"], "config": b["config"],
                           "group": b["group"], "gpu_launches": b["gpu_launches"],
                           "clocks": b["clocks"]}
        for key in ("served_200_per_s", "served_20_per_s"):
            v = forms[key]
            line[key] = {"metric": v["metric"], "value": v["value"], "unit": v["unit"],
                         "latency": v["latency"], "config": v["config"],
                         "plain_serial_solves_per_s": v["plain_serial"]["solves_per_s"],
                         "speedup_vs_plain": v["speedup_vs_plain"],
                         "retired_by_rms_tolerance": v["retired_by_rms_tolerance"],
                         "retired_by_iteration_cap": v["retired_by_iteration_cap"],
                         "iterations": v["iterations"],
                         "max_active_solves": v["max_active_solves_rank0"],
                         "plain_serial": v["plain_serial"], "clocks": v["clocks"]}
    if dist.rank == 0:
        print(json.dumps(line))


class AppTiming(C.Structure):
    _fields_ = [("t_declare", C.c_double), ("t_iterate", C.c_double), ("t_fetch", C.c_double),
                ("t_total", C.c_double), ("h2d_bytes", C.c_longlong), ("d2h_bytes", C.c_longlong)]


def run_e2e(mesh, fp64, niter, strategy, dist, renumber=None):
    """A complete solve through the C API (oplus2_matlab_b200/apps/airfoil_app.cpp):
    declarations from pinned host arrays, niter iterations with the rms read
    back after every update, q fetched to the host.  Wall-clock timed."""
    from oplus2_matlab_b200 import _lib
    from oplus2_matlab_b200 import api
    cr = cudart()
    lib = _lib.load()
    app = C.CDLL(os.path.join(ROOT, "oplus2_matlab_b200", "lib", "libop2b200_apps.so"))
    app.op2b_airfoil_app_renumbered.argtypes = [C.POINTER(_lib.op2b_mesh), C.c_int, C.c_int,
                                                C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                C.POINTER(AppTiming)]
    dt = np.float64 if fp64 else np.float32
    # pinned host copies of every input
    keep = []

    def pinned(a):
        a = np.ascontiguousarray(a)
        p = C.c_void_p()
        assert cr.cudaMallocHost(C.byref(p), max(1, a.nbytes)) == 0
        buf = np.frombuffer((C.c_char * a.nbytes).from_address(p.value), dtype=a.dtype).reshape(a.shape)
        buf[...] = a
        keep.append(p)
        return buf

    m = _lib.op2b_mesh()
    arrs = {k: pinned(getattr(mesh, k)) for k in ("cell", "edge", "ecell", "bedge", "becell", "bound",
                                                  "x64", "x32")}
    m.nnode, m.ncell, m.nedge, m.nbedge = mesh.nnode, mesh.ncell, mesh.nedge, mesh.nbedge
    for k in ("cell", "edge", "ecell", "bedge", "becell", "bound"):
        setattr(m, k, arrs[k].ctypes.data_as(C.POINTER(C.c_int)))
    m.x64 = arrs["x64"].ctypes.data_as(C.POINTER(C.c_double))
    m.x32 = arrs["x32"].ctypes.data_as(C.POINTER(C.c_float))
    from oplus2_matlab_b200.apps import airfoil_consts
    qinf = np.asarray(airfoil_consts(dt)["qinf"], dt)
    q = pinned(np.tile(qinf, (mesh.ncell, 1)))
    rms = np.zeros(niter, np.float64)
    t = AppTiming()
    api.set_error_mode(api.ERRORS_RETURN)
    dist.barrier()
    rc = app.op2b_airfoil_app_renumbered(C.byref(m), 1 if fp64 else 0, niter, q.ctypes.data,
                                         rms.ctypes.data, 1 if strategy == "gather" else 2,
                                         {None: 0, "cm": 1, "rcb": 2}[renumber], C.byref(t))
    total = dist.max(t.t_total)
    for p in keep:
        cr.cudaFreeHost(p)
    if rc != 0:
        return None
    return {"value": dist.world * niter / total, "unit": UNIT,
            "h2d_bytes_per_step": t.h2d_bytes / niter, "d2h_bytes_per_step": t.d2h_bytes / niter,
            "iterations": niter, "seconds": total,
            "phases_s": {"declare_h2d": t.t_declare, "iterate": t.t_iterate, "fetch_d2h": t.t_fetch},
            "rms_final": float(rms[-1]),
            "path": "C API (libop2b200_apps.so: op_decl_* from pinned host arrays, op_par_loop_* "
                    "with rms to the host every update, op_fetch_data)"}


def cpu_baseline(mesh, fp64):
    """The reference OpenMP build on a bounded sample (about 10-30 s)."""
    probe = run_reference_openmp(mesh.I, mesh.J, 3, fp64=fp64)
    if probe is None or probe[0] is None:
        return None
    rate = probe[0]
    niter = int(min(400, max(5, 15.0 * rate)))
    res = run_reference_openmp(mesh.I, mesh.J, niter, fp64=fp64)
    if res is None or res[0] is None:
        return None
    return {"value": res[0], "unit": UNIT, "cores": res[2], "kind": "reference",
            "sample": "%d iterations of the 720k mesh (reference airfoil_op, OpenMP, "
                      "sum of its op_timing_output)" % niter}


# ------------------------------------------------------ batched / served ----

MESH_ARRAYS = ("cell", "edge", "ecell", "bedge", "becell", "bound", "x64", "x32")


def pinned_mesh(mesh, keep):
    """A copy of `mesh` whose arrays live in pinned host memory: the inputs
    the timed region copies to the device come from pinned memory, as an
    application that stages its meshes for a GPU would hold them.  The copy
    is input preparation, untimed like the mesh generation; `keep` collects
    the allocations for free_pinned."""
    cr = cudart()

    def pin(a):
        a = np.ascontiguousarray(a)
        p = C.c_void_p()
        assert cr.cudaMallocHost(C.byref(p), max(1, a.nbytes)) == 0
        keep.append(p)
        buf = np.frombuffer((C.c_char * max(1, a.nbytes)).from_address(p.value), dtype=a.dtype,
                            count=a.size).reshape(a.shape)
        buf[...] = a
        return buf
    return dataclasses.replace(mesh, **{k: pin(getattr(mesh, k)) for k in MESH_ARRAYS})


def pinned_array(shape, dtype, keep):
    """A zeroed array in pinned host memory; `keep` collects the allocation."""
    cr = cudart()
    nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
    p = C.c_void_p()
    assert cr.cudaMallocHost(C.byref(p), max(1, nbytes)) == 0
    keep.append(p)
    a = np.frombuffer((C.c_char * max(1, nbytes)).from_address(p.value), dtype=dtype,
                      count=int(np.prod(shape))).reshape(shape)
    a[...] = 0
    return a


def free_pinned(keep):
    cr = cudart()
    for p in keep:
        cr.cudaFreeHost(p)
    keep.clear()


def gen_meshes(dims):
    """{(I, J): mesh} for every distinct (I, J) in dims, generated on a pool
    of host threads (the generator is C++ called through ctypes, which
    releases the GIL); input preparation, never timed."""
    import concurrent.futures
    from oplus2_matlab_b200 import mesh as M
    want = sorted(set(dims), key=lambda d: -d[0] * d[1])
    workers = max(1, min(32, (os.cpu_count() or 2) - 1))
    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as ex:
        return dict(zip(want, ex.map(lambda d: M.naca0012(d[0], d[1]), want)))


def warm_paths(dt, tiled=False):
    """Untimed: create the CUDA context and load the kernels of both paths
    (lazy module loading) on a tiny mesh, so neither timed region pays the
    process's one-time start-up."""
    from oplus2_matlab_b200 import group as G
    from oplus2_matlab_b200 import mesh as M
    tiny = M.naca0012(10, 15)
    g = G.Group(dt)
    if tiled:
        g.set_tiled(True)
    g.add(tiny, 0.5, 1.0, 3)
    g.autotune(1)
    g.run(3)
    g.sync()
    g.close()
    G.plain_solve(tiny, 0.5, 1.0, 3, dt)


def impl_batched(args, dist):
    """--mode batched: the batched workload's own JSON line."""
    line = measure_batched(args, dist, args.instances, args.iters)
    if dist.rank == 0:
        print(json.dumps(line))


def measure_batched(args, dist, instances, n):
    """`instances` seeded instances (20k-720k cells, Mach 0.3-0.7, alpha
    -2..6 deg), n iterations each: the group engine (every loop one launch
    over all instances, edge tile autotuned) against the same instances
    solved one after another through the plain C API.  Both timed end to
    end: host arrays in, rms histories and q out; mesh generation (the
    input) is not timed.  N ranks share the instances by greedy cell
    balance.  Returns the measurement as a JSON-able dict."""
    from oplus2_matlab_b200 import group as G
    from oplus2_matlab_b200 import mesh as M
    from oplus2_matlab_b200 import serve as S
    from oplus2_matlab_b200 import api
    dt = np.float64 if args.fp64 else np.float32
    inst = G.draw_instances(instances, cmin=20000, cmax=720000)
    cells = [3 * I * J for I, J, _, _ in inst]
    mine = S.shard_by_cells(cells, dist.world)[dist.rank]
    pins = []
    meshes = {k: pinned_mesh(v, pins) for k, v in gen_meshes([inst[i][:2] for i in mine]).items()}
    # results land in pinned host memory in both paths, as inputs come from it
    qbuf = {i: pinned_array((meshes[inst[i][:2]].ncell, 4), dt, pins) for i in mine}
    qbuf_plain = {i: pinned_array((meshes[inst[i][:2]].ncell, 4), dt, pins) for i in mine}
    api.set_error_mode(api.ERRORS_RETURN)
    for kv in args.tune:
        k, v = kv.split("=")
        api.lib().op2b_set_tuning(k.encode(), int(v))
    warm_paths(dt, args.group_tiled)

    clocks = Clocks(dist.local)
    dist.barrier()
    t0 = time.perf_counter()
    g = G.Group(dt)
    if args.group_tiled:
        g.set_tiled(True)
    # Admission in chunks: a chunk's uploads and list building (on the
    # group's admission stream) overlap the iterations already enqueued for
    # the solves admitted before it; a solve's results do not depend on when
    # it joined.  Then the launch shapes are tuned on real iterations, and
    # the group runs until every solve has stopped at its n iterations.
    ids, graph_launches, t_add, active_cells = [], 0, 0.0, 0
    chunk = max(1, args.admit_chunk)
    for c in range(0, len(mine), chunk):
        ta = time.perf_counter()
        ids += [g.add(meshes[inst[i][:2]], inst[i][2], inst[i][3], n) for i in mine[c:c + chunk]]
        t_add += time.perf_counter() - ta
        active_cells += sum(meshes[inst[i][:2]].ncell for i in mine[c:c + chunk])
        if c + chunk < len(mine):
            # about admit_ms of device work (an iteration moves about 12M
            # cells per ms) to cover the next chunk's admission
            k = int(min(n, max(8, args.admit_ms * 12e6 / max(1, active_cells))))
            g.run(k)
            graph_launches += k
    tt = time.perf_counter()
    graph_launches += g.autotune_run(3)
    t_tune = time.perf_counter() - tt
    tile = g.lib.op2b_group_edge_tile(g.h)
    ti = time.perf_counter()
    # each solve's q is copied out as soon as it has stopped, while the
    # others iterate
    stopped = 0
    q_of = dict(zip(ids, mine))
    while stopped < len(ids):
        g.run(50)
        graph_launches += 50
        done = g.poll()
        stopped += len(done)
        for sid in done:
            g.fetch_q_async(sid, qbuf[q_of[sid]])
    g.sync()
    t_iter = time.perf_counter() - ti
    tf = time.perf_counter()
    hist = [g.history(s) for s in ids]
    qg = [qbuf[i] for i in mine]
    t_fetch = time.perf_counter() - tf
    t_group = dist.max(time.perf_counter() - t0)
    gbytes = g.device_bytes()
    g.close()

    plain, t_plain = None, None
    if not args.no_plain:
        dist.barrier()
        t0 = time.perf_counter()
        plain = [G.plain_solve(meshes[inst[i][:2]], inst[i][2], inst[i][3], n, dt,
                               q_out=qbuf_plain[i]) for i in mine]
        t_plain = dist.max(time.perf_counter() - t0)
    clk = clocks.stop()

    exact = rel = None
    if plain:
        exact = sum(int(a.tobytes() == p[0].astype(dt).tobytes()) for a, p in zip(qg, plain))
        rel = max(float(np.max(np.abs(h - p[1]) / np.abs(p[1]))) for h, p in zip(hist, plain))
    s = 8 if args.fp64 else 4
    my_bytes = sum(iteration_bytes(meshes[inst[i][:2]], s) for i in mine) * n
    del meshes
    free_pinned(pins)
    total = len(inst)
    line = {
        "metric": "batched airfoil solves/s", "value": total / t_group, "unit": "solves/s",
        "n_gpus": dist.world, "steps": n, "warmup": 0, "ms_per_step": 1e3 * t_group / n,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64" if args.fp64 else "f32",
        "data": "synthetic: %d seeded NACA0012 C-meshes, cells log-uniform 20k-720k, "
                "Mach U[0.3,0.7], alpha U[-2,6] deg (splitmix64 seed %d)" % (total, M.SEED),
        "config": {"workload": "airfoil batched: %d instances x %d iterations, %d cells in all"
                               % (total, n, sum(cells)),
                   "instances": total, "iterations": n, "cells_total": sum(cells),
                   "timing": "wall clock, host arrays in (pinned) to rms histories and q "
                             "out, mesh generation excluded",
                   "parallelism": "instances sharded by cells over %d GPU(s)" % dist.world},
        "group": {"seconds": t_group, "iterate_seconds_rank0": t_iter,
                  "phases_s_rank0": {"admit_host": t_add, "autotune": t_tune,
                                     "iterate": t_iter, "fetch": t_fetch},
                  "phases_note": "admission overlaps iterations (chunks of %d solves, about "
                                 "%g ms of iterations enqueued after each); the autotuner's "
                                 "11 trials of 3 iterations are real iterations"
                                 % (chunk, args.admit_ms),
                  "edge_tile_autotuned": tile, "tiled_chain": bool(args.group_tiled),
                  "device_bytes_rank0": gbytes,
                  "autotuned": "edge tile and L2 block size, on real iterations",
                  "iteration_gbs_rank0": my_bytes / (t_group - t_fetch) / 1e9},
        "plain_back_to_back": None if plain is None else {
            "seconds": t_plain, "solves_per_s": total / t_plain,
            "path": "op2b_airfoil_app_flow per instance (op_par_loop, rms to the host after "
                    "every update)"},
        "speedup_vs_plain": None if plain is None else t_plain / t_group,
        "parity_rank0": None if plain is None else {
            "q_bit_identical": "%d/%d" % (exact, len(mine)), "max_rms_rel_diff": rel},
        # graph launches (iterations: 4 kernels each, 2 with the tiled chain;
        # more when the tuned blocks split the solves), priming save_soln +
        # adt_calc launches, list building at admission (6 per solve)
        "gpu_launches": (2 if args.group_tiled else 4) * graph_launches + 1 + 6 * len(mine),
        "clocks": clk,
    }
    return line


def impl_served(args, dist):
    """--mode served: the served workload's own JSON line."""
    line = measure_served(args, dist, args.requests, args.rate, args.max_iter, args.rel_tol)
    if dist.rank == 0:
        print(json.dumps(line))


def measure_served(args, dist, requests, rate, max_iter, rel_tol):
    """A Poisson request stream (rate, seeded) of meshes of 10k-720k cells,
    each solved until rms < rel_tol x its first rms or max_iter iterations,
    through the continuous-batching server under an HBM budget; p50/p99
    latency from arrival to result and solves/s.  Against: the same
    requests' solves through the plain C API, one after another, timed on a
    sample and scaled.  Ranks take every N-th request.  Returns the
    measurement as a JSON-able dict."""
    from oplus2_matlab_b200 import group as G
    from oplus2_matlab_b200 import mesh as M
    from oplus2_matlab_b200 import serve as S
    from oplus2_matlab_b200 import api
    dt = np.float64 if args.fp64 else np.float32
    inst = G.draw_instances(requests, seed=M.SEED + 1, cmin=10000, cmax=720000)
    rng = np.random.default_rng(M.SEED)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, requests))
    mine = list(range(dist.rank, requests, dist.world))
    meshes = gen_meshes([inst[i][:2] for i in mine])
    api.set_error_mode(api.ERRORS_RETURN)
    warm_paths(dt, args.group_tiled)
    grp = G.Group(dt)
    if args.group_tiled:
        grp.set_tiled(True)
    srv = S.Server(dt, budget_bytes=args.budget_gb * 1e9, iters_per_step=args.iters_per_step,
                   max_active=args.max_active, policy=args.policy, group=grp)
    reqs = [S.Request(i, meshes[inst[i][:2]], inst[i][2], inst[i][3], max_iter,
                      rel_tol, float(arrivals[i])) for i in mine]
    clocks = Clocks(dist.local)
    dist.barrier()
    t0 = time.perf_counter()
    base = srv.now()  # arrivals and latencies on the C++ server's clock
    for r in reqs:
        r.arrival += base
    nxt = 0
    while nxt < len(reqs) or not srv.idle():
        now = srv.now()
        while nxt < len(reqs) and reqs[nxt].arrival <= now:
            srv.submit(reqs[nxt])
            nxt += 1
        if srv.idle() and nxt < len(reqs):
            time.sleep(max(0.0, min(reqs[nxt].arrival - srv.now(), 0.01)))
            continue
        srv.step()
    wall = dist.max(time.perf_counter() - t0)
    clk = clocks.stop()
    stats = S.latency_stats(srv.done)
    iters = np.array([r.iterations for r in srv.done])
    by_tol = int(sum(1 for r in srv.done if r.iterations < r.max_iter))
    max_active = srv.peak_active
    srv.close()

    # the plain path on a sample of the same requests, same iteration counts
    # a uniform sample of the stream (in arrival order), not the first to finish
    by_arrival = sorted(srv.done, key=lambda r: r.arrival)
    ns = max(1, min(args.plain_sample, len(by_arrival)))
    sample = [by_arrival[(2 * k + 1) * len(by_arrival) // (2 * ns)] for k in range(ns)]
    t0 = time.perf_counter()
    for r in sample:
        G.plain_solve(r.mesh, r.mach, r.alpha, r.iterations, dt)
    t_sample = time.perf_counter() - t0
    frac = sum(r.iterations * r.mesh.ncell for r in sample) / max(
        1, sum(r.iterations * r.mesh.ncell for r in srv.done))
    plain_serial_s = t_sample / max(frac, 1e-12)  # the whole stream, scaled by cell-iterations
    line = {
        "metric": "served airfoil solves/s", "value": requests / wall, "unit": "solves/s",
        "n_gpus": dist.world, "steps": requests, "warmup": 0,
        "ms_per_step": 1e3 * wall / requests, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64" if args.fp64 else "f32",
        "data": "synthetic: Poisson(%g/s) arrivals, seeded NACA0012 meshes 10k-720k cells, "
                "Mach U[0.3,0.7], alpha U[-2,6] deg" % rate,
        "config": {"workload": "airfoil served: %d requests, stop at rms < %g x first or %d "
                               "iterations, %g GB budget" % (requests, rel_tol,
                                                              max_iter, args.budget_gb),
                   "rate_per_s": rate,
                   "iters_per_step": args.iters_per_step, "policy": args.policy,
                   "max_active": args.max_active,
                   "parallelism": "requests dealt round-robin over %d GPU(s)" % dist.world},
        "latency": stats,
        "wall_seconds": wall,
        "iterations": {"mean": float(iters.mean()), "min": int(iters.min()),
                       "max": int(iters.max())},
        "max_active_solves_rank0": max_active,
        "retired_by_rms_tolerance": by_tol, "retired_by_iteration_cap": len(srv.done) - by_tol,
        "plain_serial": {"sample": len(sample), "sample_seconds": t_sample,
                         "estimated_seconds": plain_serial_s,
                         "solves_per_s": requests / plain_serial_s,
                         "scaled_by": "cell-iterations of the sample over the stream"},
        "speedup_vs_plain": plain_serial_s / wall,
        "clocks": clk,
    }
    return line


def run_reference_jac(NN, niter, threads=None, variant=1):
    """The reference's OpenMP jac1 or jac2 (oracle/_ref/jac<v>_op) at NN, niter;
    returns (iterations/s from its own op_timing_output, seconds, cores) or None."""
    binary = os.path.join(ROOT, "oracle", "_ref", "jac%d_op" % variant)
    if not os.path.exists(binary):
        return None
    cores = threads or os.cpu_count()
    env = dict(os.environ, OMP_NUM_THREADS=str(cores), OMP_PROC_BIND="close",
               OP2REF_NN=str(NN), OP2REF_NITER=str(niter))
    r = subprocess.run([binary], env=env, capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        return None
    tot = 0.0
    for line in r.stdout.splitlines():
        f = line.split()
        if len(f) >= 4 and f[0].isdigit() and f[-1] in ("res", "update"):
            tot += float(f[1])
    return (niter / tot if tot > 0 else None), tot, cores


def run_jac_e2e(jm, niter, dist):
    """A complete jac1 solve through the C API (apps/jac_app.cpp): the grid
    from pinned host arrays, niter iterations with u_max and u_sum returned
    after every update, u fetched to the host.  Wall-clock timed."""
    from oplus2_matlab_b200 import api
    cr = cudart()
    app = C.CDLL(os.path.join(ROOT, "oplus2_matlab_b200", "lib", "libop2b200_apps.so"))
    app.op2b_jac1_app.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(AppTiming)]
    pins = []
    pp = pinned_array(jm.pp.shape, np.int32, pins)
    pp[...] = jm.pp
    A = pinned_array((jm.nedge,), np.float32, pins)
    A[...] = jm.A.reshape(-1)
    r = pinned_array((jm.nnode,), np.float32, pins)
    r[...] = jm.r.reshape(-1)
    u = pinned_array((jm.nnode,), np.float32, pins)
    umax = np.zeros(niter, np.float64)
    urms = np.zeros(niter, np.float64)
    t = AppTiming()
    api.set_error_mode(api.ERRORS_RETURN)
    dist.barrier()
    rc = app.op2b_jac1_app(jm.nnode, jm.nedge, pp.ctypes.data, A.ctypes.data, r.ctypes.data,
                           niter, u.ctypes.data, umax.ctypes.data, urms.ctypes.data, C.byref(t))
    total = dist.max(t.t_total)
    ok = rc == 0 and bool(np.isfinite(u).all())
    free_pinned(pins)
    if not ok:
        return None
    return {"value": dist.world * niter / total, "unit": "iters/s",
            "h2d_bytes_per_step": t.h2d_bytes / niter, "d2h_bytes_per_step": t.d2h_bytes / niter,
            "iterations": niter, "seconds": total,
            "phases_s": {"declare_h2d": t.t_declare, "iterate": t.t_iterate,
                         "fetch_d2h": t.t_fetch},
            "path": "C API (libop2b200_apps.so op2b_jac1_app: op_decl_* from pinned host "
                    "arrays, op_par_loop_res / op_par_loop_update with u_max and u_sum to the "
                    "host every update, op_fetch_data)"}


def impl_jac(args, dist):
    """jac1 (config 0 of the reference's apps): an (NN-1)^2-node Jacobi grid
    stored unstructured, 100 iterations of res (indirect OP_INC) + update
    (direct, sum and max reductions).  value: one iteration per CUDA-graph
    launch, reductions deferred, L2 flushed before each; e2e: the same
    iterations through the C API with both reductions returned to the host
    every iteration; cpu_baseline: the reference's OpenMP jac1_op."""
    from oplus2_matlab_b200 import api, apps
    from oplus2_matlab_b200 import mesh as M
    lib = api.lib()
    cr = cudart()
    NN, niter, V = args.nn, max(args.steps, 1), args.jac_variant
    jm = M.jac(NN, V)
    api.set_error_mode(api.ERRORS_RETURN)
    api.op_init([], 0)
    api.set_strategy(api.STRATEGY_GATHER)
    api.set_reduction(api.REDUCE_TREE)
    for kv in args.tune:
        k, v = kv.split("=")
        lib.op2b_set_tuning(k.encode(), int(v))
    J = apps.Jac(jm, V)
    J.iterate(max(3, args.warmup))
    api.sync()
    # e2e (Python path, kept for comparison): every iteration returns u_sum
    # and u_max to the host
    t0 = time.perf_counter()
    J.iterate(niter)
    e2e_py_s = time.perf_counter() - t0
    # device: two iterations per graph launch, reductions deferred.  Rotated:
    # a res runs first, and each graph holds update, res, update, res (two
    # fused launches for jac1, each writing u and du to the other of two
    # buffers: two per graph leave them where they were); the last update
    # runs after the timed steps
    api.set_gbl_deferred(1)
    res = lambda: api.op_par_loop("res", J.edges, *J.res_args)
    upd = lambda: api.op_par_loop("update", J.nodes, *J.upd_args)
    res()
    upd()
    res()  # plans of the fused step built outside the capture
    api.sync()
    assert lib.op2b_l2_flush() == 0
    assert lib.op2b_capture_begin(0) == 1, api.last_error()
    for rep in range(2):
        if rep:
            assert lib.op2b_l2_flush() == 0  # the second iteration starts cold too
        upd()
        res()
    g = lib.op2b_capture_end()
    assert g, api.last_error()
    nk = (lib.op2b_graph_nkernels(g) - 1) / 2.0
    assert lib.op2b_capture_begin(0) == 1, api.last_error()
    assert lib.op2b_l2_flush() == 0
    gf = lib.op2b_capture_end()
    assert gf, api.last_error()
    stream = lib.op2b_get_stream()
    assert lib.op2b_l2_flush() == 0
    ev = []
    for _ in range(2 * niter):
        e = C.c_void_p()
        cr.cudaEventCreate(C.byref(e))
        ev.append(e)
    for _ in range(3):
        lib.op2b_graph_launch(g)
    clocks = Clocks(dist.local)
    dist.barrier()
    cr.cudaStreamSynchronize(stream)
    for k in range(niter):
        lib.op2b_l2_flush()
        cr.cudaEventRecord(ev[2 * k], stream)
        lib.op2b_graph_launch(g)
        cr.cudaEventRecord(ev[2 * k + 1], stream)
    cr.cudaStreamSynchronize(stream)
    clk = clocks.stop()
    ms = []
    for k in range(niter):
        m = C.c_float()
        cr.cudaEventElapsedTime(C.byref(m), ev[2 * k], ev[2 * k + 1])
        ms.append(m.value)
    # the captured sweep between the two iterations, timed alone the same way
    sweep = []
    for k in range(niter):
        lib.op2b_l2_flush()
        cr.cudaEventRecord(ev[2 * k], stream)
        lib.op2b_graph_launch(gf)
        cr.cudaEventRecord(ev[2 * k + 1], stream)
    cr.cudaStreamSynchronize(stream)
    for k in range(niter):
        m = C.c_float()
        cr.cudaEventElapsedTime(C.byref(m), ev[2 * k], ev[2 * k + 1])
        sweep.append(m.value)
    ms = [a - float(np.mean(sweep)) for a in ms]
    total = dist.max(sum(ms) * 1e-3)
    lib.op2b_graph_destroy(g)
    lib.op2b_graph_destroy(gf)
    upd()
    api.sync()
    api.set_gbl_deferred(0)
    u = J.fetch().copy()
    ok = bool(np.isfinite(u).all())
    api.op_exit()
    value = dist.world * 2 * niter / total  # two iterations per graph launch
    # end to end through the C API (jac1: libop2b200_apps.so op2b_jac1_app,
    # the reference's main over the caller's arrays, u_max and u_sum to the
    # host after every update; three solves, the median), else the Python app
    e2e = {"value": niter / e2e_py_s, "unit": "iters/s", "h2d_bytes_per_step": 0,
           "d2h_bytes_per_step": 16,
           "path": "Python Jac app over the C API, u_sum and u_max to the host every "
                   "iteration"}
    if V == 1:
        runs = [run_jac_e2e(jm, args.e2e_iters, dist) for _ in range(3)]
        runs = sorted([r for r in runs if r], key=lambda r: r["value"])
        if runs:
            e2e = dict(runs[len(runs) // 2], all_values=[r["value"] for r in runs],
                       python_app_iters_per_s=niter / e2e_py_s)
    # compulsory bytes per iteration: res = A and the map pair per edge, u
    # read and du read+write per node; update = r, du rw, u rw per node.
    # jac1: 4 + 8 per edge, 4 + 8 + (4 + 8 + 8) per node; jac2 (A double[3],
    # u float[2], du float[3], r float[2]): 24 + 8, 8 + 24 + (8 + 24 + 16)
    if V == 1:
        it_bytes = 12.0 * jm.nedge + 12.0 * jm.nnode + 20.0 * jm.nnode
    else:
        it_bytes = 32.0 * jm.nedge + 32.0 * jm.nnode + 48.0 * jm.nnode
    peak, peak_kind = measured_peak()
    cpu = None
    if not args.no_cpu_baseline and dist.rank == 0 and dist.world == 1:
        r = run_reference_jac(NN, min(niter, 100), variant=V)
        if r and r[0]:
            cpu = {"value": r[0], "unit": "iters/s", "cores": r[2], "kind": "reference",
                   "sample": "%d iterations at NN=%d (reference jac%d_op, OpenMP, sum of its "
                             "op_timing_output)" % (min(niter, 100), NN, V)}
    line = {
        "metric": "jac%d iters/s" % V, "value": value, "unit": "iters/s", "n_gpus": dist.world,
        "steps": niter, "warmup": max(3, args.warmup), "ms_per_step": 1e3 * total / niter,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: the reference's jac%d grid generator (jac%d/jac.cpp)" % (V, V),
        "config": {"workload": "jac%d NN=%d: %d nodes, %d edges, two iterations (res + update "
                               "each; rotated: update then the next res) per step"
                               % (V, NN, jm.nnode, jm.nedge),
                   "l2": "flushed before every iteration (a sweep captured between the "
                         "two iterations of a step, its time measured alone and subtracted)",
                   "parallelism": "single GPU"},
        "roofline": {"bound": "hbm", "kernel": "res + update (one iteration)",
                     "achieved": it_bytes * value / dist.world / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": it_bytes * value / dist.world / 1e9 / peak,
                     "traffic": None, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": it_bytes},
        "e2e": e2e,
        "gpu_launches": int(2 * nk * niter), "kernels_per_iteration": nk,
        "finite": ok, "cpu_baseline": cpu, "clocks": clk,
    }
    if dist.rank == 0:
        print(json.dumps(line))


def impl_layout(args, dist):
    """--mode layout: res_calc's flux pass on the 720k mesh with the datasets
    stored AoS (the library's layout) and SoA, same arithmetic, outputs
    compared bit for bit (op2b_layout_ab); L2 flushed before each launch."""
    from oplus2_matlab_b200 import api, apps
    from oplus2_matlab_b200 import mesh as M
    lib = api.lib()
    mesh = plain_mesh(args)
    K = apps.airfoil_consts(np.float32)
    rng = np.random.default_rng(MESH_SEED)
    q = (np.tile(K["qinf"], (mesh.ncell, 1)) *
         (1.0 + 0.01 * rng.standard_normal((mesh.ncell, 4)))).astype(np.float32)
    adt = rng.uniform(1.0, 50.0, mesh.ncell).astype(np.float32)
    x = np.ascontiguousarray(mesh.x(np.float32), np.float32)
    pe = np.ascontiguousarray(mesh.edge, np.int32)
    pc = np.ascontiguousarray(mesh.ecell, np.int32)
    ta, ts = C.c_double(), C.c_double()
    clocks = Clocks(dist.local)
    rc = lib.op2b_layout_ab(mesh.nedge, mesh.ncell, mesh.nnode, pe.ctypes.data, pc.ctypes.data,
                            x.ctypes.data, q.ctypes.data, adt.ctypes.data, float(K["gm1"]),
                            float(K["eps"]), max(3, args.steps), C.byref(ta), C.byref(ts))
    clk = clocks.stop()
    # compulsory bytes: pedge + pecell (16 per edge), q (16) and adt (4) per
    # cell, x (8) per node, the flux record written (16 per edge)
    algo = 32.0 * mesh.nedge + 20.0 * mesh.ncell + 8.0 * mesh.nnode
    peak, kind = measured_peak()
    line = {"metric": "res_calc flux pass us per launch, AoS vs SoA", "unit": "us",
            "value": ta.value, "higher_is_better": False, "n_gpus": 1, "steps": max(3, args.steps),
            "warmup": 1, "dtype": "f32", "data": "synthetic: 720k mesh, perturbed free stream",
            "config": {"workload": "flux pass over %d interior edges" % mesh.nedge},
            "aos_us": ta.value, "soa_us": ts.value, "soa_over_aos": ts.value / ta.value,
            "outputs_bit_identical": rc == 0, "rc": rc,
            "algorithmic_bytes": algo, "aos_gbs": algo / ta.value / 1e3,
            "soa_gbs": algo / ts.value / 1e3, "peak_gbs": peak, "peak_source": kind,
            "clocks": clk}
    print(json.dumps(line))


def main():
    args = parse()
    dist = Dist()
    try:
        if args.impl == "reference":
            impl_reference(args, dist)
        elif args.mode == "batched":
            impl_batched(args, dist)
        elif args.mode == "served":
            impl_served(args, dist)
        elif args.mode == "jac":
            impl_jac(args, dist)
        elif args.mode == "layout":
            impl_layout(args, dist)
        else:
            impl_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
