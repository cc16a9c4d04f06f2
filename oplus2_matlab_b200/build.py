"""Build libop2b200.so (the OP2 drop-in library) in-tree for sm_100a.

    python -m oplus2_matlab_b200.build          # incremental
    python -m oplus2_matlab_b200.build --force  # rebuild everything

Every .cu / .cpp under csrc/ is compiled by nvcc for sm_100a only, with
-fmad=false and IEEE division and square root so per-element arithmetic matches
the reference's x86 build bit for bit.  The result lands in lib/, next to this
file, which is where the ctypes loader looks for it.
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libop2b200.so")
APPS = os.path.join(HERE, "apps")
APPS_LIB = os.path.join(LIBDIR, "libop2b200_apps.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-ftz=false", "-Xcompiler", "-fPIC,-O3,-ffp-contract=off", "-I" + os.path.join(ROOT, "include"),
    "-I" + CSRC, "--expt-relaxed-constexpr",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(ROOT, "include")
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return hs


def _compile(src, obj, force):
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return None
    cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return r.stderr.strip() or None


def build(force=False, verbose=True):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sources()
    objs = [os.path.join(BUILD, os.path.basename(s) + ".o") for s in srcs]
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        futs = {ex.submit(_compile, s, o, force): s for s, o in zip(srcs, objs)}
        for f in concurrent.futures.as_completed(futs):
            msg = f.result()
            if msg and verbose:
                print("[%s] %s" % (os.path.basename(futs[f]), msg))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    # the apps (C++ over the public C API only) link against the library
    app_srcs = sorted(os.path.join(APPS, f) for f in os.listdir(APPS) if f.endswith(".cpp"))
    newest_app = max([os.path.getmtime(s) for s in app_srcs] + [os.path.getmtime(LIB)] +
                     [os.path.getmtime(h) for h in headers()])
    if force or not os.path.exists(APPS_LIB) or os.path.getmtime(APPS_LIB) < newest_app:
        cmd = [nvcc(), "-O2", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared",
               "-I" + os.path.join(ROOT, "include"), "-o", APPS_LIB] + app_srcs + \
              ["-L" + LIBDIR, "-lop2b200", "-lcudart", "-Xlinker", "-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("apps build failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
