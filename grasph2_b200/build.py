"""In-tree build of libgrasph2_b200.so for sm_100a (nvcc; no JIT, no torch extension cache).

    python grasph2_b200/build.py [--force] [--verbose]

Flags: -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -std=c++17 -ftz=true. Denormal
results flush to zero (single-instruction reciprocal square roots in the pair loops); no
-use_fast_math, so divisions and square roots outside the pair loops stay IEEE.
"""

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libgrasph2_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
SOURCES = ["capi.cu", "pairs.cu", "integrate.cu", "spatial.cu", "noalloc.cu", "fp64.cu", "ensemble.cu", "mlp.cu", "surrogate.cu", "surrogate_run.cu", "ics.cu", "writer.cu", "h5io.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-ftz=true", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                     "--expt-relaxed-constexpr", "-I", INCLUDE]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _deps():
    out = []
    for f in os.listdir(CSRC):
        if f.endswith((".cu", ".cuh", ".h")):
            out.append(os.path.join(CSRC, f))
    out.append(os.path.join(INCLUDE, "grasph2_b200.h"))
    return out


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in _deps()):
            return LIB
    objs = []
    procs = []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for cmd, p in procs:
        out, _ = p.communicate()
        if verbose or ptxas_info:
            sys.stdout.write(out)
        if p.returncode != 0:
            failed.append((cmd, out))
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(" ".join(c) + "\n" + o for c, o in failed))
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed: %s\n%s" % (" ".join(cmd), r.stdout + r.stderr))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/spill info")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas))
