"""Build recipe for the checker libraries (test infrastructure only).

  python oracle/build_ref.py            # both: oracle/liboracle.so and oracle/_ref/*.so
  python oracle/build_ref.py --oracle   # only the FP64 restatement

oracle/liboracle.so   the FP64 restatement, oracle/oracle.cpp (g++ -O2 -fopenmp)
oracle/_ref/libref_<variant>_<fp32|fp64>.so
                      GraSPH2's own job headers compiled in place from the reference tree with
                      g++ -O3 -march=native -fopenmp against the stand-ins in oracle/ref_shim/
                      (mpUtils is not vendored with the reference and not installed). Needs the
                      reference source tree; skipped with a message when it is absent.
oracle/_ref/libref_io.so
                      GraSPH2's tsv snapshot writer (src/ResultStorageManager.cu) and tsv particle
                      source (src/initialConditions/particleSources/TextFile.h), compiled in place
                      for the host against oracle/ref_shim/ref_io.h (oracle/ref_io_driver.cpp).
oracle/_ref/libref_cuda_<variant>.so
                      GraSPH2's own CUDA path (the tile kernels of src/particles/algorithms.h, the
                      jobs of src/computeDerivatives.h, the integrator of src/integration.h) compiled
                      in place with nvcc for sm_100a, FP32 as the reference ships, against the
                      stand-ins in oracle/ref_shim_cuda/ (oracle/ref_cuda_driver.cu).

The reference tree is read in place from $GRASPH2_REFERENCE, by default /root/reference (where the
read-only GraSPH2 checkout is mounted for this build); without it the recipe builds only the FP64
restatement (oracle/liboracle.so).
"""

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ref_variants  # noqa: E402

REFERENCE_SRC = os.environ.get("GRASPH2_REFERENCE") or "/root/reference"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_oracle(force=False):
    src = os.path.join(HERE, "oracle.cpp")
    out = os.path.join(HERE, "liboracle.so")
    hdr = os.path.join(HERE, "..", "include", "grasph2_b200.h")
    if force or _stale(out, [src, hdr]):
        _run(["g++", "-std=c++17", "-O2", "-fopenmp", "-fPIC", "-shared", "-o", out, src])
    return out


def _reference_src():
    src_dir = os.path.join(REFERENCE_SRC, "src") if REFERENCE_SRC else ""
    if not src_dir or not os.path.isdir(src_dir):
        print("build_ref: reference tree not found at %s (set GRASPH2_REFERENCE); oracle/_ref not built"
              % REFERENCE_SRC)
        return None
    return src_dir


def build_ref(force=False, march="native"):
    src_dir = _reference_src()
    if src_dir is None:
        return []
    out_dir = os.path.join(HERE, "_ref")
    os.makedirs(out_dir, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim")
    deps = [os.path.join(HERE, "ref_driver.cpp"), os.path.join(HERE, "ref_variants.py")]
    for root, _, files in os.walk(shim):
        deps += [os.path.join(root, f) for f in files]
    outs = []
    for name, v in ref_variants.VARIANTS.items():
        for double in (False, True):
            out = os.path.join(out_dir, "libref_%s_%s.so" % (name, "fp64" if double else "fp32"))
            outs.append(out)
            if not (force or _stale(out, deps)):
                continue
            cmd = ["g++", "-std=c++17", "-O3", "-march=%s" % march, "-fopenmp", "-fPIC", "-shared", "-w",
                   "-I", shim, "-I", src_dir, "-o", out, os.path.join(HERE, "ref_driver.cpp")]
            cmd += ref_variants.compile_defines(v, double)
            _run(cmd)
    return outs


def build_ref_io(force=False):
    """GraSPH2's tsv writer and reader (src/ResultStorageManager.cu, TextFile.h) for the host."""
    src_dir = _reference_src()
    if src_dir is None:
        return []
    out = os.path.join(HERE, "_ref", "libref_io.so")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    deps = [os.path.join(HERE, "ref_io_driver.cpp"), os.path.join(HERE, "ref_shim", "ref_io.h"),
            os.path.join(HERE, "ref_shim", "settings.h"), os.path.join(HERE, "ref_variants.py")]
    if force or _stale(out, deps):
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-w", "-I", os.path.join(HERE, "ref_shim"),
               "-I", src_dir, "-o", out, os.path.join(HERE, "ref_io_driver.cpp"), "-lpthread"]
        cmd += ref_variants.compile_defines(ref_variants.VARIANTS["nbody"], False)
        _run(cmd)
    return [out]


def build_ref_cuda(force=False):
    """GraSPH2's CUDA path for sm_100a, one FP32 library per physics variant (built in parallel)."""
    src_dir = _reference_src()
    if src_dir is None or not os.path.exists(NVCC):
        return []
    out_dir = os.path.join(HERE, "_ref")
    os.makedirs(out_dir, exist_ok=True)
    deps = [os.path.join(HERE, "ref_cuda_driver.cu"), os.path.join(HERE, "ref_variants.py"),
            os.path.join(HERE, "ref_shim", "settings.h")]
    for root, _, files in os.walk(os.path.join(HERE, "ref_shim_cuda")):
        deps += [os.path.join(root, f) for f in files]
    procs, outs = [], []
    for name, v in ref_variants.VARIANTS.items():
        out = os.path.join(out_dir, "libref_cuda_%s.so" % name)
        outs.append(out)
        if not (force or _stale(out, deps)):
            continue
        cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
               "--default-stream", "per-thread", "-Xcompiler", "-fPIC", "-shared", "-w",
               "-I", os.path.join(HERE, "ref_shim_cuda"), "-I", os.path.join(HERE, "ref_shim"), "-I", src_dir,
               "-o", out, os.path.join(HERE, "ref_cuda_driver.cu")]
        cmd += ref_variants.compile_defines(v, False)
        if "VARIABLE_TIMESTEP" in v["switches"]:
            cmd.append("-DREF_VARIABLE_TIMESTEP=1")
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for cmd, p in procs:
        o, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("build failed: %s\n%s" % (" ".join(cmd), o))
    return outs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--oracle", action="store_true", help="build only liboracle.so")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build_oracle(a.force))
    if not a.oracle:
        for o in build_ref(a.force) + build_ref_io(a.force) + build_ref_cuda(a.force):
            print(o)


if __name__ == "__main__":
    main()
