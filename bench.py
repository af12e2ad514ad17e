"""Benchmark of the per-step hot path: one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload plummer|impact|fluid|ensemble|surrogate|mlp] [--accum plain|compensated]
                    [--legs auto|none|impact,ensemble,surrogate] [--no-cpu-baseline]

Workload (default): the pure N-body Plummer sphere at N = 1,048,576 (scale radius a = 1, masses 1/N,
velocities from the Plummer distribution function, G = 1, eps = 0.01, dt = 1e-3), seeded synthetic
initial conditions: the plain FP32 all-pairs path whose throughput is quoted against the FP32 peak. A
step is computeDerivatives + integrate (the captured step graph). At one GPU the default run adds the
other workloads as legs of the same line ("workloads"): the elastic-plastic two-sphere impact at
N = 65,536 with its energy drift over 1,000 steps against the FP64 form, the batched ensemble of 512
spheres against the same simulations run one by one, and the learned K = 8 surrogate at N = 262,144
against the plain solver.

Timing: W untimed steps, then K steps, each bracketed by CUDA events on the launching stream, with a
256 MiB write between steps (outside the events) to flush the 126 MB L2; barrier + synchronize on both
sides; the max over ranks. N > 1 runs independent replicas (the path is not sharded across GPUs) and
reports the whole-job rate.

--impl reference times GraSPH2's own CPU hot path (its job headers compiled for the host with OpenMP,
oracle/_ref) on this machine's cores, on bounded row samples of the same workload, extrapolated. The
cpu_baseline of our arm is that same reference arm, run as a child process.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/s & pair-interactions/s, chosen vs plain form at ≤1e-4 energy drift"

# Algorithmic flop model (frozen): per pair of the N^2 sweep and per neighbour pair (0 < r <= h) of
# the SPH passes.
FLOP_GRAV_PAIR = 20        # softened gravity, the GPU Gems 3 ch. 31 convention
FLOP_DENS_PAIR = 8         # distance test of the density sum
FLOP_DENS_NB = 10          # W(r) and the accumulation per neighbour
FLOP_FUSED_NB = 160        # strain/rotation rates, div v, stress acceleration, AV per neighbour (solids)
FLOP_ACC_NB = 60           # pressure acceleration + AV per neighbour (fluid, acceleration pass only)

FLUSH_BYTES = 256 << 20

# DRAM bytes (read + write) per launch of the dominant kernel, from one ncu capture of the same kernel
# and launch shape, on a smaller case where the full one is too large to capture (profiles/ holds the
# commands): key (workload, kernel slot, gravity form, symmetric groups; for the ensemble its number of
# simulations) -> (bytes per launch, particles of the captured case). The symmetric gravity kernel's
# traffic is its j-records (16 B per particle, read once from DRAM, then from L2) plus its partial slots
# ((G + 1) x 12 B per particle, written once), so at fixed G it scales with N.
MEASURED_TRAFFIC = {
    ("plummer", "gravity", "symmetric", 128): (356643200.0, 262144),  # ncu, N = 262,144, 2 launches (mean)
    ("impact", "gravity", "symmetric", 64): (2185728.0, 65536),  # ncu, the impact itself, 2 launches (mean)
    # the 512-simulation ensemble itself (4,630,521 particles, DENS j-tile 512), 2 launches (mean): the
    # neighbour lists the DENS stage writes and the SPH stage reads dominate it
    ("ensemble", "k_ensemble", "one-sided", 512): (5093712128.0, 4630521),
}
FLAG_DEAL_WITH_NO_PARTNERS = 1 << 3  # GSPH_DEAL_WITH_NO_PARTNERS


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference", "reference-cuda"], default="ours",
                    help="ours; reference = GraSPH2's CPU hot path on the host cores (the reference arm); "
                         "reference-cuda = GraSPH2's own CUDA path built for sm_100a (N % 256 == 0 only)")
    ap.add_argument("--workload", choices=["plummer", "impact", "fluid", "ensemble", "surrogate", "mlp"],
                    default="plummer")
    ap.add_argument("--legs", default="auto",
                    help="other workloads measured in the same run at one GPU (comma list of impact, ensemble, "
                         "surrogate; 'auto' = all three for the default Plummer workload, 'none' = off)")
    ap.add_argument("--windows", type=int, default=8, help="surrogate: windows of M proposals")
    ap.add_argument("--model", default=os.path.join(ROOT, "grasph2_b200", "data", "surrogate_impact_n262144.npz"),
                    help="surrogate: trained model (grasph2_b200/train_surrogate.py)")
    ap.add_argument("--nsims", type=int, default=512, help="simulations of the ensemble workload")
    ap.add_argument("--no-sequential", action="store_true",
                    help="ensemble: skip timing the simulations one by one in their own contexts")
    ap.add_argument("--accum", choices=["plain", "compensated"], default="plain")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0,
                    help="seconds of CPU work for the cpu_baseline (the reference arm run as a child process)")
    ap.add_argument("--ref-budget", type=float, default=100.0,
                    help="--impl reference: seconds of CPU work over all warm-up and timed steps")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-peak", action="store_true", help="skip the FFMA peak probe (profiling runs)")
    ap.add_argument("--n", type=int, default=0, help="particle count of the fluid / plummer workloads")
    ap.add_argument("--no-cull", action="store_true", help="all-pairs SPH sweeps (no chunk culling)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--scalar-fp32", action="store_true", help="scalar instead of paired f32x2 gravity kernel")
    ap.add_argument("--gravity", choices=["auto", "one-sided", "symmetric"], default="auto",
                    help="all-pairs gravity kernel: every ordered pair, or every unordered pair once")
    ap.add_argument("--gravity-groups", type=int, default=0, help="symmetric gravity: particle groups (0 = auto)")
    ap.add_argument("--drift-steps", type=int, default=-1,
                    help="steps of the energy-drift comparison (plain, compensated, FP64); default 1000 on the "
                         "impact workload, 0 (off) elsewhere")
    ap.add_argument("--drift-every", type=int, default=100, help="steps between energy samples of the drift run")
    return ap.parse_args(argv)


# ---- workloads ------------------------------------------------------------------------------------
def workload(name, n=0):
    """(params, state, description, reference variant) of a single-context workload."""
    from grasph2_b200 import ics
    from grasph2_b200.params import config0_params, config1_params, config2_params
    if name == "impact":
        st = ics.two_sphere_impact(seed=20261203)
        desc = ("elastic-plastic two-sphere impact, N=65536 (R=1: 58254, R=0.5: 7282), rho0=1, Murnaghan K=10, "
                "shear=5, von Mises Y=0.5, AV alpha=1 beta=2, h=2.5x mean spacing, G=1 eps=0.01, dt=1e-4")
        return config1_params(), st, desc, "impact"
    if name == "fluid":
        n = n or 4096
        st = ics.uniform_sphere(n, radius=1.0, rho0=0.239, omega=(0, 0, 0.1), seed=20261203)
        return config0_params(), st, "SPH + self-gravity fluid sphere, N=%d, h=0.15, eps=0.02" % n, "fluid"
    n = n or (1 << 20)
    st = ics.plummer_sphere(n, seed=20261203)
    return config2_params(), st, "Plummer sphere N-body, N=%d, a=1, eps=0.01, dt=1e-3" % n, "plummer"


def flops_per_step(params, st, counts, culled):
    """Algorithmic flops of each timed kernel slot in one step. With culling, gravity is its own
    all-pairs kernel and the SPH slots carry only the neighbour work; without it the acceleration
    pass also carries the N^2 gravity sweep and the density pass its N^2 distance tests."""
    from grasph2_b200._abi import FLAG_BITS as F
    n = st["mass"].shape[0]
    n2 = float(n) * n
    nb = counts
    out = {}
    grav = bool(params.flags & F["SELF_GRAVITY"])
    if params.flags & F["SPH"]:
        solids = params.flags & F["SOLIDS"]
        per_nb = FLOP_FUSED_NB if solids else FLOP_ACC_NB
        if not params.flags & F["INTEGRATE_DENSITY"]:
            out["density"] = FLOP_DENS_NB * nb + (0 if culled else FLOP_DENS_PAIR * n2)
        if culled:
            out["pairs"] = per_nb * nb
            if grav:
                out["gravity"] = FLOP_GRAV_PAIR * n2
        else:
            out["pairs"] = per_nb * nb + (FLOP_GRAV_PAIR * n2 if grav else 0)
    elif grav:
        out["gravity"] = FLOP_GRAV_PAIR * n2
    return out


def neighbour_pairs(pos, h, device):
    """Number of ordered pairs with 0 < r <= h (for the flop model), counted on the GPU with torch."""
    import torch
    x = torch.as_tensor(np.asarray(pos, dtype=np.float32), device=device)
    n = x.shape[0]
    total = 0
    chunk = 4096
    for i0 in range(0, n, chunk):
        d2 = torch.cdist(x[i0:i0 + chunk], x).pow_(2)
        total += int(((d2 > 0) & (d2 <= h * h)).sum().item())
    return total


# ---- clocks ---------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), "grasph2_clocks_%d.csv" % os.getpid())
        sel = self._selector(device_index)
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", sel, "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    @staticmethod
    def _selector(device_index):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        if vis:
            parts = [p.strip() for p in vis.split(",") if p.strip()]
            if device_index < len(parts):
                return parts[device_index]
        return str(device_index)

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as fh:
            lines = fh.readlines()
        try:
            os.remove(self.path)
        except OSError:
            pass
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                rows.append((float(f[0]), float(f[1]), float(f[2]), f[3], f[4], f[5], f[6], f[7]))
            except ValueError:
                continue
        if not rows:
            return None
        loaded = [r for r in rows if r[2] > 200.0] or rows
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in loaded:
            for nm, val in zip(names, r[4:8]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": max(r[1] for r in rows),
                "samples": len(loaded), "power_w_max": max(r[2] for r in rows), "reasons": sorted(reasons)}


# ---- CPU reference timing ------------------------------------------------------------------------
def reference_step_sampler(variant, st):
    """A timing sampler of the reference's own hot path (oracle/_ref, FP32 as shipped, OpenMP on all host
    cores): sample(m) runs computeDerivatives over target rows [0, m) (every pass, the density sum
    included) and integrate over all N, and returns (seconds of the row pass, seconds of integrate).
    Falls back to the FP64 oracle port (kind "port") where the reference build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from grasph2_b200.state import as_dtype
    if pyoracle.ref_available(variant):
        R = pyoracle.RefBuild(variant, double=False)
        s32 = as_dtype(st, np.float32)

        def sample(m):
            t0 = time.perf_counter()
            R.compute_derivatives_rows(s32, 0, m)
            t1 = time.perf_counter()
            R.integrate(s32, True)
            return t1 - t0, time.perf_counter() - t1
        return sample, "reference"
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        return None, None
    O = pyoracle.Oracle()
    params = workload(variant, st["mass"].shape[0])[0]
    s64 = as_dtype(st, np.float64)

    def sample(m):
        t0 = time.perf_counter()
        O.compute_derivatives(params, s64, 0, m)
        t1 = time.perf_counter()
        O.integrate(params, s64, True)
        return t1 - t0, time.perf_counter() - t1
    return sample, "port"


def rows_for_budget(sample, n, budget_s):
    """Target rows whose row pass takes about budget_s seconds (doubling from 64 rows)."""
    m = 64
    t = sample(m)[0]
    while t < 0.5 * budget_s and m < n:
        m = min(n, int(m * max(2.0, 0.7 * budget_s / max(t, 1e-3))))
        t = sample(m)[0]
    return m


def cpu_baseline_child(workload_name, n, budget_s):
    """The reference arm (--impl reference) on the same workload, run as a child process so that it has
    the host to itself (no CUDA context or GPU-side threads in the process): its steps/s is the
    cpu_baseline of our arm."""
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", workload_name,
           "--steps", "3", "--warmup", "1", "--ref-budget", str(budget_s)]
    if n:
        cmd += ["--n", str(n)]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "LOCAL_WORLD_SIZE")}
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=30 + 6 * budget_s)
    except subprocess.TimeoutExpired:
        return {"unavailable": "reference arm timed out"}
    for line in reversed(r.stdout.strip().splitlines()):
        try:
            d = json.loads(line)
        except ValueError:
            continue
        if "cpu_baseline" in d:
            return dict(d["cpu_baseline"], child="bench.py --impl reference --steps 3 --warmup 1 --ref-budget %g"
                        % budget_s)
        if "unavailable" in d:
            return {"unavailable": d["unavailable"]}
    return {"unavailable": "reference arm printed no line (rc %d): %s" % (r.returncode, r.stderr[-300:])}


def reference_line(args, value, t_rows, t_int, m, n, cores, kind, desc, workload_desc, pairs):
    return {
        "metric": METRIC, "value": value, "unit": "steps/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": dict(workload_desc, sample=desc),
        "pair_interactions_per_s": pairs * value,
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cores, "kind": kind, "sample": desc,
                         "row_pass_s": t_rows, "integrate_s": t_int},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference_arm(args, rank, world):
    """GraSPH2's own CPU hot path on this host's cores, on the workload of our arm: each step times
    computeDerivatives over a bounded row sample (extrapolated x N/rows, as the pair passes cost N per
    row) plus integrate over all N; steps/s = 1 / the mean of those step times."""
    if world > 1 and rank != 0:
        return None
    cores = os.cpu_count() or 1
    if args.workload in ("surrogate", "mlp"):
        return {"impl": "reference", "unavailable": "the reference has no %s" % args.workload}
    if args.workload == "ensemble":  # the reference's host path on the largest simulation, scaled by sum N_k^2
        params, sizes, states, desc = ensemble_workload(args.nsims)
        big = int(np.argmax(sizes))
        scale = float((sizes.astype(np.float64) ** 2).sum()) / float(sizes[big]) ** 2
        st = states[big]
        variant = "fluid"
        wdesc = {"workload": desc, "nsims": int(len(sizes)), "n_total": int(sizes.sum())}
        pairs = float((sizes.astype(np.float64) ** 2).sum())
    else:
        params, st, desc, variant = workload(args.workload, args.n)
        scale = 1.0
        wdesc = {"workload": desc, "n": int(st["mass"].shape[0])}
        pairs = flops_pairs(params, st["mass"].shape[0])
    sample, kind = reference_step_sampler(variant, st)
    if sample is None:
        return {"impl": "reference", "unavailable": "neither oracle/_ref nor oracle/liboracle.so is built"}
    n = st["mass"].shape[0]
    per = max(0.05, args.ref_budget / float(args.steps + args.warmup + 2))
    m = rows_for_budget(sample, n, per)
    rows, ints = [], []
    for k in range(args.warmup + args.steps):
        tr, ti = sample(m)
        if k >= args.warmup:
            rows.append(tr)
            ints.append(ti)
    t_rows = sum(rows) / len(rows)
    t_int = sum(ints) / len(ints)
    t_step = (t_rows * n / m + t_int) * scale
    value = 1.0 / t_step
    sdesc = ("GraSPH2 host jobs (FP32, OpenMP, %d threads): computeDerivatives on target rows [0,%d) of N=%d per "
             "step, extrapolated x N/rows, plus integrate of all N" % (cores, m, n))
    if kind == "port":
        sdesc = sdesc.replace("GraSPH2 host jobs (FP32,", "FP64 oracle port (")
    if scale != 1.0:
        sdesc += "; the largest simulation, scaled by sum N_k^2 / N^2 = %.1f" % scale
    return reference_line(args, value, t_rows, t_int, m, n, cores, kind, sdesc, wdesc, pairs)


def run_reference_cuda(args, rank, world):
    """GraSPH2's own CUDA path (oracle/_ref/libref_cuda_<variant>.so: its tile kernels, jobs and
    integrator compiled for sm_100a) on our arm's workload, where the reference can express it (its
    softening is eps == h and its AV signal coefficient 3; the cost per pair is the same). Steps are
    {computeDerivatives; integrate(true)} timed with CUDA events; valid for N % 256 == 0 only."""
    if world > 1 and rank != 0:
        return None
    if args.workload not in ("plummer", "impact", "fluid"):
        return {"impl": "reference-cuda", "unavailable": "no single-simulation reference run for %s" % args.workload}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    import torch
    from grasph2_b200.state import as_dtype
    params, st, desc, variant = workload(args.workload, args.n)
    n = st["mass"].shape[0]
    if not pyoracle.ref_cuda_available(variant):
        return {"impl": "reference-cuda", "unavailable": "oracle/_ref/libref_cuda_%s.so is not built" % variant}
    if n % 256:
        return {"impl": "reference-cuda", "unavailable": "N=%d is not a multiple of 256 (algorithms.h:285-301)" % n}
    torch.cuda.init()
    with pyoracle.RefCuda(variant, n) as r:
        r.upload(as_dtype(st, np.float32))
        r.set_timestep(0.0, 0.0)
        t1 = r.time_steps(1)  # warm-up, and the size of one step
        steps = int(max(1, min(args.steps, 4000.0 / max(t1, 1e-3))))
        ms = r.time_steps(steps)
    value = steps / (ms * 1e-3)
    return {"metric": METRIC, "value": value, "unit": "steps/s", "impl": "reference-cuda", "n_gpus": 1,
            "steps": steps, "warmup": 1, "ms_per_step": ms / steps, "higher_is_better": True, "dtype": "f32",
            "config": {"workload": desc, "n": n, "reference_variant": variant},
            "pair_interactions_per_s": flops_pairs(params, n) * value,
            "note": "GraSPH2's CUDA path recompiled for sm_100a (one thread per particle, 256-particle shared-memory "
                    "tiles), the reference's physics constants of this workload (eps == h, AV signal coefficient 3)"}


def reference_cuda_child(workload_name, n, steps):
    """run_reference_cuda in a child process: the reference's CUDA module stays out of our arm's process."""
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference-cuda", "--workload", workload_name,
           "--steps", str(steps), "--warmup", "1"]
    if n:
        cmd += ["--n", str(n)]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "LOCAL_WORLD_SIZE")}
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=300)
    except subprocess.TimeoutExpired:
        return {"unavailable": "reference CUDA run timed out"}
    for line in reversed(r.stdout.strip().splitlines()):
        try:
            d = json.loads(line)
        except ValueError:
            continue
        d.pop("metric", None)
        return d
    return {"unavailable": "reference CUDA run printed no line (rc %d): %s" % (r.returncode, r.stderr[-300:])}


def max_over_ranks(x, dist=None, device=None):
    """The largest of a local value over all ranks (a job's time is its slowest rank's)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(steps, world, total_ms):
    """Units all ranks processed / the slowest rank's time (replicas: every rank does `steps`)."""
    return steps * world / (total_ms * 1e-3)


def integrator_bytes(params):
    """Algorithmic bytes per particle of the leapfrog: read x64 24 + v 16 + a 16 (+ rho 4 + drho/dt 4 with
    SPH, + S 24 + dS/dt 24 with solids), write x64 24 + posm 16 + v 16 (+ rho 4, + S 24): 196 for the
    impact, 112 for gravity alone."""
    from grasph2_b200._abi import FLAG_BITS as F
    b = 56 + 56
    if params.flags & F["SPH"]:
        b += 12
        if params.flags & F["SOLIDS"]:
            b += 72
    return b


def integrator_roofline(prof, n, params):
    """HBM roofline of the leapfrog kernels: algorithmic bytes per launch / the launch's event time."""
    ms, cnt = prof.get("integrate", (0.0, 0))
    if not cnt:
        return None
    INTEGRATOR_BYTES = integrator_bytes(params)
    peaks = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks))["hbm_gbs"] if os.path.exists(peaks) else 6650.0
    gbs = INTEGRATOR_BYTES * n / (ms / cnt * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": "k_leapfrog_*", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
            "bytes_per_launch": INTEGRATOR_BYTES * n, "us_per_launch": ms / cnt * 1e3, "traffic": None,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if os.path.exists(peaks) else "fallback"}


def total_energy(d):
    return d["e_kin"] + d["e_grav"] + d["e_int"] + d["e_shear"]


def energy_drift(params, st, steps, every, stream, forms=("plain", "compensated"), autotune=True):
    """Total energy along `steps` steps of each FP32 form and of the double-precision form, all from
    the same float32-representable state. Every `every` steps the derivatives are refreshed at the
    current positions and the energy is taken at the synchronous velocity v + a dt/2. Returns, per
    form, max_t |E(t) - E_fp64(t)| / |E_fp64(0)| (the drift against the FP64 trajectory), its own
    max_t |E(t) - E(0)| / |E(0)|, and the simulated time per wall-second of its stepping (CUDA events
    around the step launches, diagnostics excluded). Each FP32 form first takes its own autotuned launch
    shapes, as the headline runs do (the tuner evaluates derivatives only: the state does not move)."""
    import torch
    from grasph2_b200.params import make_options
    from grasph2_b200.sim import DeviceParticleBuffer
    from grasph2_b200.state import as_dtype
    st = as_dtype(as_dtype(st, np.float32), np.float64)
    n = st["mass"].shape[0]
    dt = params.fixed_dt
    runs = {}
    for form in ("fp64",) + tuple(forms):
        opt = make_options(precision="double") if form == "fp64" else make_options(accum=form)
        energies, ms = [], 0.0
        with DeviceParticleBuffer(params, n, opt) as pb:
            pb.upload_f64(st, stream=stream)
            if form != "fp64" and autotune:
                pb.autotune(stream=stream)
            done = 0
            while True:
                pb.compute_derivatives(stream)
                energies.append(total_energy(pb.diagnostics(half_kick=0.5 * dt, stream=stream)))
                if done >= steps:
                    break
                k = min(every, steps - done)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                pb.step(k, stream)
                b.record(stream)
                b.synchronize()
                ms += a.elapsed_time(b)
                done += k
        runs[form] = (np.array(energies), ms)
    e64 = runs["fp64"][0]
    out = {"steps": steps, "sample_every": every, "reference": "double-precision GPU form",
           "forms": {}}
    for form, (e, ms) in runs.items():
        out["forms"][form] = {
            "rel_drift_vs_fp64": float(np.abs(e - e64).max() / abs(e64[0])),
            "rel_energy_change": float(np.abs(e - e[0]).max() / abs(e[0])),
            "sim_time_per_wall_s": steps * dt / (ms * 1e-3),
            "steps_per_s": steps / (ms * 1e-3),
        }
    return out


def flops_pairs(params, n):
    from grasph2_b200._abi import FLAG_BITS as F
    passes = 1
    if params.flags & F["SPH"]:
        passes = 2 if not params.flags & F["INTEGRATE_DENSITY"] else 1
        if params.flags & F["BALSARA_SWITCH"]:
            passes += 1
    return float(n) * n * passes


# ---- our arm ----------------------------------------------------------------------------------------
def ensemble_workload(nsims, seed=20261206):
    """Batched ensemble: nsims self-gravitating SPH spheres with the fluid physics (h=0.15, eps=0.02,
    c_s=1, rho0=0.239, dt=1e-3), each N a seeded log-uniform integer in [1024, 32768], radius 1,
    rigid rotation omega ~ U[0, 0.5] about z."""
    from grasph2_b200 import ics
    from grasph2_b200.params import config0_params
    sizes = ics.ensemble_sizes(nsims, seed=seed)
    rng = np.random.default_rng(seed + 1)
    params = config0_params()
    # h = 0.15 is fixed while N_k goes down to 1024: the smallest spheres have a mean spacing (0.16)
    # above h, so a particle can have no neighbour and a zero summed density. The reference's own
    # DEAL_WITH_NO_PARTNERS floor (rho < 0.001 -> 0.01 rho0, computeDerivatives.h:85-88) keeps them finite.
    params.flags |= FLAG_DEAL_WITH_NO_PARTNERS
    states = [ics.uniform_sphere(int(n), radius=1.0, rho0=0.239, omega=(0.0, 0.0, rng.uniform(0.0, 0.5)),
                                 seed=seed + 2 + k) for k, n in enumerate(sizes)]
    desc = ("batched ensemble of %d self-gravitating SPH spheres, N_k log-uniform in [1024, 32768] (total %d), "
            "radius 1, omega ~ U[0,0.5], h=0.15, eps=0.02, c_s=1, rho0=0.239, dt=1e-3, density floor "
            "DEAL_WITH_NO_PARTNERS" % (nsims, int(sizes.sum())))
    return params, sizes, states, desc


def ensemble_drift(params, states, steps, every, stream):
    """Energy of each simulation along `steps` steps run as an ensemble (FP32, the batched form) and one by
    one in the double-precision form, from the same float32-representable states. Returns per simulation
    max_t |E_ens(t) - E_fp64(t)| / |E_fp64(0)|, with the energy at the synchronous velocity after a
    derivative refresh every `every` steps (as energy_drift)."""
    from grasph2_b200.params import make_options
    from grasph2_b200.sim import DeviceParticleBuffer, Ensemble, pack_states
    from grasph2_b200.state import as_dtype
    states = [as_dtype(as_dtype(s, np.float32), np.float64) for s in states]
    sizes = [s["mass"].shape[0] for s in states]
    dt = params.fixed_dt
    e_ens = []
    with Ensemble(params, sizes) as ens:
        ens.upload(pack_states([as_dtype(s, np.float32) for s in states]), stream=stream)
        done = 0
        while True:
            ens.compute_derivatives(stream)
            e_ens.append([total_energy(d) for d in ens.diagnostics(0.5 * dt, stream)])
            if done >= steps:
                break
            k = min(every, steps - done)
            ens.step(k, stream)
            done += k
    e_ens = np.array(e_ens)
    out = []
    for j, st in enumerate(states):
        e64 = []
        with DeviceParticleBuffer(params, sizes[j], make_options(precision="double")) as pb:
            pb.upload_f64(st, stream=stream)
            done = 0
            while True:
                pb.compute_derivatives(stream)
                e64.append(total_energy(pb.diagnostics(0.5 * dt, stream)))
                if done >= steps:
                    break
                k = min(every, steps - done)
                pb.step(k, stream)
                done += k
        e64 = np.array(e64)
        out.append(float(np.abs(e_ens[:, j] - e64).max() / abs(e64[0])))
    return out


def run_ensemble(args, rank, world, local):
    """One step = every simulation of the ensemble advanced once (one persistent launch)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    from grasph2_b200.params import make_options
    from grasph2_b200.sim import DeviceParticleBuffer, Ensemble, measure_fp32_peak, pack_states
    from grasph2_b200.state import new_state

    # each rank advances its own ensemble of nsims simulations (different seeds): the simulations are the
    # units, sharded across ranks with no exchange; the whole job advances nsims x world of them
    params, sizes, states, desc = ensemble_workload(args.nsims, seed=20261206 + 1000 * rank)
    packed = pack_states(states)
    n_total = int(sizes.sum())
    pairs = float((sizes.astype(np.float64) ** 2).sum())
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    peak_tflops = None if args.no_peak else measure_fp32_peak(0.5)
    ens = Ensemble(params, sizes, make_options(accum=args.accum, gravity=args.gravity))
    ens.upload(packed, stream=stream)
    shape = {"tile": 512, "ctas_per_sm": 0} if args.no_autotune else ens.autotune(1, stream)
    for _ in range(args.warmup):
        flush.zero_()
        ens.step(1, stream)
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = ens.launch_count()
    sampler = ClockSampler(local)
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    for k in range(args.steps):
        flush.zero_()
        ev0[k].record(stream)
        ens.step(1, stream)
        ev1[k].record(stream)
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    gpu_launches = ens.launch_count() - launches0
    total_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in zip(ev0, ev1)), dist, dev)
    ms_per_step = total_ms / args.steps

    # e2e through the public API with pinned host buffers: upload, one step, download
    up_names = ["pos", "mass", "vel", "density"]
    down_names = ["pos", "vel", "acc", "density"]
    pinned_in = {k: torch.from_numpy(np.ascontiguousarray(packed[k], dtype=np.float32)).pin_memory().numpy()
                 for k in up_names}
    host_out = new_state(n_total, np.float32)
    pinned_out = {k: torch.empty(host_out[k].shape, dtype=torch.float32).pin_memory().numpy() for k in down_names}
    h2d = sum(a.nbytes for a in pinned_in.values())
    d2h = sum(a.nbytes for a in pinned_out.values())
    e2e_steps = 0 if args.no_e2e else max(3, min(args.steps, 10))
    e2e_ms = 0.0
    with Ensemble(params, sizes, make_options(accum=args.accum, gravity=args.gravity)) as e2:
        for k in range(e2e_steps + 2 if e2e_steps else 0):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            e2.upload(pinned_in, stream=stream)
            e2.step(1, stream)
            e2.download(down_names, stream=stream, out=pinned_out)
            b.record(stream)
            b.synchronize()
            if k >= 2:
                e2e_ms += a.elapsed_time(b)

    # the same simulations one after another, each in its own single-simulation context (plain path):
    # every 8th simulation in size order, each standing for 8
    seq_ms = None
    if not args.no_sequential and rank == 0:
        order = np.argsort(sizes)
        stride = max(1, len(order) // 64)
        pick = order[stride // 2::stride]
        tot = 0.0
        for k in pick:
            with DeviceParticleBuffer(params, int(sizes[k]), make_options(accum=args.accum)) as pb:
                pb.upload(states[k], stream=stream)
                pb.step(2, stream)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                pb.step(5, stream)
                b.record(stream)
                b.synchronize()
                tot += a.elapsed_time(b) / 5
        seq_ms = tot * len(order) / len(pick)

    if rank != 0:
        ens.close()
        if dist is not None:
            dist.destroy_process_group()
        return None
    value = whole_job_rate(args.steps, world, total_ms)
    nb = sum(neighbour_pairs(s["pos"], params.H, dev) for s in states[::8]) * 8
    flops = FLOP_GRAV_PAIR * pairs + FLOP_DENS_PAIR * pairs + (FLOP_DENS_NB + FLOP_ACC_NB) * nb
    achieved = flops / (ms_per_step * 1e-3) / 1e12
    cpu = None
    if not args.no_cpu_baseline:
        cpu = cpu_baseline_child("ensemble", 0, args.cpu_budget)
    drift = None
    if args.drift_steps != 0:
        nd = args.drift_steps if args.drift_steps > 0 else 1000
        order = np.argsort(sizes)
        pick = order[np.linspace(0, len(order) - 1, 8).astype(int)]
        d = ensemble_drift(params, [states[k] for k in pick], nd, args.drift_every, stream)
        # mean neighbours within h of a uniform sphere of radius 1: N (4/3 pi h^3) / (4/3 pi) = N h^3
        nbm = [float(sizes[k]) * params.H ** 3 for k in pick]
        resolved = [x for x, m in zip(d, nbm) if m >= 20.0]
        drift = {"steps": nd, "simulations": [int(sizes[k]) for k in pick], "mean_neighbours": nbm,
                 "rel_drift_vs_fp64": d,
                 "max_rel_drift_vs_fp64_resolved": max(resolved) if resolved else None,
                 "note": "simulations with fewer than 20 mean SPH neighbours (N < 5926 at h = 0.15) are below SPH "
                         "resolution: pairs entering and leaving h and the density floor make their trajectories "
                         "diverge at the particle level in any precision, so their energy comparison is not a "
                         "precision measure",
                 "sample": "8 simulations spanning the size range, run as an ensemble (FP32) and one by one in FP64"}
    form = "symmetric" if args.gravity == "symmetric" else "one-sided"
    ens_traffic = MEASURED_TRAFFIC.get(("ensemble", "k_ensemble", form, len(sizes)))
    if ens_traffic is not None:
        ens_traffic = ens_traffic[0] * n_total / ens_traffic[1]
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded initial conditions)",
        "energy_drift": drift,
        "config": {"workload": desc, "nsims": int(len(sizes)), "n_total": n_total, "form": args.accum,
                   "l2": "flushed between timed steps (256 MiB write)",
                   "step": "every simulation: computeDerivatives + integrate, one persistent launch in a CUDA graph",
                   "launch_shape": dict(shape, autotuned=not args.no_autotune),
                   "parallelism": ("%d ensembles of %d simulations, one per GPU" % (world, len(sizes)))
                   if world > 1 else "single GPU"},
        "simulation_steps_per_s": value * len(sizes),  # value already counts every rank's ensemble
        "pair_interactions_per_s": pairs * value,
        "sequential_plain_ms_per_step": seq_ms,
        "speedup_vs_sequential": (seq_ms / ms_per_step) if seq_ms else None,
        "roofline": {"bound": "fp32", "kernel": "k_ensemble", "achieved": achieved, "peak": peak_tflops,
                     "unit": "TFLOP/s", "frac": (achieved / peak_tflops) if peak_tflops else None,
                     "traffic": ens_traffic, "flops_per_launch": flops, "neighbour_pairs": nb,
                     "peak_source": "FFMA throughput measured in this run (gsph_measure_fp32_peak)"},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "e2e": ({"value": e2e_steps / (e2e_ms * 1e-3), "unit": "steps/s", "h2d_bytes_per_step": h2d,
                 "d2h_bytes_per_step": d2h} if e2e_steps else None),
        "gpu_launches": gpu_launches,
    }
    ens.close()
    if dist is not None:
        dist.destroy_process_group()
    return line


def run_surrogate(args, rank, world, local):
    """The learned K-substep surrogate on the impact at N=262,144 (v=0.5, y-offset 0.3, a seed outside the
    training set) against the plain solver over the same substeps: windows of M=4 proposals, the last
    judged by the plain integrator (accepted at <= 1e-3 relative position error and <= 1e-4 energy
    error), with the judge-calibrated energy correction. Reports simulated time per wall-second of the
    plain solver, the surrogate, the surrogate without the energy correction and the extrapolation
    without the network, the acceptance, and each trajectory's energy against the plain one every four
    windows (the energy diagnostics run outside the timed calls)."""
    import torch
    torch.cuda.set_device(local)
    from grasph2_b200 import ics
    from grasph2_b200 import surrogate as S
    from grasph2_b200.params import CONFIG4_N_BIG, CONFIG4_N_SMALL, config4_params
    from grasph2_b200.sim import DeviceParticleBuffer
    if rank != 0:
        return None
    if not os.path.exists(args.model):
        raise RuntimeError("trained model missing: %s" % args.model)
    sur = S.Surrogate.load(args.model)
    p = config4_params()
    n = CONFIG4_N_BIG + CONFIG4_N_SMALL
    st = ics.two_sphere_impact(CONFIG4_N_BIG, CONFIG4_N_SMALL, v_rel=0.5, y_offset=0.3, seed=20261299)
    M, K = 4, sur.K
    substeps = args.windows * M * K
    dt = float(np.float32(p.fixed_dt))
    chunk = 4  # windows between energy samples (taken outside the timed calls)
    forms = {"plain": None, "surrogate": (True, True), "surrogate_uncorrected": (True, False),
             "extrapolation": (False, True)}  # (network, energy correction)
    sampler = ClockSampler(local)
    out = {}
    energies = {}
    for form, how in forms.items():
        with DeviceParticleBuffer(p, n) as pb:
            pb.upload(st)
            pb.step(max(args.warmup, 1))
            if how is not None:
                sur.energy_correction(how[1], 1.0)
            torch.cuda.synchronize()
            l0 = pb.launch_count() + sur.launch_count()
            wall, acc, errs, series, done = 0.0, 0, [], [], 0
            while done < args.windows:
                w = min(chunk, args.windows - done)
                if how is None:
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    pb.step(w * M * K)
                    torch.cuda.synchronize()
                    wall += time.perf_counter() - t0
                else:
                    r = S.advance(pb, sur, w, M=M, use_net=how[0])
                    wall += r["wall_s"]
                    acc += r["accepted"]
                    errs += r["errors"]
                done += w
                d = pb.diagnostics(0.0, fast=True)
                series.append(d["e_kin"] + d["e_grav"] + d["e_int"] + d["e_shear"])
            launches = pb.launch_count() + sur.launch_count() - l0
            energies[form] = np.array(series)
            errs = np.array(errs) if errs else None
            out[form] = {"sim_time_per_wall_s": substeps * dt / wall, "substeps_per_s": substeps / wall,
                         "accepted_windows": acc if how is not None else None, "windows": args.windows,
                         "network": None if how is None else how[0],
                         "energy_correction": None if how is None else how[1],
                         "library_launches": launches,
                         "final_bias_estimate": None if how is None else list(sur.energy_bias()),
                         "position_errors": None if errs is None else [float(x) for x in errs[:, 0]],
                         "energy_errors": None if errs is None else [float(x) for x in errs[:, 1]]}
    clocks = sampler.stop()
    e0 = abs(energies["plain"][0])
    for form in out:  # |E_form - E_plain| / |E_plain| at every sample (every `chunk` windows)
        dev = np.abs(energies[form] - energies["plain"]) / e0
        out[form]["energy_vs_plain_at_end"] = float(dev[-1])
        out[form]["energy_vs_plain_max"] = float(dev.max())
        out[form]["energy_vs_plain_series"] = [float(x) for x in dev]
    value = out["surrogate"]["substeps_per_s"]
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": 1, "steps": substeps, "warmup": args.warmup,
        "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded initial conditions)",
        "config": {"workload": "learned K=8 surrogate, elastic-plastic impact N=%d (v=0.5, y-offset 0.3), windows of "
                               "M=4 proposals judged by the plain integrator (<=1e-3 position, <=1e-4 energy), "
                               "judge-calibrated energy correction" % n,
                   "model": os.path.basename(args.model), "substeps": substeps, "form": "surrogate"},
        "forms": out,
        "speedup_vs_plain": value / out["plain"]["substeps_per_s"],
        "clocks": clocks,
        "gpu_launches": out["surrogate"]["library_launches"],
    }
    return line


MLP_FWD_FLOPS = 2 * (32 * 128 + 2 * 128 * 128 + 128 * 13)                  # per row
MLP_TRAIN_FLOPS = MLP_FWD_FLOPS + 2 * (32 * 128 + 2 * 128 * 128 + 128 * 13) + 2 * (2 * 128 * 128 + 13 * 128)


def run_mlp(args, rank, world, local):
    """The surrogate's MLP on the tensor cores: forward over 1,048,576 rows and the gradient over 262,144
    rows per step (random inputs), TFLOP/s against the measured bf16 GEMM peak."""
    import torch
    torch.cuda.set_device(local)
    from grasph2_b200.mlp import MLP, init_params
    if rank != 0:
        return None
    nf, nt = 1 << 20, 1 << 18
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(nf, 32, device="cuda", generator=g)
    y = torch.empty(nf, 13, device="cuda")
    t = torch.randn(nt, 13, device="cuda", generator=g)
    w = torch.ones(13, device="cuda")
    stream = torch.cuda.current_stream()
    net = MLP(init_params(0))
    res = {}
    for name, f, rows, flops in (("forward", lambda: net.forward(x, y, nf, stream), nf, MLP_FWD_FLOPS),
                                 ("gradient", lambda: net.gradient(x, t, w, nt, stream, want=False), nt,
                                  MLP_TRAIN_FLOPS)):
        for _ in range(max(args.warmup, 1)):
            f()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for a, b in ev:
            a.record(stream)
            f()
            b.record(stream)
        torch.cuda.synchronize()
        ms = sorted(a.elapsed_time(b) for a, b in ev)[len(ev) // 2]
        res[name] = {"rows": rows, "ms": ms, "rows_per_s": rows / (ms * 1e-3), "tflops": rows * flops / (ms * 1e-3) / 1e12}
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"bf16_tflops": 1590.0}
    peak = peaks["bf16_tflops"]
    line = {"metric": "MLP rows/s (forward) on the tensor cores", "value": res["forward"]["rows_per_s"], "unit": "rows/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["forward"]["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic (random inputs)",
            "config": {"workload": "surrogate MLP 32-128-128-128-13 SiLU, BF16 operands, FP32 accumulation in TMEM",
                       "forward_rows": nf, "gradient_rows": nt},
            "kernels": res,
            "roofline": {"bound": "tensor", "kernel": "k_mlp_forward", "achieved": res["forward"]["tflops"], "peak": peak,
                         "unit": "TFLOP/s", "frac": res["forward"]["tflops"] / peak, "traffic": None,
                         "peak_source": "MEASURED_PEAKS.json bf16_tflops (cuBLAS burst)"},
            "gpu_launches": args.steps * 3}
    return line


_PEAK = {}


def fp32_peak(args):
    """FFMA throughput of this GPU (gsph_measure_fp32_peak), measured once per process."""
    if args.no_peak:
        return None
    if "tflops" not in _PEAK:
        from grasph2_b200.sim import measure_fp32_peak
        _PEAK["tflops"] = measure_fp32_peak(0.5)
    return _PEAK["tflops"]


def shape_options(shape, opts):
    """Options that reproduce an autotuned all-pairs gravity shape (gravity-only workloads)."""
    o = dict(opts)
    if shape.get("grav_sym_groups"):
        o.update(gravity="symmetric", gravity_groups=int(shape["grav_sym_groups"]))
    else:
        o.update(gravity="one-sided", i_per_thread=int(shape["grav_ipt"]), j_tile=int(shape["grav_jt"]),
                 j_split=int(shape["grav_nseg"]))
    return o


def run_context(args, rank, world, local, dist=None):
    """One simulation context (the Plummer, impact or fluid workload): the timed steps, the e2e leg, the
    roofline of the dominant kernel, the CPU baseline and (impact) the energy drift. Returns the line
    on rank 0."""
    import torch
    dev = torch.device("cuda", local)
    from grasph2_b200.params import make_options
    from grasph2_b200.sim import DeviceParticleBuffer

    params, st, desc, variant = workload(args.workload, args.n)
    n = st["mass"].shape[0]
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    peak_tflops = fp32_peak(args)
    gravity_only = not (params.flags & 2)

    def barrier():
        if dist is not None:
            dist.barrier()

    opts = dict(accum=args.accum, cull=not args.no_cull, scalar_fp32=args.scalar_fp32, gravity=args.gravity,
                gravity_groups=args.gravity_groups)
    pb = DeviceParticleBuffer(params, n, make_options(**opts))
    pb.upload(st, stream=stream)
    # gravity-only at large N: each candidate launch is a full N^2 sweep, so one timed launch per shape
    shape = pb.launch_shape() if args.no_autotune else pb.autotune(1 if gravity_only and n > 65536 else 3, stream)
    pb.profile_enable(True)
    for _ in range(args.warmup):
        flush.zero_()
        pb.step(1, stream)
        pb.profile_collect()
    pb.profile_reset()

    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = pb.launch_count()
    sampler = ClockSampler(local)
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)
    for k in range(args.steps):
        flush.zero_()
        ev0[k].record(stream)
        pb.step(1, stream)
        ev1[k].record(stream)
        pb.profile_collect()
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    gpu_launches = pb.launch_count() - launches0
    total_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in zip(ev0, ev1)), dist, dev)
    prof = pb.profile_read()

    # e2e: the public API with host buffers (pinned): upload inputs, one step, download the result
    up_names = ["pos", "mass", "vel"] + ([] if gravity_only else ["density", "dstress"])
    down_names = ["pos", "vel", "acc"] + ([] if gravity_only else ["density", "dstress"])
    from grasph2_b200.state import new_state
    pinned_in = {k: torch.from_numpy(np.ascontiguousarray(st[k], dtype=np.float32)).pin_memory().numpy()
                 for k in up_names}
    host_out = new_state(n, np.float32)
    pinned_out = {k: torch.empty(host_out[k].shape, dtype=torch.float32).pin_memory().numpy() for k in down_names}
    h2d = sum(a.nbytes for a in pinned_in.values())
    d2h = sum(a.nbytes for a in pinned_out.values())
    e2e_steps = 0 if args.no_e2e else max(3, min(args.steps, 50 if n <= 262144 else 5))
    pb.profile_enable(False)
    if gravity_only and e2e_steps:  # the same launch shape as the timed context, without re-tuning
        pb2 = DeviceParticleBuffer(params, n, make_options(**shape_options(shape, opts)))
    else:
        pb2 = DeviceParticleBuffer(params, n, make_options(**opts))
        if not args.no_autotune and e2e_steps:
            pb2.upload(pinned_in, stream=stream)
            pb2.autotune(3, stream)
    e2e_ms = 0.0
    for k in range(e2e_steps + 2 if e2e_steps else 0):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        pb2.upload(pinned_in, stream=stream)
        pb2.step(1, stream)
        pb2.download(down_names, stream=stream, out=pinned_out)
        b.record(stream)
        b.synchronize()
        if k >= 2:
            e2e_ms += a.elapsed_time(b)
    pb2.close()

    if rank != 0:
        pb.close()
        return None

    value = whole_job_rate(args.steps, world, total_ms)
    ms_per_step = total_ms / args.steps
    nb = 0 if gravity_only else neighbour_pairs(st["pos"], params.H, dev)
    fl = flops_per_step(params, st, nb, culled=not args.no_cull)
    timed = {k: prof[k][0] / prof[k][1] for k in fl if prof[k][1]}
    dominant = max(timed, key=lambda k: timed[k]) if timed else max(fl, key=lambda k: fl[k])
    ms_dom, cnt_dom = prof[dominant]
    achieved = fl[dominant] / (ms_dom / cnt_dom * 1e-3) / 1e12 if cnt_dom else None
    pairs_per_step = flops_pairs(params, n)
    sym_g = int(shape.get("grav_sym_groups") or 0)
    traffic = MEASURED_TRAFFIC.get((args.workload, dominant, "symmetric" if sym_g else "one-sided", sym_g))
    if traffic is not None:
        traffic = traffic[0] * n / traffic[1]  # bytes per particle of the captured case x N

    cpu = None
    ref_cuda = None
    if not args.no_cpu_baseline and world == 1:
        cpu = cpu_baseline_child(args.workload, args.n, args.cpu_budget)
        ref_cuda = reference_cuda_child(args.workload, args.n, 50)

    drift = None
    if args.drift_steps < 0:
        args.drift_steps = 1000 if args.workload == "impact" else 0
    if args.drift_steps > 0:
        drift = energy_drift(params, st, args.drift_steps, args.drift_every, stream, autotune=not args.no_autotune)

    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded initial conditions)",
        "config": {"workload": desc, "n": n, "form": args.accum, "culled": not args.no_cull,
                   "gravity_fp32": "scalar" if args.scalar_fp32 else "f32x2",
                   "l2": "flushed between timed steps (256 MiB write)",
                   "step": "computeDerivatives + integrate, one captured CUDA graph",
                   "launch_shape": dict(shape, autotuned=not args.no_autotune),
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "pair_interactions_per_s": pairs_per_step * value,
        "kernel_ms_per_step": {k: (v[0] / v[1] if v[1] else None) for k, v in prof.items()},
        "roofline": {"bound": "fp32", "kernel": dominant, "achieved": achieved, "peak": peak_tflops,
                     "unit": "TFLOP/s", "frac": (achieved / peak_tflops) if (achieved and peak_tflops) else None,
                     "traffic": traffic, "algorithmic_bytes": 16 * n, "flops_per_launch": fl[dominant],
                     "neighbour_pairs": nb,
                     "peak_source": "FFMA throughput measured in this run (gsph_measure_fp32_peak)"},
        "integrator_roofline": integrator_roofline(prof, n, params),
        "cpu_baseline": cpu,
        "reference_cuda": ref_cuda,
        "clocks": clocks,
        "e2e": ({"value": e2e_steps / (e2e_ms * 1e-3), "unit": "steps/s", "h2d_bytes_per_step": h2d,
                 "d2h_bytes_per_step": d2h} if e2e_steps else None),
        "gpu_launches": gpu_launches,
        "energy_drift": drift,
    }
    pb.close()
    return line


def leg_args(args, **over):
    a = argparse.Namespace(**vars(args))
    for k, v in over.items():
        setattr(a, k, v)
    return a


def run_legs(args, rank, world, local):
    """The other workloads of the default run (one GPU): each as its own line under "workloads"."""
    legs = args.legs
    if legs == "none" or world > 1 or rank != 0:
        return None
    if legs == "auto":
        if args.workload != "plummer" or args.n:
            return None
        legs = "impact,ensemble,surrogate"
    out = {}
    for leg in [x.strip() for x in legs.split(",") if x.strip()]:
        t0 = time.perf_counter()
        try:
            if leg == "impact":
                a = leg_args(args, workload="impact", n=0, steps=300, warmup=10, drift_steps=1000, gravity="auto",
                             gravity_groups=0, cpu_budget=min(args.cpu_budget, 10.0))
                line = run_context(a, rank, 1, local)
            elif leg == "ensemble":
                a = leg_args(args, workload="ensemble", steps=5, warmup=3, drift_steps=0,
                             cpu_budget=min(args.cpu_budget, 10.0))
                line = run_ensemble(a, rank, 1, local)
            elif leg == "surrogate":
                a = leg_args(args, workload="surrogate", warmup=1, windows=8)
                line = run_surrogate(a, rank, 1, local)
            else:
                line = {"error": "unknown leg %s" % leg}
        except Exception as e:  # a failing leg is reported, the headline line stands
            line = {"error": "%s: %s" % (type(e).__name__, e)}
        line["leg_wall_s"] = time.perf_counter() - t0
        out[leg] = line
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl in ("reference", "reference-cuda"):
        line = (run_reference_arm if args.impl == "reference" else run_reference_cuda)(args, rank, world)
        if line is not None:
            print(json.dumps(line))
        return

    if args.workload == "ensemble":
        line = run_ensemble(args, rank, world, local)
    elif args.workload == "surrogate":
        line = run_surrogate(args, rank, world, local)
    elif args.workload == "mlp":
        line = run_mlp(args, rank, world, local)
    else:
        import torch
        torch.cuda.set_device(local)
        dist = None
        if world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        line = run_context(args, rank, world, local, dist)
        if dist is not None:
            dist.destroy_process_group()
        if line is not None:
            legs = run_legs(args, rank, world, local)
            if legs:
                line["workloads"] = legs
    if line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
