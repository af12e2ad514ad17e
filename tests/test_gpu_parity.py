"""Parity of the CUDA path (through the C-ABI) with GraSPH2's own FP64 results and the FP64 oracle.

Bound, per value, after one computeDerivatives on float32-representable inputs:

    |x_gpu - x_ref| <= TOL * max|x_ref| + 32 * s

TOL is the north-star bound: 1e-5 for accelerations (and the other rates), 1e-6 for density. s is
the FP64 oracle's own change when the float32 inputs move by one ulp (helpers.fp32_sensitivity).
s is negligible for well-conditioned particles, so for them the plain norm-wise bound holds.
For a particle at the edge of the kernel support, the density sums a few (1-q)^3 terms; rounding
the inputs to float32 already moves that particle by far more than 1e-5. GraSPH2's own FP32 build
shows the same deviations (test_oracle.py::test_reference_fp32_close_to_fp64). Positions after
steps are compared as displacements from the start.
"""

import os

import numpy as np
import pytest

import ref_variants
from grasph2_b200 import ics
from grasph2_b200._abi import FLAG_BITS as F
from grasph2_b200.params import config0_params, config1_params, config2_params, make_options, make_params
from grasph2_b200.sim import DeviceParticleBuffer, GsphError
from grasph2_b200.state import as_dtype
from helpers import (NORM_LOG, check_within, copy_state, f32_exact, fp32_sensitivity, golden_state, rel_max,
                     vec_rel)

pytestmark = pytest.mark.gpu

TOL_ACC = 1e-5
TOL_RHO = 1e-6
TOL_RATE = 1e-5
TOL_STEP = 1e-5

GOLDEN_DIR = os.path.join(os.path.dirname(__file__), "golden")


def variant_params(name):
    return make_params(**ref_variants.params_dict(ref_variants.VARIANTS[name]))


def load_golden(name):
    return np.load(os.path.join(GOLDEN_DIR, "ref_%s.npz" % name))


def derivative_fields(params):
    f = {"acc": TOL_ACC}
    if params.flags & F["SPH"]:
        f["density"] = TOL_RHO
        f["maxvsig"] = TOL_RATE
        if params.flags & (F["SOLIDS"] | F["INTEGRATE_DENSITY"] | F["BALSARA_SWITCH"]):
            f.update(dstress_dt=TOL_RATE, density_dt=TOL_RATE, balsara=TOL_RATE)
        if params.flags & F["XSPH"]:
            f["xvel"] = TOL_RATE
    return f


def oracle_derivs(oracle, params, i0=0, i1=-1):
    def run(st):
        oracle.ts.current = oracle.ts.next = 0.0
        oracle.compute_derivatives(params, st, i0, i1)
        return st
    return run


def oracle_steps(oracle, params, nsteps):
    def run(st):
        x0 = st["pos"].copy()
        oracle.ts.current = oracle.ts.next = 0.0
        for _ in range(nsteps):
            oracle.compute_derivatives(params, st)
            oracle.integrate(params, st, True)
        st["disp"] = st["pos"] - x0
        return st
    return run


def gpu_derivatives(params, state, accum="plain", cull=True, **opt):
    with DeviceParticleBuffer(params, state["mass"].shape[0], make_options(accum=accum, cull=cull, **opt)) as pb:
        pb.upload(state)
        pb.compute_derivatives()
        return pb.download()


def check_derivatives(got, want, sens, params, what, rows=slice(None)):
    for k, tol in derivative_fields(params).items():
        check_within(got[k][rows], want[k][rows], sens[k][rows], tol, "%s %s" % (what, k))


@pytest.mark.parametrize("cull", [True, False], ids=["culled", "allpairs"])
@pytest.mark.parametrize("accum", ["plain", "compensated"])
@pytest.mark.parametrize("name", list(ref_variants.VARIANTS))
def test_golden_derivatives(oracle, name, accum, cull):
    """computeDerivatives vs the reference's own FP64 results (tests/golden)."""
    z = load_golden(name)
    p = variant_params(name)
    st = golden_state(z, "in_")
    _, sens = fp32_sensitivity(oracle_derivs(oracle, p), st)
    got = gpu_derivatives(p, st, accum, cull)
    check_derivatives(got, golden_state(z, "d64_"), sens, p, "%s/%s/cull=%s" % (name, accum, cull))


@pytest.mark.parametrize("accum", ["plain", "compensated"])
@pytest.mark.parametrize("name", list(ref_variants.VARIANTS))
def test_golden_three_steps(oracle, name, accum):
    """3 x {computeDerivatives; integrate(notFirstStep=true)} vs the reference's FP64 run."""
    z = load_golden(name)
    p = variant_params(name)
    st = golden_state(z, "in_")
    _, sens = fp32_sensitivity(oracle_steps(oracle, p, 3), st)
    with DeviceParticleBuffer(p, st["mass"].shape[0], make_options(accum=accum)) as pb:
        pb.upload(st)
        dts = []
        for _ in range(3):
            pb.compute_derivatives()
            pb.integrate(True)
            dts.append(pb.current_timestep())
        got = pb.download()
        pos64 = pb.download_pos64()
    ref = golden_state(z, "s64_")
    what = "%s/%s 3 steps" % (name, accum)
    check_within(pos64 - st["pos"], ref["pos"] - st["pos"], sens["disp"], TOL_STEP, what + " displacement")
    for k in ("vel", "density", "dstress"):
        check_within(got[k], ref[k], sens[k], TOL_STEP, what + " " + k)
    np.testing.assert_allclose(dts, z["dt64"], rtol=1e-6)


def _edge_state(name, n, seed):
    v = ref_variants.VARIANTS[name]
    rng = np.random.default_rng(seed)
    st = ics.uniform_sphere(n, radius=1.0, rho0=v["rho0"], omega=(0.0, 0.0, 0.3), seed=seed)
    st["vel"] += 0.02 * rng.normal(size=(n, 3))
    st["density"][:] = v["rho0"] * (1 + 0.02 * rng.normal(size=n))
    S = rng.normal(size=(n, 3, 3)) * 0.05
    st["dstress"][:] = 0.5 * (S + S.transpose(0, 2, 1))
    return f32_exact(st)


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 127, 128, 129, 255, 256, 257, 1000, 1023, 1025, 3000])
@pytest.mark.parametrize("name", ["nbody", "fluid", "solid", "solid_mc", "fluid_full"])
def test_edge_sizes_vs_oracle(oracle, name, n):
    """Every N works (the reference's tile loop needs N % 256 == 0, algorithms.h:285-301), with and
    without the chunk culling (chunks of 64, groups of 128)."""
    p = variant_params(name)
    st = _edge_state(name, n, seed=n)
    ref, sens = fp32_sensitivity(oracle_derivs(oracle, p), st)
    for cull in (True, False):
        got = gpu_derivatives(p, st, cull=cull)
        check_derivatives(got, ref, sens, p, "%s/n=%d/cull=%s" % (name, n, cull))


@pytest.mark.parametrize("opt", [
    dict(j_split=1), dict(j_split=3), dict(j_split=7), dict(j_tile=64), dict(j_tile=1024),
    dict(threads=64), dict(threads=256), dict(i_per_thread=1), dict(i_per_thread=2), dict(i_per_thread=8),
    dict(j_tile=512, threads=256, j_split=5),
])
@pytest.mark.parametrize("name", ["nbody", "solid"])
def test_launch_shapes_vs_oracle(oracle, name, opt):
    p = variant_params(name)
    st = _edge_state(name, 2500, seed=11)
    ref, sens = fp32_sensitivity(oracle_derivs(oracle, p), st)
    for accum in ("plain", "compensated"):
        for cull in (True, False):
            got = gpu_derivatives(p, st, accum, cull, **opt)
            check_derivatives(got, ref, sens, p, "%s/%s/%s/cull=%s" % (name, opt, accum, cull))


def test_config0_one_step_vs_oracle(oracle):
    """SPH + gravity fluid sphere, N=4096 (eps=0.02 != h=0.15): derivatives, then one full step."""
    p = config0_params()
    st = f32_exact(ics.uniform_sphere(4096, radius=1.0, rho0=0.239, omega=(0, 0, 0.1), seed=20261203))
    d_ref, d_sens = fp32_sensitivity(oracle_derivs(oracle, p), st)
    s_ref, s_sens = fp32_sensitivity(oracle_steps(oracle, p, 1), st)
    with DeviceParticleBuffer(p, 4096) as pb:
        pb.upload(st)
        pb.compute_derivatives()
        got_d = pb.download()
        pb.integrate(True)
        got = pb.download()
        pos64 = pb.download_pos64()
    check_derivatives(got_d, d_ref, d_sens, p, "config0")
    check_within(pos64 - st["pos"], s_ref["disp"], s_sens["disp"], TOL_STEP, "config0 displacement")
    check_within(got["vel"], s_ref["vel"], s_sens["vel"], TOL_STEP, "config0 vel")


@pytest.mark.slow
def test_config1_subsample_vs_oracle(oracle):
    """Elastic-plastic impact at full size N=65536; oracle rows on two target windows."""
    p = config1_params()
    st = ics.two_sphere_impact(seed=20261204)
    rng = np.random.default_rng(5)
    S = rng.normal(size=(st["mass"].shape[0], 3, 3)) * 0.05
    st["dstress"][:] = 0.5 * (S + S.transpose(0, 2, 1))
    st = f32_exact(st)
    with DeviceParticleBuffer(p, 65536) as pb:
        pb.upload(st)
        pb.compute_derivatives()
        got = pb.download()
    for i0, i1 in ((0, 256), (65536 - 256, 65536)):
        ref, sens = fp32_sensitivity(oracle_derivs(oracle, p, i0, i1), st, trials=1)
        check_derivatives(got, ref, sens, p, "config1[%d:%d]" % (i0, i1), rows=slice(i0, i1))
        check_within(got["density"], ref["density"], sens["density"], TOL_RHO, "config1 density (all)")


@pytest.mark.slow
def test_config2_gravity_subsample_vs_oracle(oracle):
    """Plummer sphere N=1,048,576: accelerations of a seeded 16,384-particle target subsample vs FP64
    (all N sources); both the plain and the compensated FP32 forms are held to the 1e-5 norm-wise bound
    and their errors are logged."""
    p = config2_params()
    st = f32_exact(ics.plummer_sphere(1 << 20, seed=20261205))
    idx = np.random.default_rng(1).choice(1 << 20, 16384, replace=False)
    ref = oracle.gravity_targets(p, st["pos"], st["mass"], idx)
    for accum in ("plain", "compensated"):
        got = gpu_derivatives(p, st, accum)
        e = rel_max(got["acc"][idx], ref)
        v = vec_rel(got["acc"][idx], ref)
        NORM_LOG.append("config2 Plummer N=2^20 %-11s acc: max|da|/max|a| %.3e, max_i |da_i|/rms|a| %.3e "
                        "(16384 targets)" % (accum, e, v))
        assert e <= TOL_ACC, "config2 %s: %.3e > %.1e" % (accum, e, TOL_ACC)


def test_graph_step_matches_eager():
    p = variant_params("solid_mc")
    st = _edge_state("solid_mc", 3000, seed=3)
    with DeviceParticleBuffer(p, 3000) as a, DeviceParticleBuffer(p, 3000) as b:
        a.upload(st)
        b.upload(st)
        for _ in range(4):
            a.compute_derivatives()
            a.integrate(True)
        b.step(4)
        x, y = a.download(), b.download()
        assert a.current_timestep() == b.current_timestep()
    for k in x:
        np.testing.assert_array_equal(x[k], y[k], err_msg=k)


def test_deterministic():
    p = variant_params("solid")
    st = _edge_state("solid", 5000, seed=4)
    r1 = gpu_derivatives(p, st)
    r2 = gpu_derivatives(p, st)
    for k in r1:
        np.testing.assert_array_equal(r1[k], r2[k], err_msg=k)


def test_momentum_conservation_gpu():
    p = make_params(switches=("SELF_GRAVITY", "SPH", "SOLIDS", "ARTIFICIAL_VISCOSITY", "INTEGRATE_DENSITY"),
                    H=0.3, rho0=1.0, bulk=10.0, soundspeed=3.0, shear=5.0)
    st = _edge_state("solid", 3000, seed=9)
    for accum in ("plain", "compensated"):
        got = gpu_derivatives(p, st, accum)
        f = st["mass"][:, None] * got["acc"].astype(np.float64)
        assert np.abs(f.sum(0)).max() < 1e-5 * np.abs(f).sum(0).max()


@pytest.mark.parametrize("name", ["solid", "fluid", "nbody"])
def test_diagnostics_vs_oracle(oracle, name):
    p = variant_params(name)
    st = _edge_state(name, 3000, seed=8)
    ref = copy_state(st)
    oracle.compute_derivatives(p, ref)
    with DeviceParticleBuffer(p, 3000) as pb:
        pb.upload(st)
        pb.compute_derivatives()
        d = pb.diagnostics(half_kick=0.5e-3)
    o = oracle.diagnostics(p, ref, half_kick=0.5e-3)
    for k in ("e_grav", "mass"):
        assert abs(d[k] - o[k]) <= 1e-9 * max(abs(o[k]), 1e-30), (k, d[k], o[k])
    for k in ("e_kin", "e_int", "e_shear"):  # these read the FP32 rates / densities of the device
        assert abs(d[k] - o[k]) <= 1e-5 * max(abs(o[k]), abs(o["e_kin"]), 1e-30), (k, d[k], o[k])
    for k in ("momentum", "ang_mom"):
        scale = abs(o["e_kin"]) ** 0.5 + 1e-12
        assert np.abs(np.array(d[k]) - np.array(o[k])).max() < 1e-5 * scale, k


def test_error_paths_on_device():
    p = variant_params("fluid")
    st = _edge_state("fluid", 100, seed=1)
    with DeviceParticleBuffer(p, 100, make_options(check_finite=1)) as pb:
        pb.upload(st)
        with pytest.raises(ValueError):
            pb.upload({"pos": st["pos"][:50]})
        bad = as_dtype(st, np.float32)
        bad["vel"][7, 1] = np.nan
        with pytest.raises(GsphError) as e:
            pb.upload(bad)
        assert e.value.code == -5
        pb.upload(st)  # the scan reports once, then the context is usable again
        pb.compute_derivatives()
        pb.download()
        lib = pb.lib
        assert lib.gsph_upload(pb.handle, 1 << 20, None, None) == -1
        from grasph2_b200._abi import GsphHostParticles
        import ctypes
        hp = GsphHostParticles()
        assert lib.gsph_upload(pb.handle, 1, ctypes.byref(hp), None) == -1
        assert b"NULL" in lib.gsph_last_error(pb.handle)


def test_profile_and_launch_count():
    p = variant_params("solid")
    st = _edge_state("solid", 2000, seed=2)
    with DeviceParticleBuffer(p, 2000) as pb:
        pb.upload(st)
        pb.profile_enable(True)
        c0 = pb.launch_count()
        pb.step(1)
        pb.profile_collect()
        pr = pb.profile_read()
        # gravity + the FP64 fold of its partials (side stream), chunk bounds + lists + work items,
        # density + finish, SPH pass + finish, leapfrog
        assert pb.launch_count() - c0 == 10
        assert pr["pairs"][1] == 1 and pr["pairs"][0] > 0 and pr["density"][1] == 1 and pr["gravity"][1] == 1
        assert pr["step"][0] >= pr["pairs"][0] + pr["gravity"][0]


def test_device_order_is_invisible():
    """The curve order on the device never shows: every transfer is in the caller's order."""
    p = variant_params("solid_mc")
    st = _edge_state("solid_mc", 3001, seed=21)
    with DeviceParticleBuffer(p, 3001) as pb:
        pb.upload(st)
        back = pb.download()
        for k in ("pos", "mass", "vel", "density", "dstress"):
            np.testing.assert_array_equal(back[k], st[k].astype(np.float32), err_msg=k)
        np.testing.assert_array_equal(pb.download_pos64(), st["pos"])
        pb.lib.gsph_reorder(pb.handle, None)
        np.testing.assert_array_equal(pb.download()["vel"], st["vel"].astype(np.float32))


def test_periodic_resort_matches(oracle):
    """Re-sorting during a run changes only the summation order."""
    p = variant_params("solid")
    st = _edge_state("solid", 2000, seed=22)
    out = []
    for interval in (0, 1):
        with DeviceParticleBuffer(p, 2000, make_options(resort_interval=interval)) as pb:
            pb.upload(st)
            pb.step(3)
            out.append(pb.download())
    _, sens = fp32_sensitivity(oracle_steps(oracle, p, 3), st)
    check_within(out[1]["vel"], out[0]["vel"], sens["vel"], TOL_STEP, "resorted vel")


@pytest.mark.parametrize("accum", ["plain", "compensated"])
@pytest.mark.parametrize("name,cull", [("solid", True), ("solid", False), ("nbody", True), ("fluid", True)])
def test_autotune_keeps_results(oracle, name, cull, accum):
    """The autotuner only changes launch shapes: results stay within the parity bound, and stepping
    re-captures the step graph with the tuned shapes."""
    p = variant_params(name)
    st = _edge_state(name, 3000, seed=31)
    ref, sens = fp32_sensitivity(oracle_derivs(oracle, p), st)
    with DeviceParticleBuffer(p, 3000, make_options(cull=cull, accum=accum)) as pb:
        pb.upload(st)
        shape = pb.autotune(2)
        assert shape["grav_ipt"] in (1, 2, 4, 8) and shape["cull"] == int(cull and bool(p.flags & F["SPH"]))
        pb.compute_derivatives()
        got = pb.download()
        pb.step(2)
        pb.download()
    check_derivatives(got, ref, sens, p, "%s autotuned cull=%s %s" % (name, cull, accum))
