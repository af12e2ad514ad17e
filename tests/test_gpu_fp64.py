"""Double-precision mode (the reference's DOUBLE_PRECISION switch, settings/precisionSettings.h:16-17)
against GraSPH2's own FP64 build (tests/golden) and the FP64 oracle.

Both sides compute in double; they differ only in summation order and in the rounding of the few
library functions (sqrt, pow), so the bound is a norm-wise FP64 one: TOL64 = 1e-11 of the field's
largest value for derivatives, TOL64_STEP after three steps.
"""

import os

import numpy as np
import pytest

import ref_variants
from grasph2_b200 import ics
from grasph2_b200._abi import FLAG_BITS as F
from grasph2_b200.params import make_options, make_params
from grasph2_b200.sim import DeviceParticleBuffer
from grasph2_b200.state import copy_state
from helpers import golden_state, rel_max

pytestmark = pytest.mark.gpu

TOL64 = 1e-11
TOL64_STEP = 1e-10
GOLDEN_DIR = os.path.join(os.path.dirname(__file__), "golden")


def variant_params(name):
    return make_params(**ref_variants.params_dict(ref_variants.VARIANTS[name]))


def fields(params):
    f = ["acc"]
    if params.flags & F["SPH"]:
        f += ["density", "maxvsig"]
        if params.flags & (F["SOLIDS"] | F["INTEGRATE_DENSITY"] | F["BALSARA_SWITCH"]):
            f += ["dstress_dt", "density_dt", "balsara"]
        if params.flags & F["XSPH"]:
            f.append("xvel")
    return f


def fp64_options(**kw):
    return make_options(precision="double", **kw)


def check64(got, want, names, tol, what):
    for k in names:
        e = rel_max(got[k], want[k])
        assert e <= tol, "%s %s: %.3e > %.1e" % (what, k, e, tol)


@pytest.mark.parametrize("name", list(ref_variants.VARIANTS))
def test_fp64_golden_derivatives(name):
    z = np.load(os.path.join(GOLDEN_DIR, "ref_%s.npz" % name))
    p = variant_params(name)
    st = golden_state(z, "in_")
    with DeviceParticleBuffer(p, st["mass"].shape[0], fp64_options()) as pb:
        pb.upload_f64(st)
        pb.compute_derivatives()
        got = pb.download_f64()
    check64(got, golden_state(z, "d64_"), fields(p), TOL64, "%s fp64" % name)


@pytest.mark.parametrize("name", list(ref_variants.VARIANTS))
def test_fp64_golden_three_steps(name):
    """3 x {computeDerivatives; integrate} vs the reference's FP64 run, time steps included."""
    z = np.load(os.path.join(GOLDEN_DIR, "ref_%s.npz" % name))
    p = variant_params(name)
    st = golden_state(z, "in_")
    with DeviceParticleBuffer(p, st["mass"].shape[0], fp64_options()) as pb:
        pb.upload_f64(st)
        dts = []
        for _ in range(3):
            pb.compute_derivatives()
            pb.integrate(True)
            dts.append(pb.current_timestep())
        got = pb.download_f64()
    ref = golden_state(z, "s64_")
    e = rel_max(got["pos"] - st["pos"], ref["pos"] - st["pos"])
    assert e <= TOL64_STEP, "%s displacement %.3e" % (name, e)
    check64(got, ref, [k for k in ("vel", "density", "dstress") if np.abs(ref[k]).max() > 0], TOL64_STEP,
            "%s 3 steps" % name)
    np.testing.assert_allclose(dts, z["dt64"], rtol=1e-12)


@pytest.mark.parametrize("n", [1, 2, 127, 128, 129, 1000, 1025])
@pytest.mark.parametrize("name", ["nbody", "solid_mc", "fluid_full"])
def test_fp64_edge_sizes_vs_oracle(oracle, name, n):
    v = ref_variants.VARIANTS[name]
    p = variant_params(name)
    rng = np.random.default_rng(n)
    st = ics.uniform_sphere(n, radius=1.0, rho0=v["rho0"], omega=(0.0, 0.0, 0.3), seed=n)
    st["vel"] += 0.02 * rng.normal(size=(n, 3))
    st["density"][:] = v["rho0"] * (1 + 0.02 * rng.normal(size=n))
    S = rng.normal(size=(n, 3, 3)) * 0.05
    st["dstress"][:] = 0.5 * (S + S.transpose(0, 2, 1))
    ref = copy_state(st)
    oracle.ts.current = oracle.ts.next = 0.0
    oracle.compute_derivatives(p, ref)
    with DeviceParticleBuffer(p, n, fp64_options()) as pb:
        pb.upload_f64(st)
        pb.compute_derivatives()
        got = pb.download_f64()
    check64(got, ref, [k for k in fields(p) if np.abs(ref[k]).max() > 0], TOL64, "%s n=%d" % (name, n))


def test_fp64_graph_step_matches_eager():
    p = variant_params("solid_mc")
    st = ics.uniform_sphere(2000, radius=1.0, rho0=1.0, omega=(0, 0, 0.3), seed=5)
    with DeviceParticleBuffer(p, 2000, fp64_options()) as a, DeviceParticleBuffer(p, 2000, fp64_options()) as b:
        a.upload_f64(st)
        b.upload_f64(st)
        for _ in range(4):
            a.compute_derivatives()
            a.integrate(True)
        b.step(4)
        x, y = a.download_f64(), b.download_f64()
        assert a.current_timestep() == b.current_timestep()
    for k in x:
        np.testing.assert_array_equal(x[k], y[k], err_msg=k)


@pytest.mark.parametrize("name", ["solid", "nbody"])
def test_fp64_diagnostics_vs_oracle(oracle, name):
    p = variant_params(name)
    st = ics.uniform_sphere(1500, radius=1.0, rho0=1.0, omega=(0, 0, 0.3), seed=6)
    ref = copy_state(st)
    oracle.ts.current = oracle.ts.next = 0.0
    oracle.compute_derivatives(p, ref)
    o = oracle.diagnostics(p, ref, half_kick=0.5e-3)
    with DeviceParticleBuffer(p, 1500, fp64_options()) as pb:
        pb.upload_f64(st)
        pb.compute_derivatives()
        d = pb.diagnostics(half_kick=0.5e-3)
    scale = abs(o["e_kin"]) + abs(o["e_grav"]) + abs(o["e_int"]) + abs(o["e_shear"])
    for k in ("e_kin", "e_grav", "e_int", "e_shear", "mass"):
        assert abs(d[k] - o[k]) <= 1e-11 * max(scale, abs(o[k])), (k, d[k], o[k])
    for k in ("momentum", "ang_mom"):
        assert np.abs(np.array(d[k]) - np.array(o[k])).max() <= 1e-11 * (scale ** 0.5 + 1e-12), k


def test_single_precision_f64_transfers_round():
    """In single precision the double transfers round to float32 and widen back exactly."""
    p = variant_params("solid")
    st = ics.uniform_sphere(777, radius=1.0, rho0=1.0, omega=(0, 0, 0.3), seed=8)
    with DeviceParticleBuffer(p, 777) as pb:
        pb.upload_f64(st)
        back = pb.download_f64(["mass", "vel", "density", "dstress"])
        for k in back:
            np.testing.assert_array_equal(back[k], st[k].astype(np.float32).astype(np.float64), err_msg=k)
        np.testing.assert_array_equal(pb.download_f64(["pos"])["pos"], st["pos"])
