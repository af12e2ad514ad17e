"""Parity with GraSPH2's own CUDA path on the same GPU.

oracle/_ref/libref_cuda_<variant>.so is the reference's computeDerivatives (its three jobs run by its
tile kernel do_for_each_pair_fast_impl, src/particles/algorithms.h:270-309) and integrate
(src/integration.h:219-244), compiled unchanged for sm_100a against a stand-in for mpUtils and the
particle engine (oracle/ref_cuda_driver.cu). It is FP32, as the reference ships.

Its tile loop is only correct for N a multiple of its 256-thread block (algorithms.h:285-301), so every
case here has N % 256 == 0; the product is correct for every N (test_gpu_parity.py's edge sizes).

Bound, per value: |x_product - x_reference_cuda| <= TOL * max|x_reference_cuda| + 32 * s, with s the
FP64 oracle's change under one-ulp input perturbations (helpers.fp32_sensitivity): both sides are FP32
with different summation orders, so particles whose results input rounding alone moves by more than
TOL get that slack, as in the FP64 comparisons.
"""

import os

import numpy as np
import pytest

import pyoracle
import ref_variants
from grasph2_b200 import ics
from grasph2_b200.params import make_options, make_params
from grasph2_b200.sim import DeviceParticleBuffer
from helpers import NORM_LOG, check_within, f32_exact, fp32_sensitivity, golden_state, rel_max

pytestmark = pytest.mark.gpu

TOL_ACC = 1e-5
TOL_RHO = 1e-6
TOL_RATE = 1e-5
TOL_STEP = 1e-5
GOLDEN_DIR = os.path.join(os.path.dirname(__file__), "golden")
VARIANTS = [v for v in ref_variants.VARIANTS if pyoracle.ref_cuda_available(v)]

if not VARIANTS:
    pytest.skip("the reference's CUDA build (oracle/_ref/libref_cuda_*.so) is not built", allow_module_level=True)


def variant_params(name):
    return make_params(**ref_variants.params_dict(ref_variants.VARIANTS[name]))


def fields(params):
    from grasph2_b200._abi import FLAG_BITS as F
    f = {"acc": TOL_ACC}
    if params.flags & F["SPH"]:
        f["density"] = TOL_RHO
        if params.flags & (F["SOLIDS"] | F["INTEGRATE_DENSITY"] | F["BALSARA_SWITCH"]):
            f.update(dstress_dt=TOL_RATE, density_dt=TOL_RATE)
        if params.flags & F["BALSARA_SWITCH"]:
            f.update(balsara=TOL_RATE, maxvsig=TOL_RATE)
        if params.flags & F["XSPH"]:
            f["xvel"] = TOL_RATE
    return f


def oracle_derivs(oracle, params, i0=0, i1=-1):
    def run(st):
        oracle.ts.current = oracle.ts.next = 0.0
        oracle.compute_derivatives(params, st, i0, i1)
        return st
    return run


def ref_cuda_derivatives(name, st):
    with pyoracle.RefCuda(name, st["mass"].shape[0]) as r:
        r.upload(st)
        r.compute_derivatives()
        return {k: v.astype(np.float64) for k, v in r.download().items()}


def product_derivatives(params, st, accum="plain"):
    with DeviceParticleBuffer(params, st["mass"].shape[0], make_options(accum=accum)) as pb:
        pb.upload(st)
        pb.compute_derivatives()
        return pb.download()


@pytest.mark.parametrize("name", VARIANTS)
def test_reference_cuda_meets_the_bound_against_its_fp64_build(oracle, name):
    """The checker itself: GraSPH2's CUDA path vs GraSPH2's FP64 host build (tests/golden, N = 256)."""
    z = np.load(os.path.join(GOLDEN_DIR, "ref_%s.npz" % name))
    p = variant_params(name)
    st = golden_state(z, "in_")
    _, sens = fp32_sensitivity(oracle_derivs(oracle, p), st)
    got = ref_cuda_derivatives(name, st)
    want = golden_state(z, "d64_")
    for k, tol in fields(p).items():
        check_within(got[k], want[k], sens[k], tol, "reference CUDA %s %s" % (name, k))


@pytest.mark.parametrize("accum", ["plain", "compensated"])
@pytest.mark.parametrize("name", VARIANTS)
def test_product_matches_reference_cuda_derivatives(oracle, name, accum):
    z = np.load(os.path.join(GOLDEN_DIR, "ref_%s.npz" % name))
    p = variant_params(name)
    st = golden_state(z, "in_")
    _, sens = fp32_sensitivity(oracle_derivs(oracle, p), st)
    want = ref_cuda_derivatives(name, st)
    got = product_derivatives(p, st, accum)
    for k, tol in fields(p).items():
        check_within(got[k], want[k], sens[k], tol, "vs reference CUDA %s/%s %s" % (name, accum, k))


@pytest.mark.parametrize("name", VARIANTS)
def test_product_matches_reference_cuda_three_steps(oracle, name):
    """3 x {computeDerivatives; integrate(notFirstStep=true)} on both paths, from the same state; the
    variable-step variants compare their time steps too (dt on the device in both)."""
    z = np.load(os.path.join(GOLDEN_DIR, "ref_%s.npz" % name))
    p = variant_params(name)
    st = golden_state(z, "in_")
    n = st["mass"].shape[0]

    def oracle_steps(s):
        x0 = s["pos"].copy()
        oracle.ts.current = oracle.ts.next = 0.0
        for _ in range(3):
            oracle.compute_derivatives(p, s)
            oracle.integrate(p, s, True)
        s["disp"] = s["pos"] - x0
        return s
    _, sens = fp32_sensitivity(oracle_steps, st)
    with pyoracle.RefCuda(name, n) as r:
        r.upload(st)
        r.set_timestep(0.0, 0.0)  # a fresh run, as the reference's process starts
        dts_r = []
        for _ in range(3):
            r.compute_derivatives()
            r.integrate(True)
            dts_r.append(r.current_timestep())
        want = {k: v.astype(np.float64) for k, v in r.download().items()}
    with DeviceParticleBuffer(p, n) as pb:
        pb.upload(st)
        dts = []
        for _ in range(3):
            pb.compute_derivatives()
            pb.integrate(True)
            dts.append(pb.current_timestep())
        got = pb.download()
        pos64 = pb.download_pos64()
    what = "vs reference CUDA %s 3 steps" % name
    # the reference's positions are FP32 (x += v dt rounded to float each step); ours keep an FP64
    # master: compare displacements, allowing the reference's own rounding of x (half an ulp of |x| per
    # step, three steps) on top of the bound
    disp_ref = want["pos"] - st["pos"]
    x_round = 3 * 0.5 * np.abs(want["pos"]) * 2.0 ** -23
    check_within(pos64 - st["pos"], disp_ref, sens["disp"], TOL_STEP, what + " displacement", extra=x_round)
    for k in ("vel", "density", "dstress"):
        check_within(got[k], want[k], sens[k], TOL_STEP, what + " " + k)
    np.testing.assert_allclose(dts, dts_r, rtol=1e-5)


def test_product_matches_reference_cuda_fluid_n4096(oracle):
    """The config-0 size (N = 4096) in the fluid physics the reference can express (eps == h)."""
    name = "fluid"
    p = variant_params(name)
    st = f32_exact(ics.uniform_sphere(4096, radius=1.0, rho0=0.239, omega=(0, 0, 0.1), seed=20261203))
    _, sens = fp32_sensitivity(oracle_derivs(oracle, p), st, trials=1)
    want = ref_cuda_derivatives(name, st)
    got = product_derivatives(p, st)
    errs = []
    for k, tol in fields(p).items():
        errs.append("%s %.2e" % (k, check_within(got[k], want[k], sens[k], tol, "vs reference CUDA fluid N=4096 " + k)))
    NORM_LOG.append("fluid N=4096 plain vs the reference's CUDA path (norm-wise): " + ", ".join(errs))


@pytest.mark.slow
def test_product_matches_reference_cuda_impact_n65536(oracle):
    """The impact at full size (N = 65536) in the physics the reference can express (eps == h, AV signal
    coefficient 3), on two 256-row windows (first and last rows) with the FP64 oracle on the same rows:
    the product meets the condition-aware bound against FP64; against the reference's CUDA path the
    bound is widened by that path's own deviation from FP64 (both are FP32 with different summation
    orders, so where the reference's rounding error exceeds the tolerance the two cannot agree closer)."""
    name = "impact"
    p = variant_params(name)
    st = ics.two_sphere_impact(seed=20261204)
    rng = np.random.default_rng(5)
    S = rng.normal(size=(65536, 3, 3)) * 0.05
    st["dstress"][:] = 0.5 * (S + S.transpose(0, 2, 1))
    st = f32_exact(st)
    want = ref_cuda_derivatives(name, st)
    got = product_derivatives(p, st)
    errs = []
    for i0, i1 in ((0, 256), (65536 - 256, 65536)):
        ref, sens = fp32_sensitivity(oracle_derivs(oracle, p, i0, i1), st, trials=1)
        for k, tol in fields(p).items():
            r = ref[k][i0:i1]
            e_got = check_within(got[k][i0:i1], r, sens[k][i0:i1], tol, "impact[%d:%d] %s vs FP64" % (i0, i1, k))
            ref_dev = np.abs(want[k][i0:i1] - r)
            e_ref = float(ref_dev.max() / np.abs(r).max()) if np.abs(r).max() > 0 else float(ref_dev.max())
            check_within(got[k][i0:i1], want[k][i0:i1], sens[k][i0:i1], tol,
                         "vs reference CUDA impact[%d:%d] %s" % (i0, i1, k), extra=ref_dev)
            errs.append("%s[%d:%d] ours %.2e, reference CUDA %.2e" % (k, i0, i1, e_got, e_ref))
    NORM_LOG.append("impact N=65536 (reference physics) vs FP64, norm-wise: " + "; ".join(errs))


@pytest.mark.slow
def test_product_matches_reference_cuda_plummer_n262144(oracle):
    """Softened N-body at N = 262,144 (eps = 0.01 == h): the product and the reference's CUDA path, each
    against FP64 on 2048 targets. The product meets 1e-5; the reference's single running FP32 sum per
    particle does not at this size, so the two agree to within the reference's own error plus 1e-5."""
    name = "plummer"
    p = variant_params(name)
    st = f32_exact(ics.plummer_sphere(1 << 18, seed=20261205))
    idx = np.random.default_rng(3).choice(1 << 18, 2048, replace=False)
    ref = oracle.gravity_targets(p, st["pos"], st["mass"], idx)
    want = ref_cuda_derivatives(name, st)
    got = product_derivatives(p, st)
    e_ref = rel_max(want["acc"][idx], ref)
    e_got = rel_max(got["acc"][idx], ref)
    e_pair = rel_max(got["acc"][idx], want["acc"][idx])
    NORM_LOG.append("Plummer N=2^18 vs FP64 (2048 targets): the reference's CUDA path %.2e, the product %.2e; "
                    "product vs reference CUDA %.2e" % (e_ref, e_got, e_pair))
    assert e_got <= TOL_ACC
    assert e_pair <= e_ref + TOL_ACC
