"""The symmetric all-pairs gravity kernel (each unordered pair once, applied to both particles):
accelerations against the FP64 oracle and against the one-sided kernel, over one task (a single block),
a few groups, ragged last groups, unsoftened gravity, compensated accumulation and the culled SPH path."""

import numpy as np
import pytest

from grasph2_b200 import ics
from grasph2_b200.params import make_options, make_params
from grasph2_b200.sim import DeviceParticleBuffer
from helpers import f32_exact

pytestmark = pytest.mark.gpu


def nbody(eps):
    return make_params(switches=("SELF_GRAVITY",), H=0.05, grav_eps=eps, fixed_dt=1e-3)


def accel(p, st, **opt):
    with DeviceParticleBuffer(p, st["mass"].shape[0], make_options(**opt)) as pb:
        pb.upload(st)
        pb.compute_derivatives()
        shape = pb.launch_shape()
        return pb.download()["acc"].astype(np.float64), shape


def per_target(got, ref):
    """max over targets of |a - a_ref| / (|a_ref| + 1e-3 max |a_ref|)."""
    d = np.linalg.norm(got - ref, axis=1)
    r = np.linalg.norm(ref, axis=1)
    return float((d / (r + 1e-3 * r.max())).max())


@pytest.mark.parametrize("accum,tol", [("plain", 2e-5), ("compensated", 2e-6)])
@pytest.mark.parametrize("n,groups", [(1000, 0), (3000, 0), (20000, 0), (70000, 20), (70000, 0)])
def test_symmetric_vs_oracle(oracle, n, groups, accum, tol):
    p = nbody(0.01)
    st = f32_exact(ics.plummer_sphere(n, seed=100 + n))
    idx = np.unique(np.concatenate([np.arange(min(n, 64)), np.random.default_rng(n).choice(n, 512), [n - 1]]))
    ref = oracle.gravity_targets(p, st["pos"], st["mass"], idx)
    got, shape = accel(p, st, accum=accum, gravity="symmetric", gravity_groups=groups)
    assert shape["grav_sym_groups"] > 0
    assert per_target(got[idx], ref) <= tol
    one, shape1 = accel(p, st, accum=accum, gravity="one-sided")
    assert shape1["grav_sym_groups"] == 0
    assert per_target(got, one) <= tol


def test_symmetric_unsoftened(oracle):
    p = nbody(0.0)
    st = f32_exact(ics.plummer_sphere(30000, seed=7))
    idx = np.random.default_rng(2).choice(30000, 512, replace=False)
    ref = oracle.gravity_targets(p, st["pos"], st["mass"], idx)
    got, _ = accel(p, st, gravity="symmetric")
    assert np.isfinite(got).all()
    assert per_target(got[idx], ref) <= 2e-5


def test_symmetric_deterministic_and_momentum():
    p = nbody(0.01)
    st = f32_exact(ics.plummer_sphere(50000, seed=3))
    a1, _ = accel(p, st, gravity="symmetric")
    a2, _ = accel(p, st, gravity="symmetric")
    np.testing.assert_array_equal(a1, a2)
    f = st["mass"][:, None] * a1
    assert np.abs(f.sum(0)).max() < 1e-5 * np.abs(f).sum(0).max()


@pytest.mark.parametrize("accum", ["plain", "compensated"])
def test_symmetric_in_the_culled_sph_path(accum):
    """An SPH + gravity context whose separate gravity kernel is the symmetric one: same derivatives as
    with the one-sided kernel to rounding."""
    p = make_params(switches=("SELF_GRAVITY", "SPH", "SOLIDS", "ARTIFICIAL_VISCOSITY", "PLASTICITY_MIESE"),
                    H=0.08, grav_eps=0.01, rho0=1.0, bulk=10.0, dbulk_dp=1.0, soundspeed=10 ** 0.5, shear=5.0,
                    Y=0.5, av_alpha=1.0, av_beta=2.0, fixed_dt=1e-4)
    st = f32_exact(ics.two_sphere_impact(26000, 3250, v_rel=0.5, y_offset=0.3, seed=5))
    n = 29250
    out = {}
    for form in ("symmetric", "one-sided"):
        with DeviceParticleBuffer(p, n, make_options(accum=accum, gravity=form)) as pb:
            pb.upload(st)
            pb.compute_derivatives()
            assert (pb.launch_shape()["grav_sym_groups"] > 0) == (form == "symmetric")
            out[form] = pb.download()
    a, b = out["symmetric"]["acc"].astype(np.float64), out["one-sided"]["acc"].astype(np.float64)
    assert per_target(a, b) <= (2e-5 if accum == "plain" else 2e-6)
    for k in ("density", "dstress_dt", "density_dt"):
        np.testing.assert_array_equal(out["symmetric"][k], out["one-sided"][k], err_msg=k)


def test_autotune_may_pick_either_form():
    p = nbody(0.01)
    st = f32_exact(ics.plummer_sphere(40000, seed=4))
    ref, _ = accel(p, st, gravity="one-sided")
    with DeviceParticleBuffer(p, 40000) as pb:
        pb.upload(st)
        shape = pb.autotune(2)
        pb.compute_derivatives()
        got = pb.download()["acc"].astype(np.float64)
    assert shape["grav_sym_groups"] >= 0
    assert per_target(got, ref) <= 2e-5
