"""Host-side logic: parameter sets, the named workloads and the seeded initial conditions."""

import math

import numpy as np
import pytest

from grasph2_b200 import ics
from grasph2_b200._abi import FLAG_BITS
from grasph2_b200.params import (config0_params, config1_params, config2_params, impact_smoothing_length,
                                 make_params, params_to_dict)


def test_make_params_switches_and_defaults():
    p = make_params(switches=("SELF_GRAVITY", "SPH"), H=0.2)
    assert p.flags == FLAG_BITS["SELF_GRAVITY"] | FLAG_BITS["SPH"]
    assert p.grav_eps == 0.2  # the reference softens with H
    assert abs(p.normalsep - 0.06) < 1e-15
    d = params_to_dict(p)
    assert d["switches"] == ("SELF_GRAVITY", "SPH") and d["H"] == 0.2
    with pytest.raises(KeyError):
        make_params(switches=("NOPE",))
    with pytest.raises(KeyError):
        make_params(bogus=1)


def test_workload_parameters():
    p0 = config0_params()
    assert p0.H == 0.15 and p0.grav_eps == 0.02 and p0.soundspeed == 1.0 and p0.rho0 == 0.239
    assert not p0.flags & FLAG_BITS["ARTIFICIAL_VISCOSITY"]
    p1 = config1_params()
    assert abs(p1.H - 0.10396) < 1e-4  # 2.5 x (V/N)^(1/3) of the two-sphere impact
    assert p1.av_beta == 2.0 and p1.grav_eps == 0.01 and p1.fixed_dt == 1e-4
    assert abs(impact_smoothing_length() - p1.H) < 1e-15
    p2 = config2_params()
    assert p2.flags == FLAG_BITS["SELF_GRAVITY"] and p2.grav_eps == 0.01


def test_uniform_sphere():
    st = ics.uniform_sphere(20000, radius=2.0, total_mass=3.0, rho0=1.5, omega=(0, 0, 0.1), seed=1)
    r = np.linalg.norm(st["pos"], axis=1)
    assert r.max() <= 2.0 + 0.05  # the centre-of-mass shift moves the sphere by ~R/sqrt(N)
    assert abs(np.median(r) - 2.0 * 0.5 ** (1 / 3)) < 0.02
    assert abs(st["mass"].sum() - 3.0) < 1e-12
    assert np.abs((st["mass"][:, None] * st["pos"]).sum(0)).max() < 1e-12
    assert np.all(st["density"] == 1.5)
    # rigid rotation about z: v = omega x r (after the COM-velocity correction, which is ~0)
    assert np.allclose(st["vel"][:, 2], 0.0)


def test_two_sphere_impact_counts_and_frame():
    st = ics.two_sphere_impact(seed=3)
    assert st["mass"].shape[0] == 65536
    m = st["mass"]
    assert np.allclose(m, m[0]) and abs(m[0] - 4.0 / 3 * math.pi * 1.125 / 65536) < 1e-12
    assert np.abs((m[:, None] * st["vel"]).sum(0)).max() < 1e-12
    vrel = st["vel"][60000:, 0].mean() - st["vel"][:50000, 0].mean()
    assert abs(vrel - 0.5) < 1e-9


def test_plummer_sphere():
    st = ics.plummer_sphere(50000, seed=2)
    r = np.linalg.norm(st["pos"], axis=1)
    # half-mass radius of a Plummer sphere: a / sqrt(2^(2/3) - 1) = 1.3048 a
    assert abs(np.median(r) - 1.3048) < 0.03
    v = np.linalg.norm(st["vel"], axis=1)
    vesc = np.sqrt(2.0 / np.sqrt(r * r + 1.0))
    assert np.all(v <= vesc * 1.01 + 1e-3)


def test_ensemble_sizes():
    s = ics.ensemble_sizes(512, seed=0)
    assert s.shape == (512,) and s.min() >= 1024 and s.max() <= 32768
    assert 3.5e6 < s.sum() < 6e6
