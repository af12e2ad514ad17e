"""Device initial-condition generators against their host restatement and the target distributions."""

import numpy as np
import pytest

import ics_oracle as O
from grasph2_b200 import ics

pytestmark = pytest.mark.gpu


def test_uniform_sphere_matches_host():
    n = 20000
    st = ics.uniform_sphere_device(n, radius=1.5, total_mass=2.0, rho0=0.3, omega=(0.0, 0.1, 0.4), seed=7,
                                   com_correct=False)
    ref = O.uniform_sphere(n, 1.5, 2.0, 0.3, (0.0, 0.1, 0.4), 7)
    for k in ("pos", "vel", "mass", "density"):
        got = st[k].cpu().numpy().astype(np.float64)
        np.testing.assert_allclose(got, ref[k], rtol=2e-6, atol=2e-7, err_msg=k)
    r = np.linalg.norm(ref["pos"], axis=1)
    assert r.max() <= 1.5
    # radial CDF of a uniform ball: (r/R)^3 (Kolmogorov-Smirnov distance)
    rs = np.sort(r / 1.5)
    assert np.abs(rs ** 3 - (np.arange(1, n + 1) / n)).max() < 0.015


def test_plummer_matches_host_and_com():
    n = 30000
    st = ics.plummer_sphere_device(n, a=1.0, seed=11, com_correct=False)
    ref = O.plummer(n, 1.0, 1.0, 1.0, 11)
    for k in ("pos", "vel", "mass"):
        np.testing.assert_allclose(st[k].cpu().numpy().astype(np.float64), ref[k], rtol=2e-5, atol=1e-6, err_msg=k)
    c = ics.plummer_sphere_device(n, a=1.0, seed=11, com_correct=True)
    m = c["mass"].cpu().numpy().astype(np.float64)
    for k in ("pos", "vel"):
        com = (m[:, None] * c[k].cpu().numpy().astype(np.float64)).sum(0) / m.sum()
        assert np.abs(com).max() < 1e-6, (k, com)


def test_device_upload_equals_host_upload():
    from grasph2_b200.params import config0_params
    from grasph2_b200.sim import DeviceParticleBuffer
    n = 3000
    st = ics.uniform_sphere_device(n, rho0=0.239, omega=(0, 0, 0.1), seed=3)
    host = {k: v.cpu().numpy() for k, v in st.items()}
    p = config0_params()
    with DeviceParticleBuffer(p, n) as a, DeviceParticleBuffer(p, n) as b:
        a.upload_device(st)
        b.upload(host)
        a.compute_derivatives()
        b.compute_derivatives()
        x, y = a.download(), b.download()
    for k in x:
        np.testing.assert_array_equal(x[k], y[k], err_msg=k)
