"""gsph_gravity_accel_static: the entry point for callers that may not allocate device memory.

Such a caller owns every device buffer (a host program with a device-memory pool fixed at start-up,
or a loop that must not stall on cudaMalloc), so the entry point keeps its scratch in a fixed device
array inside the library. This file is collected last so a failure here does not hide the others.

Checks, all through the C-ABI: the accelerations against the FP64 oracle (softened gravity of every
target against all sources) and against the context path (gsph_compute_derivatives, gravity only),
to the 1e-5 norm-wise bound of the parity tests, on two calls in a row of different sizes (the second
call must not see the first call's leftovers); the unsoftened form (eps = 0, its own kernel variant)
on the small-N launch shape; and the failure path: a call that starts with the timeout bit set (as if
a device-side wait had given up; no wait is made to run out) writes NaN and its status query reports
GSPH_E_TIMEOUT, and the next call is clean again.
"""

import ctypes

import numpy as np
import pytest

from grasph2_b200 import _abi, ics
from grasph2_b200.params import make_params
from grasph2_b200.sim import DeviceParticleBuffer

pytestmark = pytest.mark.gpu

TOL_ACC = 1e-5


def context_gravity(params, st):
    with DeviceParticleBuffer(params, st["mass"].shape[0]) as pb:
        pb.upload(st)
        pb.compute_derivatives()
        return pb.download(["acc"])["acc"].astype(np.float64)


def static_gravity(lib, st, G, eps):
    import torch
    n = st["mass"].shape[0]
    posm = np.concatenate([st["pos"], st["mass"][:, None]], axis=1).astype(np.float32)
    d_posm = torch.from_numpy(posm).cuda()
    d_acc = torch.full((n, 4), float("nan"), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = lib.gsph_gravity_accel_static(ctypes.c_void_p(d_posm.data_ptr()), n, G, eps,
                                       ctypes.c_void_p(d_acc.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, lib.gsph_last_error(None)
    status = lib.gsph_gravity_accel_static_status(ctypes.c_void_p(stream.cuda_stream))
    out = d_acc.cpu().numpy().astype(np.float64)
    return out, status


def f32_plummer(n, seed):
    st = ics.plummer_sphere(n, seed=seed)
    return {k: v.astype(np.float32).astype(np.float64) for k, v in st.items()}


def test_static_gravity_matches_oracle_and_context_path_twice(oracle):
    lib = _abi.load_library()
    G, eps = 1.0, 0.01
    params = make_params(switches=("SELF_GRAVITY",), H=eps, grav_eps=eps, grav_G=G)
    for n, seed in ((70000, 1), (3001, 2)):  # a large then a small call: leftovers must not leak
        st = f32_plummer(n, seed)
        out, status = static_gravity(lib, st, G, eps)
        assert status == 0, lib.gsph_last_error(None)
        assert np.all(out[:, 3] == 0.0)
        got = out[:, :3]
        idx = np.random.default_rng(seed).choice(n, min(n, 1024), replace=False)
        want = oracle.gravity_targets(params, st["pos"], st["mass"], idx)
        err = np.abs(got[idx] - want).max() / np.abs(want).max()
        assert err <= TOL_ACC, "n=%d vs the FP64 oracle: %.3e" % (n, err)
        ctx = context_gravity(params, st)
        err = np.abs(got - ctx).max() / np.abs(ctx).max()
        assert err <= TOL_ACC, "n=%d vs the context path: %.3e" % (n, err)


def test_static_gravity_unsoftened_small_n(oracle):
    """eps = 0 (the unsoftened kernel variant, 1/r clamped for coincident points) at n = 1000, which
    pads to exactly 1024 particles and takes the small-N launch shape."""
    lib = _abi.load_library()
    G = 1.0
    n = 1000
    st = f32_plummer(n, 5)
    assert len(np.unique(st["pos"], axis=0)) == n
    params = make_params(switches=("SELF_GRAVITY",), H=0.01, grav_eps=0.0, grav_G=G)
    out, status = static_gravity(lib, st, G, 0.0)
    assert status == 0, lib.gsph_last_error(None)
    got = out[:, :3]
    want = oracle.gravity_targets(params, st["pos"], st["mass"], np.arange(n))
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err <= TOL_ACC, "eps=0 vs the FP64 oracle: %.3e" % err
    ctx = context_gravity(params, st)
    err = np.abs(got - ctx).max() / np.abs(ctx).max()
    assert err <= TOL_ACC, "eps=0 vs the context path: %.3e" % err


def test_static_gravity_reports_a_timeout_as_nan():
    lib = _abi.load_library()
    st = f32_plummer(2048, 7)
    assert lib.gsph_inject_static_timeout(1) == 0
    out, status = static_gravity(lib, st, 1.0, 0.01)
    assert status == _abi.GSPH_E_TIMEOUT
    assert b"gave up" in lib.gsph_last_error(None)
    assert np.all(np.isnan(out))
    out, status = static_gravity(lib, st, 1.0, 0.01)  # one-shot: the next call is clean
    assert status == 0
    assert np.all(np.isfinite(out))


def test_static_gravity_rejects_oversize_and_bad_pointers():
    lib = _abi.load_library()
    import torch
    buf = torch.zeros((16, 4), dtype=torch.float32, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    assert lib.gsph_gravity_accel_static(p, 524289, 1.0, 0.01, p, None) == _abi.GSPH_E_INVALID
    assert b"524288" in lib.gsph_last_error(None)
    assert lib.gsph_gravity_accel_static(None, 16, 1.0, 0.01, p, None) == _abi.GSPH_E_INVALID
    misaligned = ctypes.c_void_p(buf.data_ptr() + 4)
    assert lib.gsph_gravity_accel_static(misaligned, 8, 1.0, 0.01, p, None) == _abi.GSPH_E_INVALID
