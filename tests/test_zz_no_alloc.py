"""gsph_gravity_accel_static: the entry point for callers that may not allocate device memory.

Such a caller owns every device buffer (a host program with a device-memory pool fixed at start-up,
or a loop that must not stall on cudaMalloc), so the entry point keeps its scratch in a fixed device
array inside the library. This file is collected last so a failure here does not hide the others.
The reference is the context path (gsph_compute_derivatives, gravity only), called through the C-ABI
with the same particles; the two must agree to the 1e-5 norm-wise bound of the parity tests, on two
calls in a row of different sizes (the second call must not see the first call's leftovers).
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
    torch.cuda.synchronize()
    out = d_acc.cpu().numpy().astype(np.float64)
    assert np.all(out[:, 3] == 0.0)
    return out[:, :3]


def test_static_gravity_matches_context_path_twice():
    lib = _abi.load_library()
    G, eps = 1.0, 0.01
    params = make_params(switches=("SELF_GRAVITY",), H=eps, grav_eps=eps, grav_G=G)
    for n, seed in ((70000, 1), (3001, 2)):  # a large then a small call: leftovers must not leak
        st = ics.plummer_sphere(n, seed=seed)
        st = {k: v.astype(np.float32).astype(np.float64) for k, v in st.items()}
        want = context_gravity(params, st)
        got = static_gravity(lib, st, G, eps)
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err <= TOL_ACC, "n=%d: %.3e" % (n, err)


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
