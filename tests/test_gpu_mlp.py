"""Tensor-core kernels of the surrogate's MLP: operand encodings against host products."""

import ctypes

import numpy as np
import pytest

from grasph2_b200._abi import load_library

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("b_mn", [0, 1])
@pytest.mark.parametrize("a_mn", [0, 1])
@pytest.mark.parametrize("N,K", [(16, 16), (128, 32), (64, 128), (128, 128), (16, 128), (32, 64)])
def test_tc_gemm_check(N, K, a_mn, b_mn):
    import torch
    lib = load_library()
    g = torch.Generator().manual_seed(N * 1000 + K * 10 + 2 * a_mn + b_mn)
    A = torch.randn(128, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)
    dA, dB = A.cuda(), B.cuda()
    D = torch.zeros(128, N, dtype=torch.float32, device="cuda")
    rc = lib.gsph_tc_gemm_check(ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()),
                                ctypes.c_void_p(D.data_ptr()), N, K, a_mn, b_mn)
    assert rc == 0, lib.gsph_last_error(None)
    want = A.double().numpy() @ B.double().numpy().T
    err = np.abs(D.cpu().numpy() - want).max() / np.abs(want).max()
    assert err < 1e-5, (N, K, a_mn, b_mn, err)


# ---- the surrogate's MLP against the CPU oracle ------------------------------------------------
import mlp_oracle as M  # noqa: E402


def _setup(n, seed):
    rng = np.random.default_rng(seed)
    p = M.init_params(seed)
    p[M.COUNT - 13:] = rng.normal(size=13) * 0.1
    for name_off in (4096, 4096 + 128 + 16384, 4096 + 128 + 16384 + 128 + 16384):  # b1, b2, b3
        p[name_off:name_off + 128] = rng.normal(size=128) * 0.1
    x = rng.normal(size=(n, M.IN)).astype(np.float32)
    t = rng.normal(size=(n, M.OUT)).astype(np.float32)
    w = rng.uniform(0.5, 2.0, size=M.OUT).astype(np.float32)
    return p, x, t, w


def _blocks(g):
    out, o = {}, 0
    for name, shape in M.SHAPES:
        k = int(np.prod(shape))
        out[name] = g[o:o + k]
        o += k
    return out


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 40000, 300001])
def test_mlp_forward_vs_oracle(n):
    import torch
    from grasph2_b200.mlp import MLP
    p, x, _, _ = _setup(n, 11)
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros(n, M.OUT, device="cuda")
    with MLP(p) as net:
        net.forward(xd, yd, n)
        torch.cuda.synchronize()
    y = yd.cpu().numpy().astype(np.float64)
    want, _ = M.forward(p, x, emulate=True)
    exact, _ = M.forward(p, x, emulate=False)
    scale = np.abs(want).max()
    assert np.abs(y - want).max() / scale < 5e-3, np.abs(y - want).max() / scale
    assert np.abs(y - exact).max() / scale < 5e-2


@pytest.mark.parametrize("n", [100, 1000, 20000])
def test_mlp_gradient_vs_oracle(n):
    import torch
    from grasph2_b200.mlp import MLP
    p, x, t, w = _setup(n, 12)
    xd, td, wd = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(w).cuda()
    with MLP(p) as net:
        g, loss = net.gradient(xd, td, wd, n)
    want, wl = M.gradient(p, x.astype(np.float64), t.astype(np.float64), w.astype(np.float64), emulate=True)
    exact, _ = M.gradient(p, x.astype(np.float64), t.astype(np.float64), w.astype(np.float64), emulate=False)
    assert abs(loss - wl) <= 1e-3 * wl, (loss, wl)
    G, W, E = _blocks(g.astype(np.float64)), _blocks(want), _blocks(exact)
    for name in G:
        scale = np.abs(W[name]).max()
        e = np.abs(G[name] - W[name]).max() / scale
        assert e < 1e-2, (name, e)
        assert np.abs(G[name] - E[name]).max() / np.abs(E[name]).max() < 8e-2, name


def test_mlp_gradient_deterministic():
    import torch
    from grasph2_b200.mlp import MLP
    p, x, t, w = _setup(5000, 13)
    xd, td, wd = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(w).cuda()
    with MLP(p) as net:
        g1, l1 = net.gradient(xd, td, wd, 5000)
        g2, l2 = net.gradient(xd, td, wd, 5000)
    np.testing.assert_array_equal(g1, g2)
    assert l1 == l2


def test_mlp_training_fits_a_teacher():
    """Adam on the device fits a fixed random teacher network: the loss falls by 10x."""
    import torch
    from grasph2_b200.mlp import MLP
    n = 4096
    teacher = M.init_params(21) * 0.5
    rng = np.random.default_rng(22)
    x = rng.normal(size=(n, M.IN)).astype(np.float32)
    t = M.forward(teacher, x, emulate=False)[0].astype(np.float32)
    w = np.ones(M.OUT, dtype=np.float32)
    xd, td, wd = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(w).cuda()
    with MLP(M.init_params(23)) as net:
        _, l0 = net.gradient(xd, td, wd, n)
        for _ in range(300):
            net.gradient(xd, td, wd, n, want=False)
            net.adam(lr=2e-3)
        _, l1 = net.gradient(xd, td, wd, n)
    assert l1 < 0.1 * l0, (l0, l1)


@pytest.mark.parametrize("clip", [0.0, 1e-3, 1e6])
def test_adam_with_gradient_clipping_matches_host(clip):
    """Two Adam steps on the device against the host restatement: g scaled by min(1, clip / ||g||_2)
    (clip 0 = off, a tiny clip always scales, a huge one never does), then Adam with bias correction."""
    import torch
    from grasph2_b200.mlp import MLP
    p, x, t, w = _setup(3000, 17)
    xd, td, wd = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(w).cuda()
    lr, b1, b2, eps = 1e-3, 0.9, 0.999, 1e-8
    with MLP(p) as net:
        net.set_grad_clip(clip)
        wh = net.params().astype(np.float64)
        mh = np.zeros_like(wh)
        vh = np.zeros_like(wh)
        for step in (1, 2):
            g, _ = net.gradient(xd, td, wd, 3000)
            g = g.astype(np.float64)
            nrm = np.sqrt((g * g).sum())
            if clip > 0 and nrm > clip:
                g = g * (clip / nrm)
            mh = b1 * mh + (1 - b1) * g
            vh = b2 * vh + (1 - b2) * g * g
            wh = wh - lr * (mh / (1 - b1 ** step)) / (np.sqrt(vh / (1 - b2 ** step)) + eps)
            net.adam(lr=lr, beta1=b1, beta2=b2, eps=eps)
            got = net.params().astype(np.float64)
            np.testing.assert_allclose(got, wh, rtol=0, atol=2e-6 * max(1.0, np.abs(wh).max()))
            wh = got  # continue from the device's FP32 parameters


def test_mlp_forward_rejects_misaligned_inputs():
    """The input rows are read as 16-byte vectors: an input pointer off a 16-byte boundary is an error,
    not a fault."""
    import torch
    from grasph2_b200.mlp import MLP
    from grasph2_b200.sim import GsphError
    p, x, _, _ = _setup(100, 3)
    xd = torch.from_numpy(np.concatenate([np.zeros(1, np.float32), x.ravel()])).cuda()
    yd = torch.zeros(100, M.OUT, device="cuda")
    with MLP(p) as net:
        with pytest.raises(GsphError) as e:
            net.forward(xd.data_ptr() + 4, yd, 100)
        assert e.value.code == -1
