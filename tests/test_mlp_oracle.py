"""The CPU oracle of the surrogate's MLP: BF16 rounding and gradients against finite differences."""

import numpy as np

import mlp_oracle as M


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(0)
    a = (rng.normal(size=10000) * 10.0 ** rng.integers(-6, 6, size=10000)).astype(np.float32)
    want = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy().astype(np.float64)
    np.testing.assert_array_equal(M.bf16(a), want)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = M.init_params(3).astype(np.float64)
    p[M.COUNT - 13:] = rng.normal(size=13) * 0.1  # nonzero b4
    x = rng.normal(size=(40, M.IN))
    t = rng.normal(size=(40, M.OUT))
    w = rng.uniform(0.5, 2.0, size=M.OUT)
    g, loss = M.gradient(p, x, t, w, emulate=False)
    idx = rng.choice(M.COUNT, 60, replace=False)
    for i in idx:
        e = np.zeros_like(p)
        e[i] = 1e-6
        lp = M.gradient(p + e, x, t, w, emulate=False)[1]
        lm = M.gradient(p - e, x, t, w, emulate=False)[1]
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])
