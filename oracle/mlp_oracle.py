"""CPU oracle of the surrogate's MLP (test infrastructure only): forward and backward of
32 -> 128 -> 128 -> 128 -> 13 with SiLU, in FP64, optionally rounding the tensors the GPU stores in
BF16 at the same points (inputs, weights, activations, output gradient, layer gradients), so that the
GPU's tensor-core kernels can be compared with what they compute up to FP32 summation order.

The parameter layout is the flat vector of include/grasph2_b200.h (gsph_mlp_*).
"""

import numpy as np

IN, HID, OUT = 32, 128, 13
SHAPES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)), ("b3", (HID,)),
          ("W4", (OUT, HID)), ("b4", (OUT,))]
COUNT = sum(int(np.prod(s)) for _, s in SHAPES)


def unflatten(v):
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = np.asarray(v[o:o + k], dtype=np.float64).reshape(shape)
        o += k
    return out


def flatten(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def bf16(a):
    """Round to bfloat16 (round to nearest even) and back."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def init_params(seed=0):
    """Kaiming-uniform weights for SiLU layers, zero biases."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in SHAPES:
        if name.startswith("W"):
            bound = np.sqrt(6.0 / shape[1])
            d[name] = rng.uniform(-bound, bound, size=shape)
        else:
            d[name] = np.zeros(shape)
    return flatten(d).astype(np.float32)


def forward(params, x, emulate=True):
    P = unflatten(params)
    r = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    h = r(x)
    cache = {"h0": h}
    for l in (1, 2, 3):
        z = h @ r(P["W%d" % l]).T + P["b%d" % l]
        h = r(silu(z))
        cache["z%d" % l] = z
        cache["h%d" % l] = h
    y = h @ r(P["W4"]).T + P["b4"]
    return y, cache


def gradient(params, x, target, wout, emulate=True):
    """(grad vector, loss) of L = (1/n) sum w_o (y - t)^2."""
    P = unflatten(params)
    r = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    n = x.shape[0]
    y, c = forward(params, x, emulate)
    d = y - target
    loss = float((wout[None, :] * d * d).sum() / n)
    g = r(2.0 * wout[None, :] * d / n)
    G = {"W4": g.T @ c["h3"], "b4": g.sum(0)}
    dh = g @ r(P["W4"])
    for l in (3, 2, 1):
        dz = r(dh * dsilu(c["z%d" % l]))
        G["W%d" % l] = dz.T @ c["h%d" % (l - 1)]
        G["b%d" % l] = dz.sum(0)
        dh = dz @ r(P["W%d" % l])
    return flatten(G), loss
