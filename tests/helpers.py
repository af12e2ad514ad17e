"""Shared helpers of the parity tests: error metrics and state conversion."""

import numpy as np

from grasph2_b200.state import as_dtype, copy_state


def f32_exact(state):
    """Round a state to float32 and back: the values both the CUDA path and the oracle receive."""
    return as_dtype(as_dtype(state, np.float32), np.float64)


def rel_max(a, b, axis=None):
    """max |a - b| / max |b| (norm-wise relative error)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s) if s > 0 else float(np.abs(a - b).max())


def vec_rel(a, b):
    """Vector field error: max_i |a_i - b_i| / rms_i |b_i| (rows are vectors)."""
    a = np.asarray(a, dtype=np.float64).reshape(len(a), -1)
    b = np.asarray(b, dtype=np.float64).reshape(len(b), -1)
    rms = np.sqrt((b * b).sum(1).mean())
    d = np.sqrt(((a - b) ** 2).sum(1)).max()
    return float(d / rms) if rms > 0 else float(d)


def pointwise_rel(a, b):
    """max_i |a_i - b_i| / |b_i| for a positive scalar field."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float((np.abs(a - b) / np.abs(b)).max())


def golden_state(z, prefix):
    return {k[len(prefix):]: np.array(z[k]) for k in z.files if k.startswith(prefix)}


__all__ = ["f32_exact", "rel_max", "vec_rel", "pointwise_rel", "golden_state", "copy_state"]


# ---- condition-aware comparison ------------------------------------------------------------------
ULP32 = 2.0 ** -24
INPUTS = ("pos", "mass", "vel", "density", "dstress", "balsara")


def perturb_ulp(state, rng):
    """Every input value times (1 +- 2^-24): a random one-ulp float32 rounding of the inputs."""
    out = copy_state(state)
    for k in INPUTS:
        a = out[k]
        out[k] = a * (1.0 + ULP32 * rng.choice([-1.0, 1.0], size=a.shape))
    return out


def fp32_sensitivity(run, state, trials=2, seed=0):
    """run(state) -> dict of FP64 outputs. Returns (outputs, per-value sensitivity): the largest change
    of the outputs over `trials` one-ulp perturbations of the inputs. It measures how much float32
    rounding alone can move each result (large for particles at the edge of the kernel support,
    whose density sums only a few (1-q)^3 terms)."""
    rng = np.random.default_rng(seed)
    base = run(copy_state(state))
    sens = {k: np.zeros_like(np.asarray(v, dtype=np.float64)) for k, v in base.items()}
    for _ in range(trials):
        out = run(perturb_ulp(state, rng))
        for k in sens:
            sens[k] = np.maximum(sens[k], np.abs(np.asarray(out[k], np.float64) - np.asarray(base[k], np.float64)))
    return base, sens


COND_FACTOR = 32.0
# Per checked field: (what, norm-wise error, values that needed the sensitivity term, values,
# largest err / (tol * max|want|)); printed in the pytest terminal summary.
SLACK_LOG = []
NORM_LOG = []  # error lines the tests add (norm-wise errors of the plain and compensated forms per config)


def check_within(got, want, sens, tol, what, factor=COND_FACTOR, extra=0.0):
    """Per value: |got - want| <= tol * max|want| + factor * sensitivity + extra. Returns the norm-wise
    error, and records how many values needed the sensitivity (and extra) terms (SLACK_LOG)."""
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    sens = np.asarray(sens, np.float64)
    scale = np.abs(want).max()
    err = np.abs(got - want)
    allowed = tol * scale + factor * sens + extra
    if scale == 0:
        allowed = allowed + tol
    base = tol * scale if scale > 0 else tol
    n_slack = int((err > base).sum())
    SLACK_LOG.append((what, float(err.max() / scale) if scale else float(err.max()), n_slack, int(err.size),
                      float(err.max() / base)))
    bad = err > allowed
    if bad.any():
        i = np.unravel_index(np.argmax(err - allowed), err.shape)
        raise AssertionError("%s: %d values out of bound; worst at %s: err %.3e allowed %.3e (tol part %.3e, "
                             "sensitivity %.3e); norm-wise %.3e" % (what, int(bad.sum()), i, err[i], allowed[i],
                                                                    tol * scale, sens[i],
                                                                    err.max() / scale if scale else err.max()))
    return float(err.max() / scale) if scale else float(err.max())
