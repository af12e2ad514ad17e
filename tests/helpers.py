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
