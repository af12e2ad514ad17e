"""Python side of the surrogate's per-particle MLP (gsph_mlp_*): parameters on the device, forward and
gradient on the tensor cores, Adam. Inputs and outputs are device arrays (torch CUDA tensors or raw
pointers); the library fails loudly when it is missing.
"""

import ctypes
import math

import numpy as np

from ._abi import load_library
from .sim import GsphError, _stream_handle

IN, OUT = 32, 13


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(int(a))


SHAPES = [(128, 32), (128,), (128, 128), (128,), (128, 128), (128,), (13, 128), (13,)]


def init_params(seed=0):
    """Kaiming-uniform weights (bound sqrt(6 / fan_in), suited to SiLU), zero biases, as the flat vector."""
    rng = np.random.default_rng(seed)
    parts = []
    for shape in SHAPES:
        if len(shape) == 2:
            b = math.sqrt(6.0 / shape[1])
            parts.append(rng.uniform(-b, b, size=shape).ravel())
        else:
            parts.append(np.zeros(shape))
    return np.concatenate(parts).astype(np.float32)


class MLP:
    def __init__(self, params=None):
        self.lib = load_library()
        self.count = int(self.lib.gsph_mlp_param_count())
        self._h = ctypes.c_void_p()
        p = None
        if params is not None:
            params = np.ascontiguousarray(params, dtype=np.float32)
            if params.shape != (self.count,):
                raise ValueError("params must have %d values" % self.count)
            p = params.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        rc = self.lib.gsph_mlp_create(p, ctypes.byref(self._h))
        if rc != 0:
            raise GsphError(rc, self.lib.gsph_last_error(None).decode())

    @classmethod
    def borrow(cls, handle, owner):
        """A view of an MLP owned by another native object (`owner` is kept alive; close() is a no-op)."""
        self = cls.__new__(cls)
        self.lib = load_library()
        self.count = int(self.lib.gsph_mlp_param_count())
        self._h = ctypes.c_void_p(handle)
        self._owner = owner
        return self

    def close(self):
        if getattr(self, "_owner", None) is not None:
            return
        if self._h:
            self.lib.gsph_mlp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != 0:
            raise GsphError(rc, self.lib.gsph_mlp_last_error(self._h).decode())

    def params(self):
        out = np.empty(self.count, dtype=np.float32)
        self._check(self.lib.gsph_mlp_get_params(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def set_params(self, params):
        params = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self.lib.gsph_mlp_set_params(self._h, params.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def forward(self, x, y, n, stream=None):
        """y[n][13] = MLP(x[n][32]) on device arrays."""
        self._check(self.lib.gsph_mlp_forward(self._h, _ptr(x), _ptr(y), int(n), _stream_handle(stream)))

    def gradient(self, x, target, wout, n, stream=None, want=True):
        """Gradient of (1/n) sum w_o (y - t)^2; returns (grad, loss) on the host when `want`."""
        grad = np.empty(self.count, dtype=np.float32) if want else None
        loss = ctypes.c_double(0.0)
        self._check(self.lib.gsph_mlp_gradient(
            self._h, _ptr(x), _ptr(target), _ptr(wout), int(n),
            grad.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if want else None,
            ctypes.byref(loss) if want else None, _stream_handle(stream)))
        return (grad, loss.value) if want else None

    def set_grad_clip(self, max_norm):
        """Global-norm clipping of the gradient in the following Adam steps (0: off)."""
        self._check(self.lib.gsph_mlp_set_grad_clip(self._h, float(max_norm)))

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        self._check(self.lib.gsph_mlp_adam(self._h, float(lr), float(beta1), float(beta2), float(eps),
                                           _stream_handle(stream)))
