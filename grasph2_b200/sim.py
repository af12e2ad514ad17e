"""Host-side mirror of GraSPH2's hot-path interface, on top of the C-ABI.

    pb = DeviceParticleBuffer(params, n)     # DeviceParticleBuffer<...>(n)  (Device_base.h:126-145)
    pb.upload(host_state)                    # pb = hostBuffer                (Device_base.h:163-181)
    computeDerivatives(pb)                   # src/computeDerivatives.h:315-328
    integrate(pb, notFirstStep=True)         # src/integration.h:219-244
    dt = getCurrentTimestep(pb)              # src/integration.h:246-255
    state = pb.download()                    # HostParticleBuffer(pb)

Errors raise GsphError carrying the C status code and the library's message (the reference's
assert_cuda aborts instead). There is no CPU fallback: the CUDA library must be built and a GPU
present, or construction fails.
"""

import ctypes

import numpy as np

from . import _abi
from ._abi import (ALL_ATTRIBS, ATTR_BITS, GsphDiag, GsphHostParticles, GsphOptions, GsphParams, STATUS_NAMES,
                   load_library)
from .state import new_state, pointer_struct, state_size


class GsphError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (STATUS_NAMES.get(code, "?"), code, msg))
        self.code = code


def _stream_handle(stream):
    """Accept None (legacy default stream), an integer handle or a torch.cuda.Stream."""
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    h = getattr(stream, "cuda_stream", None)
    if h is not None:
        return int(h)
    raise TypeError("unsupported stream object %r" % (stream,))


def mask_of(names):
    m = 0
    for n in names:
        m |= ATTR_BITS[n]
    return m


class DeviceParticleBuffer:
    """Device-resident particles of one simulation (owns the C context)."""

    def __init__(self, params, n, options=None):
        if not isinstance(params, GsphParams):
            raise TypeError("params must be a GsphParams (see grasph2_b200.params.make_params)")
        self.lib = load_library()
        self.params = params
        self.n = int(n)
        self._ctx = ctypes.c_void_p()
        opt = ctypes.byref(options) if options is not None else None
        rc = self.lib.gsph_create(ctypes.byref(params), opt, self.n, ctypes.byref(self._ctx))
        if rc != 0:
            raise GsphError(rc, self.lib.gsph_last_error(None).decode())

    # -- lifetime ---------------------------------------------------------------------------
    def close(self):
        if self._ctx:
            self.lib.gsph_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

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
            raise GsphError(rc, self.lib.gsph_last_error(self._ctx).decode())

    def size(self):
        return self.n

    @property
    def handle(self):
        return self._ctx

    # -- transfers ----------------------------------------------------------------------------
    def upload(self, state, attributes=None, stream=None):
        """Copy host attributes (float32 arrays in the reference layout) to the device. By default
        every attribute present in `state` is uploaded."""
        names = [k for k in ATTR_BITS if k in state] if attributes is None else list(attributes)
        st = {k: np.ascontiguousarray(state[k], dtype=np.float32) for k in names}
        for k, v in st.items():
            if v.shape[0] != self.n:
                raise ValueError("attribute %s has %d rows, buffer holds %d" % (k, v.shape[0], self.n))
        hp = pointer_struct(st, GsphHostParticles, ctypes.c_float)
        self._check(self.lib.gsph_upload(self._ctx, mask_of(names), ctypes.byref(hp), _stream_handle(stream)))
        return self

    def download(self, attributes=None, stream=None, out=None):
        names = list(ATTR_BITS) if attributes is None else list(attributes)
        st = out if out is not None else new_state(self.n, np.float32)
        hp = pointer_struct({k: st[k] for k in names}, GsphHostParticles, ctypes.c_float)
        self._check(self.lib.gsph_download(self._ctx, mask_of(names), ctypes.byref(hp), _stream_handle(stream)))
        return {k: st[k] for k in names} if attributes is not None else st

    def upload_device(self, state, attributes=None, stream=None):
        """Upload from device arrays in the host layout (torch CUDA float32 tensors)."""
        names = [k for k in ATTR_BITS if k in state] if attributes is None else list(attributes)
        hp = GsphHostParticles()
        for k in names:
            v = state[k]
            if v.shape[0] != self.n or not v.is_cuda or not v.is_contiguous():
                raise ValueError("attribute %s must be a contiguous CUDA tensor with %d rows" % (k, self.n))
            setattr(hp, k, ctypes.cast(ctypes.c_void_p(v.data_ptr()), ctypes.POINTER(ctypes.c_float)))
        self._check(self.lib.gsph_upload_device(self._ctx, mask_of(names), ctypes.byref(hp), _stream_handle(stream)))
        return self

    def upload_f64(self, state, attributes=None, stream=None):
        """Double-precision host buffers (the reference's DOUBLE_PRECISION layout)."""
        names = [k for k in ATTR_BITS if k in state] if attributes is None else list(attributes)
        st = {k: np.ascontiguousarray(state[k], dtype=np.float64) for k in names}
        for k, v in st.items():
            if v.shape[0] != self.n:
                raise ValueError("attribute %s has %d rows, buffer holds %d" % (k, v.shape[0], self.n))
        hp = pointer_struct(st, _abi.GsphHostParticles64, ctypes.c_double)
        self._check(self.lib.gsph_upload_f64(self._ctx, mask_of(names), ctypes.byref(hp), _stream_handle(stream)))
        return self

    def download_f64(self, attributes=None, stream=None):
        names = list(ATTR_BITS) if attributes is None else list(attributes)
        st = new_state(self.n, np.float64)
        hp = pointer_struct({k: st[k] for k in names}, _abi.GsphHostParticles64, ctypes.c_double)
        self._check(self.lib.gsph_download_f64(self._ctx, mask_of(names), ctypes.byref(hp), _stream_handle(stream)))
        return {k: st[k] for k in names}

    def upload_pos64(self, pos, stream=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        assert pos.shape == (self.n, 3)
        self._check(self.lib.gsph_upload_pos64(self._ctx, pos.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               _stream_handle(stream)))

    def download_pos64(self, stream=None):
        pos = np.zeros((self.n, 3))
        self._check(self.lib.gsph_download_pos64(self._ctx, pos.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                 _stream_handle(stream)))
        return pos

    # -- hot path -----------------------------------------------------------------------------
    def compute_derivatives(self, stream=None):
        self._check(self.lib.gsph_compute_derivatives(self._ctx, _stream_handle(stream)))

    def integrate(self, not_first_step=True, stream=None):
        self._check(self.lib.gsph_integrate(self._ctx, int(bool(not_first_step)), _stream_handle(stream)))

    def step(self, nsteps=1, stream=None):
        self._check(self.lib.gsph_step(self._ctx, int(nsteps), _stream_handle(stream)))

    def current_timestep(self, stream=None):
        dt = ctypes.c_double()
        self._check(self.lib.gsph_current_timestep(self._ctx, ctypes.byref(dt), _stream_handle(stream)))
        return dt.value

    def diagnostics(self, half_kick=0.0, stream=None, fast=False):
        """FP64 energies, momentum, angular momentum; fast=True sums the pair potential in FP32 (compensated)."""
        d = GsphDiag()
        f = self.lib.gsph_diagnostics_fast if fast else self.lib.gsph_diagnostics
        self._check(f(self._ctx, float(half_kick), ctypes.byref(d), _stream_handle(stream)))
        return d.as_dict()

    def autotune(self, reps=3, stream=None):
        """Time candidate launch shapes on the current state and keep the fastest; returns the shape."""
        self._check(self.lib.gsph_autotune(self._ctx, int(reps), _stream_handle(stream)))
        return self.launch_shape()

    def launch_shape(self):
        sh = _abi.GsphLaunchShape()
        self._check(self.lib.gsph_launch_shape_get(self._ctx, ctypes.byref(sh)))
        return sh.as_dict()

    def launch_count(self):
        c = ctypes.c_int64()
        self._check(self.lib.gsph_launch_count(self._ctx, ctypes.byref(c)))
        return c.value

    # -- per-kernel timing ----------------------------------------------------------------------
    def profile_enable(self, on=True):
        self._check(self.lib.gsph_profile_enable(self._ctx, int(bool(on))))

    def profile_collect(self):
        self._check(self.lib.gsph_profile_collect(self._ctx))

    def profile_reset(self):
        self._check(self.lib.gsph_profile_reset(self._ctx))

    def profile_read(self):
        pr = _abi.GsphProfile()
        self._check(self.lib.gsph_profile_read(self._ctx, ctypes.byref(pr)))
        return {name: (pr.ms[k], pr.launches[k]) for k, name in enumerate(_abi.KSLOT_NAMES)}

    def device_view(self):
        v = _abi.GsphDeviceView()
        self._check(self.lib.gsph_device_view_get(self._ctx, ctypes.byref(v)))
        return v


# reference-named free functions --------------------------------------------------------------
class SnapshotWriter:
    """Asynchronous tsv snapshots of a context (gsph_writer_*): write() returns once the state is copied
    on the device; a worker thread writes the files."""

    def __init__(self, pb, attributes=("pos", "mass", "vel", "density"), depth=2):
        self.lib = pb.lib
        self._h = ctypes.c_void_p()
        rc = self.lib.gsph_writer_create(pb.handle, mask_of(attributes), int(depth), ctypes.byref(self._h))
        if rc != 0:
            raise GsphError(rc, self.lib.gsph_last_error(None).decode())

    def _check(self, rc):
        if rc != 0:
            raise GsphError(rc, self.lib.gsph_writer_last_error(self._h).decode())

    def write(self, filename, stream=None):
        self._check(self.lib.gsph_writer_write(self._h, str(filename).encode(), _stream_handle(stream)))

    def flush(self):
        n = ctypes.c_int64()
        self._check(self.lib.gsph_writer_flush(self._h, ctypes.byref(n)))
        return n.value

    def close(self):
        if self._h:
            rc = self.lib.gsph_writer_destroy(self._h)
            self._h = ctypes.c_void_p()
            if rc != 0:
                raise GsphError(rc, "snapshot writer failed")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Ensemble:
    """S independent simulations of uneven sizes with one parameter set (gsph_ensemble_*). Host states
    hold the simulations back to back, simulation k in rows offsets[k]:offsets[k+1]."""

    def __init__(self, params, counts, options=None):
        self.lib = load_library()
        self.params = params
        counts = np.ascontiguousarray(counts, dtype=np.int64)
        self.nsims = int(counts.shape[0])
        self._h = ctypes.c_void_p()
        opt = ctypes.byref(options) if options is not None else None
        rc = self.lib.gsph_ensemble_create(ctypes.byref(params), opt, self.nsims,
                                           counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(self._h))
        if rc != 0:
            raise GsphError(rc, self.lib.gsph_ensemble_last_error(None).decode())
        off = np.zeros(self.nsims + 1, dtype=np.int64)
        self._check(self.lib.gsph_ensemble_offsets(self._h, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        self.offsets = off
        self.n = int(off[-1])

    def close(self):
        if self._h:
            self.lib.gsph_ensemble_destroy(self._h)
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
            raise GsphError(rc, self.lib.gsph_ensemble_last_error(self._h).decode())

    def upload(self, state, attributes=None, stream=None):
        names = [k for k in ATTR_BITS if k in state] if attributes is None else list(attributes)
        st = {k: np.ascontiguousarray(state[k], dtype=np.float32) for k in names}
        for k, v in st.items():
            if v.shape[0] != self.n:
                raise ValueError("attribute %s has %d rows, the ensemble holds %d" % (k, v.shape[0], self.n))
        hp = pointer_struct(st, GsphHostParticles, ctypes.c_float)
        self._check(self.lib.gsph_ensemble_upload(self._h, mask_of(names), ctypes.byref(hp), _stream_handle(stream)))
        return self

    def download(self, attributes=None, stream=None, out=None):
        names = list(ATTR_BITS) if attributes is None else list(attributes)
        st = out if out is not None else new_state(self.n, np.float32)
        hp = pointer_struct({k: st[k] for k in names}, GsphHostParticles, ctypes.c_float)
        self._check(self.lib.gsph_ensemble_download(self._h, mask_of(names), ctypes.byref(hp), _stream_handle(stream)))
        return {k: st[k] for k in names}

    def upload_pos64(self, pos, stream=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        if pos.shape != (self.n, 3):
            raise ValueError("pos must have shape (%d, 3)" % self.n)
        self._check(self.lib.gsph_ensemble_upload_pos64(self._h, pos.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                        _stream_handle(stream)))

    def download_pos64(self, stream=None):
        pos = np.empty((self.n, 3), dtype=np.float64)
        self._check(self.lib.gsph_ensemble_download_pos64(self._h, pos.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                          _stream_handle(stream)))
        return pos

    def compute_derivatives(self, stream=None):
        self._check(self.lib.gsph_ensemble_compute_derivatives(self._h, _stream_handle(stream)))

    def inject_stall(self, sim):
        """Failure-path test hook: the next compute_derivatives stalls simulation `sim`'s SPH items until
        their device-side waits run out (gsph_ensemble_inject_stall)."""
        self._check(self.lib.gsph_ensemble_inject_stall(self._h, int(sim)))

    def integrate(self, not_first_step=True, stream=None):
        self._check(self.lib.gsph_ensemble_integrate(self._h, int(bool(not_first_step)), _stream_handle(stream)))

    def step(self, nsteps=1, stream=None):
        self._check(self.lib.gsph_ensemble_step(self._h, int(nsteps), _stream_handle(stream)))

    def diagnostics(self, half_kick=0.0, stream=None):
        arr = (GsphDiag * self.nsims)()
        self._check(self.lib.gsph_ensemble_diagnostics(self._h, float(half_kick), arr, _stream_handle(stream)))
        return [d.as_dict() for d in arr]

    def autotune(self, reps=2, stream=None):
        """Time the DENS j-tile and the persistent grid's CTAs per SM; keep the fastest."""
        t, c = ctypes.c_int32(), ctypes.c_int32()
        self._check(self.lib.gsph_ensemble_autotune(self._h, int(reps), ctypes.byref(t), ctypes.byref(c),
                                                    _stream_handle(stream)))
        return {"tile": t.value, "ctas_per_sm": c.value}

    def launch_count(self):
        c = ctypes.c_int64()
        self._check(self.lib.gsph_ensemble_launch_count(self._h, ctypes.byref(c)))
        return c.value

    def split(self, state):
        """Per-simulation views of a packed state."""
        return [{k: v[self.offsets[s]:self.offsets[s + 1]] for k, v in state.items()} for s in range(self.nsims)]


def pack_states(states):
    """Concatenate per-simulation states into the packed ensemble layout."""
    keys = [k for k in states[0]]
    return {k: np.concatenate([s[k] for s in states], axis=0) for k in keys}


def computeDerivatives(pb, stream=None):  # noqa: N802 (reference name)
    pb.compute_derivatives(stream)


def integrate(pb, notFirstStep=True, stream=None):  # noqa: N802,N803
    pb.integrate(notFirstStep, stream)


def getCurrentTimestep(pb, stream=None):  # noqa: N802
    return pb.current_timestep(stream)


def from_state(params, state, options=None):
    """Create a buffer sized for `state` and upload it."""
    pb = DeviceParticleBuffer(params, state_size(state), options)
    pb.upload(state)
    return pb


def validate_params(params):
    lib = load_library()
    buf = ctypes.create_string_buffer(256)
    rc = lib.gsph_params_validate(ctypes.byref(params), buf, 256)
    return rc, buf.value.decode()


def reference_default_params():
    lib = load_library()
    p = GsphParams()
    assert lib.gsph_params_reference_defaults(ctypes.byref(p)) == 0
    return p


def measure_fp32_peak(seconds=0.5):
    """FFMA throughput of the current device in TFLOP/s (FMA = 2 flops)."""
    lib = load_library()
    t = ctypes.c_double()
    rc = lib.gsph_measure_fp32_peak(float(seconds), ctypes.byref(t))
    if rc != 0:
        raise GsphError(rc, lib.gsph_last_error(None).decode())
    return t.value


def default_options():
    lib = load_library()
    o = GsphOptions()
    assert lib.gsph_options_defaults(ctypes.byref(o)) == 0
    return o


__all__ = ["DeviceParticleBuffer", "GsphError", "computeDerivatives", "integrate", "getCurrentTimestep",
           "from_state", "validate_params", "reference_default_params", "default_options", "ALL_ATTRIBS"]


# ---- HDF5 snapshots (gsph_h5_*; the system's libhdf5, loaded when first needed) -------------------
def h5_available():
    """True when libhdf5 (1.10 or later) could be loaded."""
    return bool(load_library().gsph_h5_available())


def write_h5(filename, state, attributes=("pos", "mass", "vel", "density")):
    """One float dataset per attribute (POS, MASS, VEL, DENSITY, ... as the reference names them)."""
    lib = load_library()
    names = list(attributes)
    st = {k: np.ascontiguousarray(state[k], dtype=np.float32) for k in names}
    hp = pointer_struct(st, GsphHostParticles, ctypes.c_float)
    rc = lib.gsph_h5_write(str(filename).encode(), state_size(st) if "mass" in st else st[names[0]].shape[0],
                           ctypes.byref(hp), mask_of(names))
    if rc != 0:
        raise GsphError(rc, lib.gsph_last_error(None).decode())


def read_h5(filename, attributes=("pos", "mass", "vel", "density")):
    lib = load_library()
    names = list(attributes)
    n = ctypes.c_int64(0)
    rc = lib.gsph_h5_read(str(filename).encode(), 0, None, 0, ctypes.byref(n))
    if rc != 0:
        raise GsphError(rc, lib.gsph_last_error(None).decode())
    full = new_state(n.value, np.float32)
    st = {k: full[k] for k in names}
    hp = pointer_struct(st, GsphHostParticles, ctypes.c_float)
    rc = lib.gsph_h5_read(str(filename).encode(), mask_of(names), ctypes.byref(hp), n.value, ctypes.byref(n))
    if rc != 0:
        raise GsphError(rc, lib.gsph_last_error(None).decode())
    return st
