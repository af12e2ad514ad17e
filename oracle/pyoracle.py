"""Python bindings of the checkers (test infrastructure only).

Oracle      -- oracle/liboracle.so, the FP64 restatement (oracle/oracle.cpp)
RefBuild    -- oracle/_ref/libref_<variant>_<fp32|fp64>.so, GraSPH2's own job headers built for the
               host (oracle/ref_driver.cpp); one library per physics variant (oracle/ref_variants.py)
RefCuda     -- oracle/_ref/libref_cuda_<variant>.so, GraSPH2's own CUDA path built for sm_100a
               (oracle/ref_cuda_driver.cu), FP32; valid for N a multiple of 256

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from grasph2_b200._abi import GsphParams, GsphDiag, OracleParticles  # noqa: E402
from grasph2_b200.state import as_dtype, pointer_struct, state_size  # noqa: E402

ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")


class OracleTimestep(ctypes.Structure):
    _fields_ = [("current", ctypes.c_double), ("next", ctypes.c_double)]


class Oracle:
    def __init__(self, path=ORACLE_LIB):
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: %s (run python oracle/build_ref.py)" % path)
        L = ctypes.CDLL(path)
        P = ctypes.POINTER
        L.oracle_compute_derivatives.argtypes = [P(GsphParams), ctypes.c_int64, P(OracleParticles), ctypes.c_int64,
                                                 ctypes.c_int64, P(OracleTimestep)]
        L.oracle_integrate.argtypes = [P(GsphParams), ctypes.c_int64, ctypes.c_int, P(OracleParticles),
                                       P(OracleTimestep)]
        L.oracle_gravity_targets.argtypes = [P(GsphParams), ctypes.c_int64, P(ctypes.c_double), P(ctypes.c_double),
                                             ctypes.c_int64, P(ctypes.c_int64), P(ctypes.c_double)]
        L.oracle_diagnostics.argtypes = [P(GsphParams), ctypes.c_int64, P(OracleParticles), ctypes.c_double,
                                         P(GsphDiag)]
        for f in ("oracle_w_spline", "oracle_dw_spline"):
            getattr(L, f).restype = ctypes.c_double
            getattr(L, f).argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.oracle_plasticity.argtypes = [P(ctypes.c_double), ctypes.c_double]
        L.oracle_plasticity.restype = None
        L.oracle_dstress_dt.argtypes = [P(ctypes.c_double)] * 3 + [ctypes.c_double, P(ctypes.c_double)]
        L.oracle_dstress_dt.restype = None
        self.lib = L
        self.ts = OracleTimestep(0.0, 0.0)

    @staticmethod
    def _struct(state):
        return pointer_struct(state, OracleParticles, ctypes.c_double)

    def compute_derivatives(self, params, state, i0=0, i1=-1):
        """In place on an FP64 state (dict of float64 arrays)."""
        s = self._struct(state)
        rc = self.lib.oracle_compute_derivatives(ctypes.byref(params), state_size(state), ctypes.byref(s), i0, i1,
                                                 ctypes.byref(self.ts))
        assert rc == 0, rc

    def integrate(self, params, state, not_first_step=True):
        s = self._struct(state)
        rc = self.lib.oracle_integrate(ctypes.byref(params), state_size(state), int(not_first_step), ctypes.byref(s),
                                       ctypes.byref(self.ts))
        assert rc == 0, rc

    def step(self, params, state, nsteps=1, not_first_step=True):
        for _ in range(nsteps):
            self.compute_derivatives(params, state)
            self.integrate(params, state, not_first_step)

    def gravity_targets(self, params, pos, mass, idx):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        out = np.zeros((idx.size, 3))
        dp = ctypes.POINTER(ctypes.c_double)
        rc = self.lib.oracle_gravity_targets(ctypes.byref(params), mass.size, pos.ctypes.data_as(dp),
                                             mass.ctypes.data_as(dp), idx.size,
                                             idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), out.ctypes.data_as(dp))
        assert rc == 0, rc
        return out

    def diagnostics(self, params, state, half_kick=0.0):
        s = self._struct(state)
        d = GsphDiag()
        rc = self.lib.oracle_diagnostics(ctypes.byref(params), state_size(state), ctypes.byref(s), half_kick,
                                         ctypes.byref(d))
        assert rc == 0, rc
        return d.as_dict()

    def w(self, r, h, dim=3):
        return self.lib.oracle_w_spline(dim, r, h)

    def dw(self, r, h, dim=3):
        return self.lib.oracle_dw_spline(dim, r, h)

    def plasticity(self, S, Y):
        S = np.ascontiguousarray(S, dtype=np.float64).copy()
        self.lib.oracle_plasticity(S.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), Y)
        return S

    def dstress_dt(self, edot, rdot, S, shear):
        out = np.zeros((3, 3))
        dp = ctypes.POINTER(ctypes.c_double)
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (edot, rdot, S)]
        self.lib.oracle_dstress_dt(*[a.ctypes.data_as(dp) for a in args], shear, out.ctypes.data_as(dp))
        return out


class RefParticles(ctypes.Structure):
    pass


def ref_library_path(variant, double):
    return os.path.join(REF_DIR, "libref_%s_%s.so" % (variant, "fp64" if double else "fp32"))


def ref_available(variant="fluid"):
    return os.path.exists(ref_library_path(variant, True))


class RefBuild:
    """The reference's own computeDerivatives/integrate for one variant and precision."""

    def __init__(self, variant, double=True):
        path = ref_library_path(variant, double)
        if not os.path.exists(path):
            raise RuntimeError("reference build missing: %s" % path)
        self.dtype = np.float64 if double else np.float32
        self.ctype = ctypes.c_double if double else ctypes.c_float
        L = ctypes.CDLL(path)
        fields = [(n, ctypes.POINTER(self.ctype)) for n, _ in OracleParticles._fields_]
        self.struct_type = type("RefParticles_%s" % ("fp64" if double else "fp32"), (ctypes.Structure,),
                                {"_fields_": fields})
        P = ctypes.POINTER(self.struct_type)
        L.ref_compute_derivatives.argtypes = [ctypes.c_int64, P, ctypes.c_int64, ctypes.c_int64]
        L.ref_compute_derivatives_rows.argtypes = [ctypes.c_int64, P, ctypes.c_int64, ctypes.c_int64]
        L.ref_integrate.argtypes = [ctypes.c_int64, ctypes.c_int, P]
        L.ref_integrate_variable.argtypes = [ctypes.c_int64, ctypes.c_int, P]
        for f in ("ref_current_timestep", "ref_next_timestep", "ref_fixed_timestep"):
            getattr(L, f).restype = ctypes.c_double
            getattr(L, f).argtypes = []
        L.ref_set_timestep.argtypes = [ctypes.c_double, ctypes.c_double]
        L.ref_set_timestep.restype = None
        L.ref_w_spline.restype = ctypes.c_double
        L.ref_w_spline.argtypes = [ctypes.c_double]
        L.ref_dw_spline.restype = ctypes.c_double
        L.ref_dw_spline.argtypes = [ctypes.c_double]
        L.ref_plasticity.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_double]
        L.ref_plasticity.restype = None
        L.ref_dstress_dt.argtypes = [ctypes.POINTER(ctypes.c_double)] * 3 + [ctypes.c_double,
                                                                              ctypes.POINTER(ctypes.c_double)]
        L.ref_dstress_dt.restype = None
        L.ref_precision.restype = ctypes.c_int
        L.ref_variant.restype = ctypes.c_char_p
        self.lib = L
        self.variant = variant

    def prepare(self, state):
        return as_dtype(state, self.dtype)

    def _struct(self, state):
        for k, v in state.items():
            if v.dtype != self.dtype:
                raise TypeError("state attribute %s has dtype %s, expected %s" % (k, v.dtype, self.dtype))
        return pointer_struct(state, self.struct_type, self.ctype)

    def compute_derivatives(self, state, i0=0, i1=-1):
        s = self._struct(state)
        assert self.lib.ref_compute_derivatives(state_size(state), ctypes.byref(s), i0, i1) == 0

    def compute_derivatives_rows(self, state, i0, i1):
        """Timing sample: all passes over rows [i0, i1) only."""
        s = self._struct(state)
        assert self.lib.ref_compute_derivatives_rows(state_size(state), ctypes.byref(s), i0, i1) == 0

    def integrate(self, state, not_first_step=True, variable=False):
        s = self._struct(state)
        f = self.lib.ref_integrate_variable if variable else self.lib.ref_integrate
        assert f(state_size(state), int(not_first_step), ctypes.byref(s)) == 0

    def step(self, state, nsteps=1, not_first_step=True, variable=False):
        for _ in range(nsteps):
            self.compute_derivatives(state)
            self.integrate(state, not_first_step, variable)


def ref_cuda_library_path(variant):
    return os.path.join(REF_DIR, "libref_cuda_%s.so" % variant)


def ref_cuda_available(variant="fluid"):
    return os.path.exists(ref_cuda_library_path(variant))


class RefCuda:
    """GraSPH2's own CUDA computeDerivatives / integrate on the current device, one buffer of n particles
    (the reference's layout); FP32 as the reference ships. Its tile loop is only correct for n a multiple
    of 256 (src/particles/algorithms.h:285-301)."""

    _libs = {}

    def __init__(self, variant, n):
        self.h = None
        path = ref_cuda_library_path(variant)
        if not os.path.exists(path):
            raise RuntimeError("reference CUDA build missing: %s" % path)
        if path not in RefCuda._libs:
            L = ctypes.CDLL(path)
            self.struct_type = type("RefCudaParticles", (ctypes.Structure,),
                                    {"_fields_": [(nm, ctypes.POINTER(ctypes.c_float)) for nm, _ in
                                                  OracleParticles._fields_]})
            P = ctypes.POINTER(self.struct_type)
            L.refcu_create.restype = ctypes.c_void_p
            L.refcu_create.argtypes = [ctypes.c_int64]
            L.refcu_destroy.restype = None
            L.refcu_destroy.argtypes = [ctypes.c_void_p]
            L.refcu_upload.argtypes = [ctypes.c_void_p, P]
            L.refcu_download.argtypes = [ctypes.c_void_p, P]
            L.refcu_compute_derivatives.argtypes = [ctypes.c_void_p]
            L.refcu_integrate.argtypes = [ctypes.c_void_p, ctypes.c_int]
            L.refcu_current_timestep.restype = ctypes.c_double
            L.refcu_current_timestep.argtypes = []
            L.refcu_time_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
            L.refcu_last_error.restype = ctypes.c_char_p
            L.refcu_set_timestep.argtypes = [ctypes.c_double, ctypes.c_double]
            RefCuda._libs[path] = (L, self.struct_type)
        self.lib, self.struct_type = RefCuda._libs[path]
        self.n = int(n)
        self.h = self.lib.refcu_create(self.n)
        if not self.h:
            raise RuntimeError("refcu_create: %s" % self.lib.refcu_last_error().decode())

    def close(self):
        if self.h:
            self.lib.refcu_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError("%s: %s" % (what, self.lib.refcu_last_error().decode()))

    def upload(self, state):
        from grasph2_b200.state import new_state
        full = new_state(self.n, np.float32)
        for k, a in state.items():
            if k in full:
                full[k][:] = a
        self._keep = full
        s = pointer_struct(full, self.struct_type, ctypes.c_float)
        self._check(self.lib.refcu_upload(self.h, ctypes.byref(s)), "refcu_upload")

    def download(self):
        from grasph2_b200.state import new_state
        out = new_state(self.n, np.float32)
        s = pointer_struct(out, self.struct_type, ctypes.c_float)
        self._check(self.lib.refcu_download(self.h, ctypes.byref(s)), "refcu_download")
        return out

    def compute_derivatives(self):
        self._check(self.lib.refcu_compute_derivatives(self.h), "computeDerivatives")

    def integrate(self, not_first_step=True):
        self._check(self.lib.refcu_integrate(self.h, int(not_first_step)), "integrate")

    def current_timestep(self):
        return self.lib.refcu_current_timestep()

    def set_timestep(self, current, nxt):
        self._check(self.lib.refcu_set_timestep(current, nxt), "set_timestep")

    def time_steps(self, steps):
        """Device milliseconds of `steps` x {computeDerivatives; integrate(true)} (CUDA events)."""
        ms = ctypes.c_double(0.0)
        self._check(self.lib.refcu_time_steps(self.h, int(steps), ctypes.byref(ms)), "time_steps")
        return ms.value
