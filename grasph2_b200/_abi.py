"""ctypes mirror of include/grasph2_b200.h (structs, flags, status codes) and the library loader.

The shared library is built in-tree by grasph2_b200/build.py into grasph2_b200/lib/libgrasph2_b200.so.
Loading fails loudly when it is missing: there is no CPU fallback in this package.
"""

import ctypes
import os

c_double3 = ctypes.c_double * 3

# ---- status codes -------------------------------------------------------------------------------
GSPH_OK = 0
GSPH_E_INVALID = -1
GSPH_E_CUDA = -2
GSPH_E_NOMEM = -3
GSPH_E_STATE = -4
GSPH_E_NUMERIC = -5
GSPH_E_TIMEOUT = -6
GSPH_E_UNSUPPORTED = -7
STATUS_NAMES = {0: "GSPH_OK", -1: "GSPH_E_INVALID", -2: "GSPH_E_CUDA", -3: "GSPH_E_NOMEM", -4: "GSPH_E_STATE",
                -5: "GSPH_E_NUMERIC", -6: "GSPH_E_TIMEOUT", -7: "GSPH_E_UNSUPPORTED"}

# ---- physics switches (settings/settings.h #defines) --------------------------------------------
FLAG_BITS = {
    "SELF_GRAVITY": 1 << 0, "SPH": 1 << 1, "INTEGRATE_DENSITY": 1 << 2, "DEAL_WITH_NO_PARTNERS": 1 << 3,
    "SOLIDS": 1 << 4, "VARIABLE_TIMESTEP": 1 << 5, "ACCELERATION_CRITERION": 1 << 6,
    "VELOCITY_CRITERION": 1 << 7, "PLASTICITY_MIESE": 1 << 8, "PLASTICITY_MC": 1 << 9,
    "CLOHESSY_WILTSHIRE": 1 << 10, "CONSTANT_ACCELERATION": 1 << 11, "SIMPLE_BOX_BOUNDARY": 1 << 12,
    "ARTIFICIAL_VISCOSITY": 1 << 13, "BALSARA_SWITCH": 1 << 14, "ARTIFICIAL_STRESS": 1 << 15, "XSPH": 1 << 16,
}
ALL_FLAGS = (1 << 17) - 1

# ---- particle attributes (particle_bases order) -------------------------------------------------
ATTRIBUTES = [  # name, bit, components
    ("pos", 1 << 0, 3), ("mass", 1 << 1, 1), ("vel", 1 << 2, 3), ("acc", 1 << 3, 3), ("balsara", 1 << 4, 1),
    ("xvel", 1 << 5, 3), ("density", 1 << 6, 1), ("density_dt", 1 << 7, 1), ("dstress", 1 << 8, 9),
    ("dstress_dt", 1 << 9, 9), ("maxvsig", 1 << 10, 1),
]
ATTR_BITS = {name: bit for name, bit, _ in ATTRIBUTES}
ATTR_COMPONENTS = {name: k for name, _, k in ATTRIBUTES}
ALL_ATTRIBS = (1 << 11) - 1

ACCUM_PLAIN = 0
ACCUM_COMPENSATED = 1


class GsphParams(ctypes.Structure):
    _fields_ = [
        ("flags", ctypes.c_uint32), ("dimension", ctypes.c_int32),
        ("H", ctypes.c_double), ("grav_eps", ctypes.c_double), ("grav_G", ctypes.c_double),
        ("rho0", ctypes.c_double), ("bulk", ctypes.c_double), ("dbulk_dp", ctypes.c_double),
        ("soundspeed", ctypes.c_double), ("shear", ctypes.c_double), ("Y", ctypes.c_double),
        ("tanfr", ctypes.c_double), ("cohesion", ctypes.c_double), ("av_alpha", ctypes.c_double),
        ("av_beta", ctypes.c_double), ("mateps", ctypes.c_double), ("matexp", ctypes.c_double),
        ("normalsep", ctypes.c_double), ("xsph_factor", ctypes.c_double), ("fixed_dt", ctypes.c_double),
        ("initial_dt", ctypes.c_double), ("min_dt", ctypes.c_double), ("max_dt", ctypes.c_double),
        ("accel_accuracy", ctypes.c_double), ("velocity_accuracy", ctypes.c_double), ("cw_n", ctypes.c_double),
        ("const_acc", c_double3), ("box_min", c_double3), ("box_max", c_double3),
        ("box_reflectiveness", ctypes.c_double),
    ]


class GsphOptions(ctypes.Structure):
    _fields_ = [
        ("accum", ctypes.c_int32), ("j_split", ctypes.c_int32), ("j_tile", ctypes.c_int32),
        ("i_per_thread", ctypes.c_int32), ("threads", ctypes.c_int32), ("check_finite", ctypes.c_int32),
        ("no_cull", ctypes.c_int32), ("resort_interval", ctypes.c_int32), ("scalar_fp32", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("gravity_form", ctypes.c_int32), ("gravity_groups", ctypes.c_int32),
        ("wait_limit_us", ctypes.c_int32), ("reserved", ctypes.c_int32 * 3),
    ]


_fp = ctypes.POINTER(ctypes.c_float)


class GsphHostParticles(ctypes.Structure):
    _fields_ = [(name, _fp) for name, _, _ in ATTRIBUTES]


_dp = ctypes.POINTER(ctypes.c_double)


class GsphLaunchShape(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in ("cull", "grav_ipt", "grav_jt", "grav_nseg", "grav_x2", "sph_threads",
                                               "sph_jt", "sph_nseg", "items", "grav_sym_groups")] + \
        [("reserved", ctypes.c_int32 * 6)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class GsphHostParticles64(ctypes.Structure):
    """gsph_host_particles64: the double-precision host buffers."""
    _fields_ = [(name, _dp) for name, _, _ in ATTRIBUTES]


OracleParticles = GsphHostParticles64  # same layout; the oracle bindings use it for their FP64 arrays


class GsphDiag(ctypes.Structure):
    _fields_ = [
        ("e_kin", ctypes.c_double), ("e_grav", ctypes.c_double), ("e_int", ctypes.c_double),
        ("e_shear", ctypes.c_double), ("momentum", c_double3), ("ang_mom", c_double3), ("mass", ctypes.c_double),
    ]

    def as_dict(self):
        return dict(e_kin=self.e_kin, e_grav=self.e_grav, e_int=self.e_int, e_shear=self.e_shear,
                    momentum=tuple(self.momentum), ang_mom=tuple(self.ang_mom), mass=self.mass,
                    e_total=self.e_kin + self.e_grav + self.e_int + self.e_shear)


KSLOTS = 6
KSLOT_NAMES = ("density", "vgrad", "pairs", "gravity", "step", "integrate")


class GsphProfile(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double * KSLOTS), ("launches", ctypes.c_int64 * KSLOTS)]


class GsphIcOp(ctypes.Structure):
    """gsph_ic_op"""
    _fields_ = [("kind", ctypes.c_int32), ("attr", ctypes.c_uint32), ("seed", ctypes.c_uint64),
                ("v", ctypes.c_double * 9)]


IC_MOVE, IC_ROTATE, IC_POS_NOISE, IC_ANGULAR_VEL, IC_LINEAR_VEL, IC_RANDOM_VEL, IC_SET_CONSTANT = range(1, 8)
IC_MAX_OPS = 16


class GsphDeviceView(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("posm", ctypes.c_void_p), ("velrho", ctypes.c_void_p),
                ("acc", ctypes.c_void_p), ("pos64", ctypes.c_void_p)]


PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PACKAGE_DIR, "lib", "libgrasph2_b200.so")

_lib = None

_SIGNATURES = {
    "gsph_params_reference_defaults": (ctypes.c_int, [ctypes.POINTER(GsphParams)]),
    "gsph_params_validate": (ctypes.c_int, [ctypes.POINTER(GsphParams), ctypes.c_char_p, ctypes.c_size_t]),
    "gsph_options_defaults": (ctypes.c_int, [ctypes.POINTER(GsphOptions)]),
    "gsph_create": (ctypes.c_int, [ctypes.POINTER(GsphParams), ctypes.POINTER(GsphOptions), ctypes.c_int64,
                                   ctypes.POINTER(ctypes.c_void_p)]),
    "gsph_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "gsph_upload": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(GsphHostParticles),
                                   ctypes.c_void_p]),
    "gsph_download": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(GsphHostParticles),
                                     ctypes.c_void_p]),
    "gsph_upload_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(GsphHostParticles),
                                          ctypes.c_void_p]),
    "gsph_ic_uniform_sphere": (ctypes.c_int, [ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                              ctypes.POINTER(ctypes.c_double), ctypes.c_uint64, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "gsph_ic_plummer": (ctypes.c_int, [ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]),
    "gsph_ic_com_correct": (ctypes.c_int, [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p]),
    "gsph_ic_com_set": (ctypes.c_int, [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _dp, _dp,
                                       ctypes.c_void_p, ctypes.c_void_p]),
    "gsph_ic_modify": (ctypes.c_int, [ctypes.c_int64, ctypes.POINTER(GsphIcOp), ctypes.c_int32,
                                      ctypes.POINTER(GsphHostParticles), _dp, _dp, ctypes.c_void_p]),
    "gsph_upload_f64": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(GsphHostParticles64),
                                       ctypes.c_void_p]),
    "gsph_download_f64": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(GsphHostParticles64),
                                         ctypes.c_void_p]),
    "gsph_upload_pos64": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_void_p]),
    "gsph_download_pos64": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_void_p]),
    "gsph_compute_derivatives": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "gsph_integrate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "gsph_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    "gsph_current_timestep": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_void_p]),
    "gsph_diagnostics": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(GsphDiag),
                                        ctypes.c_void_p]),
    "gsph_diagnostics_fast": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(GsphDiag),
                                             ctypes.c_void_p]),
    "gsph_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    "gsph_launch_shape_get": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GsphLaunchShape)]),
    "gsph_size": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    "gsph_reorder": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "gsph_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "gsph_device_view_get": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GsphDeviceView)]),
    "gsph_launch_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    "gsph_profile_enable": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "gsph_profile_collect": (ctypes.c_int, [ctypes.c_void_p]),
    "gsph_profile_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GsphProfile)]),
    "gsph_profile_reset": (ctypes.c_int, [ctypes.c_void_p]),
    "gsph_measure_fp32_peak": (ctypes.c_int, [ctypes.c_double, ctypes.POINTER(ctypes.c_double)]),
    "gsph_ensemble_create": (ctypes.c_int, [ctypes.POINTER(GsphParams), ctypes.POINTER(GsphOptions), ctypes.c_int32,
                                            ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_void_p)]),
    "gsph_ensemble_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "gsph_ensemble_offsets": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    "gsph_ensemble_upload": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(GsphHostParticles),
                                            ctypes.c_void_p]),
    "gsph_ensemble_download": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(GsphHostParticles),
                                              ctypes.c_void_p]),
    "gsph_ensemble_upload_pos64": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "gsph_ensemble_download_pos64": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                                    ctypes.c_void_p]),
    "gsph_ensemble_compute_derivatives": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "gsph_ensemble_integrate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    "gsph_ensemble_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    "gsph_ensemble_diagnostics": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(GsphDiag),
                                                 ctypes.c_void_p]),
    "gsph_ensemble_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                              ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p]),
    "gsph_ensemble_launch_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    "gsph_ensemble_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "gsph_ensemble_inject_stall": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "gsph_tc_gemm_check": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                          ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "gsph_surrogate_features": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_void_p]),
    "gsph_surrogate_apply": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_int32, ctypes.c_void_p]),
    "gsph_snapshot": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    "gsph_state_compare": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, _dp, ctypes.c_void_p]),
    "gsph_h5_available": (ctypes.c_int, []),
    "gsph_h5_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int64, ctypes.POINTER(GsphHostParticles),
                                     ctypes.c_uint32]),
    "gsph_h5_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint32, ctypes.POINTER(GsphHostParticles),
                                    ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "gsph_writer_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int32,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "gsph_writer_write": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]),
    "gsph_writer_flush": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    "gsph_writer_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "gsph_writer_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "gsph_mlp_param_count": (ctypes.c_int64, []),
    "gsph_mlp_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_void_p)]),
    "gsph_mlp_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "gsph_mlp_get_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "gsph_mlp_set_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "gsph_mlp_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                        ctypes.c_void_p]),
    "gsph_mlp_gradient": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_int64, ctypes.POINTER(ctypes.c_float),
                                         ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "gsph_mlp_adam": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                     ctypes.c_void_p]),
    "gsph_mlp_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "gsph_mlp_set_grad_clip": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_float]),
    "gsph_gravity_accel_static": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_void_p, ctypes.c_void_p]),
    "gsph_gravity_accel_static_status": (ctypes.c_int, [ctypes.c_void_p]),
    "gsph_inject_static_timeout": (ctypes.c_int, [ctypes.c_int]),
    "gsph_surrogate_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_float)] * 5 +
                              [ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    "gsph_surrogate_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    "gsph_surrogate_save": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "gsph_surrogate_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "gsph_surrogate_mlp": (ctypes.c_void_p, [ctypes.c_void_p]),
    "gsph_surrogate_substeps": (ctypes.c_int32, [ctypes.c_void_p]),
    "gsph_surrogate_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "gsph_surrogate_propose": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    "gsph_surrogate_judge": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_double,
                                            ctypes.c_void_p, ctypes.c_void_p]),
    "gsph_surrogate_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                              ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_void_p,
                                              ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p]),
    "gsph_surrogate_launch_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    "gsph_surrogate_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "gsph_surrogate_set_energy_correction": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_double]),
    "gsph_surrogate_energy_bias": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "gsph_state_compare_parts": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, _dp,
                                                ctypes.c_void_p]),
    "gsph_energy_adjust": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
}


class SurrogateWindow(ctypes.Structure):
    """gsph_surrogate_window"""
    _fields_ = [("pos_error", ctypes.c_double), ("energy_error", ctypes.c_double),
                ("energy_parts", ctypes.c_double * 4), ("accepted", ctypes.c_int32), ("reserved", ctypes.c_int32)]


def load_library(path=None):
    """Load libgrasph2_b200.so (once) and declare its signatures. Raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("grasph2_b200: CUDA library not built (%s missing); run "
                           "`python -c 'import __graft_entry__ as g; g.build()'` or grasph2_b200/build.py" % p)
    lib = ctypes.CDLL(p)
    for name, (res, args) in _SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def exported_symbols():
    return sorted(_SIGNATURES)
