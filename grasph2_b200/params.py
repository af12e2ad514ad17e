"""Runtime physics parameters (gsph_params) and the named workloads.

GraSPH2 configures its physics with `#define` switches and `constexpr` values in
settings/settings.h; here the same switches and values are fields of one struct passed through the
C-ABI. `make_params` builds it from switch names (the reference's macro names without the
ENABLE_/_LEAPFROG decoration) and keyword values; the defaults are the reference's shipped
settings (settings/settings.h:26-185).
"""

import math

from ._abi import FLAG_BITS, GsphParams, GsphOptions, ACCUM_PLAIN, ACCUM_COMPENSATED

# settings/settings.h values as shipped (H and rho0 follow :97-105 at particle_count = 1<<14)
_PRADIUS = 0.1 * (1 << 14) ** (-1.0 / 3.0)
REFERENCE_DEFAULTS = dict(
    switches=("SELF_GRAVITY", "SPH", "INTEGRATE_DENSITY", "SOLIDS", "VARIABLE_TIMESTEP", "ACCELERATION_CRITERION",
              "VELOCITY_CRITERION", "PLASTICITY_MC", "ARTIFICIAL_VISCOSITY", "BALSARA_SWITCH"),
    dimension=3,
    H=_PRADIUS * 2.5,
    grav_eps=_PRADIUS * 2.5,
    grav_G=1.0,
    rho0=1.0 / (1 << 14) / (4.0 / 3.0 * _PRADIUS ** 3 * math.pi),
    bulk=1024.0,
    dbulk_dp=1.0,
    soundspeed=None,  # sqrt(BULK / rho0), settings.h:108
    shear=128.0,
    Y=0.5,
    tanfr=math.tan(math.radians(45.0)),
    cohesion=0.0,
    av_alpha=1.0,
    av_beta=3.0,
    mateps=0.4,
    matexp=4.0,
    normalsep=None,  # H * 0.3, settings.h:166
    xsph_factor=0.5,
    fixed_dt=0.002,
    initial_dt=0.002,
    min_dt=0.00002,
    max_dt=0.02,
    accel_accuracy=0.01,
    velocity_accuracy=0.09,
    cw_n=math.sqrt(1.0 / 3.0),
    const_acc=(0.0, -1.0, 0.0),
    box_min=(-1.2, -1.2, -1.2),
    box_max=(1.2, 1.2, 1.2),
    box_reflectiveness=0.5,
)


def make_params(**kw):
    """gsph_params from keyword values; unspecified fields take the reference defaults.

    `switches` is an iterable of names from FLAG_BITS ("SELF_GRAVITY", "SPH", "SOLIDS", ...).
    `soundspeed` defaults to sqrt(bulk/rho0) and `normalsep` to 0.3*H, as in settings.h.
    """
    d = dict(REFERENCE_DEFAULTS)
    unknown = set(kw) - set(d)
    if unknown:
        raise KeyError("unknown parameter(s): %s" % sorted(unknown))
    d.update(kw)
    if "H" in kw and "grav_eps" not in kw:
        d["grav_eps"] = d["H"]
    if d["soundspeed"] is None:
        d["soundspeed"] = math.sqrt(d["bulk"] / d["rho0"])
    if d["normalsep"] is None:
        d["normalsep"] = d["H"] * 0.3
    p = GsphParams()
    flags = 0
    for s in d.pop("switches"):
        if s not in FLAG_BITS:
            raise KeyError("unknown switch %r" % s)
        flags |= FLAG_BITS[s]
    p.flags = flags
    for k, v in d.items():
        if k in ("const_acc", "box_min", "box_max"):
            getattr(p, k)[:] = [float(x) for x in v]
        elif k == "dimension":
            p.dimension = int(v)
        else:
            setattr(p, k, float(v))
    return p


def params_to_dict(p):
    out = {"switches": tuple(s for s, b in FLAG_BITS.items() if p.flags & b)}
    for name, _ in GsphParams._fields_:
        if name == "flags":
            continue
        v = getattr(p, name)
        out[name] = tuple(v) if name in ("const_acc", "box_min", "box_max") else v
    return out


def make_options(accum="plain", j_split=0, j_tile=0, i_per_thread=0, threads=0, check_finite=0, cull=True,
                 resort_interval=0, scalar_fp32=False, precision="single", gravity="auto", gravity_groups=0,
                 wait_limit_us=0):
    o = GsphOptions()
    o.accum = {"plain": ACCUM_PLAIN, "compensated": ACCUM_COMPENSATED}[accum] if isinstance(accum, str) else accum
    o.j_split, o.j_tile, o.i_per_thread, o.threads, o.check_finite = j_split, j_tile, i_per_thread, threads, check_finite
    o.no_cull = 0 if cull else 1
    o.resort_interval = resort_interval
    o.scalar_fp32 = 1 if scalar_fp32 else 0
    o.precision = {"single": 0, "double": 1}[precision] if isinstance(precision, str) else int(precision)
    o.gravity_form = {"auto": 0, "one-sided": 1, "symmetric": 2}[gravity] if isinstance(gravity, str) else int(gravity)
    o.gravity_groups = gravity_groups
    o.wait_limit_us = wait_limit_us
    return o


# ---- the named workloads ------------------------------------------------------------------------
def config0_params():
    """SPH + self-gravity fluid sphere, N=4096: G=1, eps=0.02, h=0.15, liquid EOS c=1, rho0=0.239,
    density by summation, no stress, no AV, fixed dt=1e-3."""
    return make_params(switches=("SELF_GRAVITY", "SPH"), H=0.15, grav_eps=0.02, rho0=0.239, bulk=0.239,
                       soundspeed=1.0, fixed_dt=1e-3)


def impact_smoothing_length(n_big=58254, r_big=1.0, n_small=7282, r_small=0.5):
    """h = 2.5 x mean particle spacing (V/N)^(1/3) of the two-sphere impact."""
    v = 4.0 / 3.0 * math.pi * (r_big ** 3 + r_small ** 3)
    return 2.5 * (v / (n_big + n_small)) ** (1.0 / 3.0)


def config1_params():
    """Elastic-plastic impact, N=65536: rho0=1, Murnaghan K=10 dK0=1, shear=5, Hooke + Jaumann,
    von Mises Y=0.5, AV alpha=1 beta=2, h=2.5 x mean spacing, G=1 eps=0.01, dt=1e-4, density by
    summation."""
    return make_params(switches=("SELF_GRAVITY", "SPH", "SOLIDS", "ARTIFICIAL_VISCOSITY", "PLASTICITY_MIESE"),
                       H=impact_smoothing_length(), grav_eps=0.01, rho0=1.0, bulk=10.0, dbulk_dp=1.0,
                       soundspeed=math.sqrt(10.0), shear=5.0, Y=0.5, av_alpha=1.0, av_beta=2.0, fixed_dt=1e-4)


CONFIG4_N_BIG, CONFIG4_N_SMALL = 233017, 29127  # N = 262,144 split 8:1 like the 65,536 impact (equal number density)


def impact_params(n_big, n_small, **over):
    """The elastic-plastic impact physics (as the N=65,536 impact) for another particle count: h = 2.5 x
    the mean spacing of n_big + n_small particles in spheres of radius 1 and 0.5."""
    kw = dict(switches=("SELF_GRAVITY", "SPH", "SOLIDS", "ARTIFICIAL_VISCOSITY", "PLASTICITY_MIESE"),
              H=impact_smoothing_length(n_big, 1.0, n_small, 0.5), grav_eps=0.01, rho0=1.0, bulk=10.0, dbulk_dp=1.0,
              soundspeed=math.sqrt(10.0), shear=5.0, Y=0.5, av_alpha=1.0, av_beta=2.0, fixed_dt=1e-4)
    kw.update(over)
    return make_params(**kw)


def config4_params():
    """The elastic-plastic impact physics at N=262,144 (h = 2.5 x mean spacing = 0.0655), for the learned
    surrogate: rho0=1, Murnaghan K=10 dK0=1, shear=5, von Mises Y=0.5, AV alpha=1 beta=2, G=1 eps=0.01,
    dt=1e-4."""
    return make_params(switches=("SELF_GRAVITY", "SPH", "SOLIDS", "ARTIFICIAL_VISCOSITY", "PLASTICITY_MIESE"),
                       H=impact_smoothing_length(CONFIG4_N_BIG, 1.0, CONFIG4_N_SMALL, 0.5), grav_eps=0.01, rho0=1.0,
                       bulk=10.0, dbulk_dp=1.0, soundspeed=math.sqrt(10.0), shear=5.0, Y=0.5, av_alpha=1.0,
                       av_beta=2.0, fixed_dt=1e-4)


def config2_params():
    """Pure N-body Plummer sphere, N=1,048,576: G=1, eps=0.01, dt=1e-3."""
    return make_params(switches=("SELF_GRAVITY",), H=0.01, grav_eps=0.01, fixed_dt=1e-3)
