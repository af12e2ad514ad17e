"""Physics variants of the reference's CPU parity build (test infrastructure only).

GraSPH2's settings are compile-time constants (settings/settings.h), so each variant below is one
build of the reference's job headers (oracle/ref_driver.cpp -> oracle/_ref/libref_<name>_<fp>.so).
The same table gives the runtime parameter set of the oracle and of the CUDA library, so the tests
compare all three on identical physics. Gravity softening equals H in every variant, because the
reference hard-wires eps == H (src/computeDerivatives.h:231); the AV signal coefficient is 3 for the
same reason (src/sph/models.h:179).
"""

import math

# switch name -> flag bit name in include/grasph2_b200.h
SWITCHES = [
    "SELF_GRAVITY", "SPH", "INTEGRATE_DENSITY", "DEAL_WITH_NO_PARTNERS", "SOLIDS",
    "VARIABLE_TIMESTEP", "ACCELERATION_CRITERION", "VELOCITY_CRITERION", "PLASTICITY_MIESE",
    "PLASTICITY_MC", "CLOHESSY_WILTSHIRE", "CONSTANT_ACCELERATION", "SIMPLE_BOX_BOUNDARY",
    "ARTIFICIAL_VISCOSITY", "BALSARA_SWITCH", "ARTIFICIAL_STRESS", "XSPH",
]

_BASE = dict(
    H=0.2, rho0=1.0, bulk=10.0, dbulk_dp=1.0, soundspeed=math.sqrt(10.0), shear=5.0, Y=0.5,
    tanfr=1.0, cohesion=0.0, av_alpha=1.0, mateps=0.4, matexp=4.0, normalsep_frac=0.3, xsph_factor=0.5,
    fixed_dt=1e-3, initial_dt=1e-3, min_dt=1e-5, max_dt=2e-2, accel_accuracy=0.01, velocity_accuracy=0.09,
    cw_n=math.sqrt(1.0 / 3.0), const_acc=(0.0, -1.0, 0.0), box_min=-1.2, box_max=1.2, box_reflectiveness=0.5,
)


def _v(name, switches, **over):
    d = dict(_BASE)
    d.update(over)
    d["name"] = name
    d["switches"] = tuple(switches)
    return d


VARIANTS = {
    # config-0 physics: gravity + SPH fluid, liquid EOS, density by summation, no AV, fixed step
    "fluid": _v("fluid", ["SELF_GRAVITY", "SPH"], H=0.3, rho0=0.239, bulk=0.239, soundspeed=1.0),
    # config-1 physics: elastic-plastic solid, Murnaghan EOS, summed density, AV, von Mises
    "solid": _v("solid", ["SELF_GRAVITY", "SPH", "SOLIDS", "ARTIFICIAL_VISCOSITY", "PLASTICITY_MIESE"],
                H=0.42, Y=0.05),
    # the reference's shipped defaults: integrated density, Balsara, Mohr-Coulomb, variable step
    "solid_mc": _v("solid_mc", ["SELF_GRAVITY", "SPH", "SOLIDS", "INTEGRATE_DENSITY", "ARTIFICIAL_VISCOSITY",
                                "BALSARA_SWITCH", "PLASTICITY_MC", "VARIABLE_TIMESTEP", "ACCELERATION_CRITERION",
                                "VELOCITY_CRITERION"], H=0.42),
    # fluid with every optional correction the reference offers
    "fluid_full": _v("fluid_full", ["SELF_GRAVITY", "SPH", "INTEGRATE_DENSITY", "ARTIFICIAL_VISCOSITY",
                                    "BALSARA_SWITCH", "ARTIFICIAL_STRESS", "XSPH", "CONSTANT_ACCELERATION",
                                    "SIMPLE_BOX_BOUNDARY"], H=0.3, rho0=0.239, bulk=0.239, soundspeed=1.0,
                     box_min=-0.9, box_max=0.9),
    # the elastic-plastic impact workload at full size (N = 65536, h = 2.5 x mean spacing), as far
    # as the reference can express it (eps == H, AV signal coefficient 3): the CPU timing baseline
    "impact": _v("impact", ["SELF_GRAVITY", "SPH", "SOLIDS", "ARTIFICIAL_VISCOSITY", "PLASTICITY_MIESE"],
                 H=2.5 * (4.0 / 3.0 * math.pi * 1.125 / 65536) ** (1.0 / 3.0), fixed_dt=1e-4),
    # pure N-body (softening == H in the reference)
    "nbody": _v("nbody", ["SELF_GRAVITY"], H=0.05),
    # config-2 physics: the Plummer sphere's softening eps = 0.01 (== H), dt = 1e-3
    "plummer": _v("plummer", ["SELF_GRAVITY"], H=0.01, fixed_dt=1e-3),
    # gravity with the environment terms (Clohessy-Wiltshire, constant acceleration) and the box
    "nbody_env": _v("nbody_env", ["SELF_GRAVITY", "CLOHESSY_WILTSHIRE", "CONSTANT_ACCELERATION",
                                  "SIMPLE_BOX_BOUNDARY"], H=0.05, box_min=-0.95, box_max=0.95),
}


def compile_defines(v, double):
    """-D flags that configure oracle/ref_shim/settings.h for variant `v`."""
    d = ["-DREF_VARIANT_NAME=\"%s_%s\"" % (v["name"], "fp64" if double else "fp32")]
    if double:
        d.append("-DREF_DOUBLE=1")
    for s in SWITCHES:
        key = {"SELF_GRAVITY": "GRAVITY"}.get(s, s)
        if s == "VARIABLE_TIMESTEP":
            continue  # the driver picks the fixed or variable dispatch at run time
        d.append("-DREF_%s=%d" % (key, 1 if s in v["switches"] else 0))
    num = dict(FIXED_DT=v["fixed_dt"], INITIAL_DT=v["initial_dt"], MIN_DT=v["min_dt"], MAX_DT=v["max_dt"],
               ACCEL_ACCURACY=v["accel_accuracy"], VELOCITY_ACCURACY=v["velocity_accuracy"], H=v["H"],
               RHO0=v["rho0"], BULK=v["bulk"], DBULKDP=v["dbulk_dp"], SOUNDSPEED=v["soundspeed"], SHEAR=v["shear"],
               Y=v["Y"], TANFR=v["tanfr"], COHESION=v["cohesion"], CW_N=v["cw_n"], CONST_ACC_X=v["const_acc"][0],
               CONST_ACC_Y=v["const_acc"][1], CONST_ACC_Z=v["const_acc"][2], BOX_MIN=v["box_min"],
               BOX_MAX=v["box_max"], BOX_REFLECT=v["box_reflectiveness"], ALPHA=v["av_alpha"],
               MATEPS=v["mateps"], MATEXP=v["matexp"], NORMALSEP_FRAC=v["normalsep_frac"],
               XSPH_FACTOR=v["xsph_factor"])
    for k, val in num.items():
        d.append("-DREF_%s=%r" % (k, float(val)))
    return d


def params_dict(v):
    """Runtime parameter set (field names of gsph_params) equal to variant `v`."""
    return dict(
        switches=v["switches"], dimension=3, H=v["H"], grav_eps=v["H"], grav_G=1.0, rho0=v["rho0"], bulk=v["bulk"],
        dbulk_dp=v["dbulk_dp"], soundspeed=v["soundspeed"], shear=v["shear"], Y=v["Y"], tanfr=v["tanfr"],
        cohesion=v["cohesion"], av_alpha=v["av_alpha"], av_beta=3.0, mateps=v["mateps"], matexp=v["matexp"],
        normalsep=v["H"] * v["normalsep_frac"], xsph_factor=v["xsph_factor"], fixed_dt=v["fixed_dt"],
        initial_dt=v["initial_dt"], min_dt=v["min_dt"], max_dt=v["max_dt"], accel_accuracy=v["accel_accuracy"],
        velocity_accuracy=v["velocity_accuracy"], cw_n=v["cw_n"], const_acc=tuple(v["const_acc"]),
        box_min=(v["box_min"],) * 3, box_max=(v["box_max"],) * 3, box_reflectiveness=v["box_reflectiveness"],
    )
