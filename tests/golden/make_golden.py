"""Generate tests/golden/*.npz from GraSPH2's own hot-path code.

    python tests/golden/make_golden.py

For every physics variant of oracle/ref_variants.py it builds (or reuses) oracle/_ref/libref_*.so --
the reference's src/computeDerivatives.h, src/integration.h and src/sph/*.h compiled for the host --
and records, for a seeded particle set:

  in_*        the input state (float32-representable values, stored as float64)
  d64_*       the state after one computeDerivatives() of the FP64 reference build
  s64_*       the state after 3 x {computeDerivatives(); integrate(notFirstStep=true)} (FP64 build)
  d32_*       the state after one computeDerivatives() of the FP32 build (the reference as shipped)
  dt64        for variable-step variants: currentTS after each of the 3 steps

The reference tree is needed only here; the fixtures are committed so that the tests run without it.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import build_ref  # noqa: E402
import pyoracle  # noqa: E402
import ref_variants  # noqa: E402
from grasph2_b200 import ics  # noqa: E402
from grasph2_b200.state import as_dtype, copy_state  # noqa: E402

N = 256
STEPS = 3


def golden_input(name, n=N, seed=7):
    """Seeded input state of variant `name`, rounded to float32-representable values."""
    v = ref_variants.VARIANTS[name]
    rng = np.random.default_rng(seed)
    if name == "plummer":
        st = ics.plummer_sphere(n, seed=seed)
    elif "SOLIDS" in v["switches"]:
        nb = (n * 8) // 9
        st = ics.two_sphere_impact(n_big=nb, n_small=n - nb, v_rel=0.5, y_offset=0.3, rho0=v["rho0"], seed=seed)
        S = rng.normal(size=(n, 3, 3)) * 0.05
        st["dstress"][:] = 0.5 * (S + S.transpose(0, 2, 1))
        st["density"][:] = v["rho0"] * (1.0 + 0.02 * rng.normal(size=n))
    else:
        st = ics.uniform_sphere(n, radius=1.0, rho0=v["rho0"], omega=(0.0, 0.0, 0.3), seed=seed)
        st["density"][:] = v["rho0"] * (1.0 + 0.02 * rng.normal(size=n))
    st["vel"] += 0.02 * rng.normal(size=(n, 3))  # no exactly rigid motion: keeps v_ij . r_ij away from 0
    st = as_dtype(as_dtype(st, np.float32), np.float64)
    return st


def run(name):
    v = ref_variants.VARIANTS[name]
    variable = "VARIABLE_TIMESTEP" in v["switches"]
    st = golden_input(name)
    out = {"in_" + k: a for k, a in st.items()}
    r64 = pyoracle.RefBuild(name, True)
    r32 = pyoracle.RefBuild(name, False)

    d = copy_state(st)
    r64.lib.ref_set_timestep(0.0, 0.0)
    r64.compute_derivatives(d)
    out.update({"d64_" + k: a for k, a in d.items()})

    d32 = as_dtype(st, np.float32)
    r32.lib.ref_set_timestep(0.0, 0.0)
    r32.compute_derivatives(d32)
    out.update({"d32_" + k: a.astype(np.float32) for k, a in d32.items()})

    s = copy_state(st)
    r64.lib.ref_set_timestep(0.0, 0.0)
    dts = []
    for _ in range(STEPS):
        r64.compute_derivatives(s)
        r64.integrate(s, True, variable)
        dts.append(r64.lib.ref_current_timestep() if variable else r64.lib.ref_fixed_timestep())
    out.update({"s64_" + k: a for k, a in s.items()})
    out["dt64"] = np.array(dts)
    out["variant"] = np.array(name)
    return out


def main(names=None):
    build_ref.build_oracle()
    build_ref.build_ref()
    for name in names or ref_variants.VARIANTS:
        out = run(name)
        path = os.path.join(HERE, "ref_%s.npz" % name)
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main(sys.argv[1:])
