"""Batched ensemble (gsph_ensemble_*): every simulation of the batch against the FP64 oracle run on that
simulation alone, with the condition-aware bound of the single-simulation tests (tests/test_gpu_parity.py):
|x_gpu - x_ref| <= TOL * max|x_ref| + 32 * s, s the oracle's change under a one-ulp float32 perturbation.
"""

import numpy as np
import pytest

import ref_variants
from grasph2_b200 import ics
from grasph2_b200._abi import FLAG_BITS as F
from grasph2_b200.params import config0_params, make_options, make_params
from grasph2_b200.sim import DeviceParticleBuffer, Ensemble, GsphError, pack_states
from grasph2_b200.state import copy_state
from helpers import check_within, f32_exact, fp32_sensitivity

pytestmark = pytest.mark.gpu

TOL_ACC = 1e-5
TOL_RHO = 1e-6
TOL_RATE = 1e-5
TOL_STEP = 1e-5


def variant_params(name, drop=()):
    d = ref_variants.params_dict(ref_variants.VARIANTS[name])
    d["switches"] = tuple(s for s in d["switches"] if s not in drop)
    return make_params(**d)


# ensemble-capable physics: no Balsara switch, fixed step
VARIANTS = {
    "fluid": lambda: variant_params("fluid"),
    "solid": lambda: variant_params("solid"),
    "nbody": lambda: variant_params("nbody"),
    "nbody_env": lambda: variant_params("nbody_env"),
    "fluid_full": lambda: variant_params("fluid_full", drop=("BALSARA_SWITCH",)),
    "solid_mc": lambda: variant_params("solid_mc", drop=("BALSARA_SWITCH", "VARIABLE_TIMESTEP")),
}


def sim_state(n, seed, rho0=1.0, omega=0.3):
    rng = np.random.default_rng(seed)
    st = ics.uniform_sphere(n, radius=1.0, rho0=rho0, omega=(0.0, 0.0, omega), seed=seed)
    st["vel"] += 0.02 * rng.normal(size=(n, 3))
    st["density"][:] = rho0 * (1 + 0.02 * rng.normal(size=n))
    S = rng.normal(size=(n, 3, 3)) * 0.05
    st["dstress"][:] = 0.5 * (S + S.transpose(0, 2, 1))
    return f32_exact(st)


def fields(p):
    f = {"acc": TOL_ACC}
    if p.flags & F["SPH"]:
        f["density"] = TOL_RHO
        if p.flags & (F["SOLIDS"] | F["INTEGRATE_DENSITY"]):
            f.update(dstress_dt=TOL_RATE, density_dt=TOL_RATE)
        if p.flags & F["XSPH"]:
            f["xvel"] = TOL_RATE
    return f


def oracle_derivs(oracle, p):
    def run(st):
        oracle.ts.current = oracle.ts.next = 0.0
        oracle.compute_derivatives(p, st)
        return st
    return run


def oracle_steps(oracle, p, nsteps):
    def run(st):
        x0 = st["pos"].copy()
        oracle.ts.current = oracle.ts.next = 0.0
        for _ in range(nsteps):
            oracle.compute_derivatives(p, st)
            oracle.integrate(p, st, True)
        st["disp"] = st["pos"] - x0
        return st
    return run


SIZES = [1, 2, 100, 511, 512, 513, 1500, 3000]


@pytest.mark.parametrize("gravity", ["auto", "symmetric"])
@pytest.mark.parametrize("accum", ["plain", "compensated"])
@pytest.mark.parametrize("name", list(VARIANTS))
def test_ensemble_derivatives_vs_oracle(oracle, name, accum, gravity):
    """Every simulation against the oracle; with gravity and SPH, `auto` is the one-sided sweep fused with
    the density pass and `symmetric` the stage of group pairs (512-particle groups, ragged last groups: the
    sizes straddle 512)."""
    p = VARIANTS[name]()
    rho0 = p.rho0
    states = [sim_state(n, seed=100 + k, rho0=rho0, omega=0.1 * k) for k, n in enumerate(SIZES)]
    with Ensemble(p, SIZES, make_options(accum=accum, gravity=gravity)) as ens:
        ens.upload(pack_states(states))
        ens.compute_derivatives()
        got = ens.split(ens.download())
    for k, st in enumerate(states):
        ref, sens = fp32_sensitivity(oracle_derivs(oracle, p), st, trials=1)
        for f, tol in fields(p).items():
            check_within(got[k][f], ref[f], sens[f], tol, "%s/%s/%s sim %d (n=%d) %s" % (name, accum, gravity, k,
                                                                                         SIZES[k], f))


@pytest.mark.parametrize("name", ["fluid", "solid", "nbody", "solid_mc"])
def test_ensemble_three_steps_vs_oracle(oracle, name):
    p = VARIANTS[name]()
    sizes = [300, 1025, 2000]
    states = [sim_state(n, seed=200 + k, rho0=p.rho0, omega=0.2) for k, n in enumerate(sizes)]
    with Ensemble(p, sizes) as ens:
        ens.upload(pack_states(states))
        for _ in range(3):
            ens.compute_derivatives()
            ens.integrate(True)
        got = ens.split(ens.download())
        pos64 = ens.download_pos64()
    for k, st in enumerate(states):
        ref, sens = fp32_sensitivity(oracle_steps(oracle, p, 3), st, trials=1)
        what = "%s sim %d" % (name, k)
        x = pos64[ens.offsets[k]:ens.offsets[k + 1]]
        check_within(x - st["pos"], ref["disp"], sens["disp"], TOL_STEP, what + " displacement")
        for f in ("vel", "density", "dstress"):
            if np.abs(ref[f]).max() > 0:
                check_within(got[k][f], ref[f], sens[f], TOL_STEP, what + " " + f)


def test_ensemble_neighbour_overflow(oracle):
    """More than 256 neighbours per particle: the SPH stage falls back to sweeping the simulation."""
    p = make_params(switches=("SELF_GRAVITY", "SPH", "SOLIDS", "ARTIFICIAL_VISCOSITY"), H=1.2, grav_eps=0.05,
                    rho0=1.0, bulk=10.0, soundspeed=3.0, shear=5.0)
    sizes = [700, 90]
    states = [sim_state(n, seed=300 + k) for k, n in enumerate(sizes)]
    with Ensemble(p, sizes) as ens:
        ens.upload(pack_states(states))
        ens.compute_derivatives()
        got = ens.split(ens.download())
    for k, st in enumerate(states):
        ref, sens = fp32_sensitivity(oracle_derivs(oracle, p), st, trials=1)
        for f, tol in fields(p).items():
            # every particle is a neighbour here: the density is a plain FP32 sum of ~700 terms
            tol = 5e-6 if f == "density" else tol
            check_within(got[k][f], ref[f], sens[f], tol, "overflow sim %d %s" % (k, f))


def test_ensemble_graph_step_matches_eager():
    p = config0_params()
    sizes = [1024, 3000, 1500, 5000]
    states = [sim_state(n, seed=400 + k, rho0=0.239, omega=0.1 * k) for k, n in enumerate(sizes)]
    packed = pack_states(states)
    with Ensemble(p, sizes) as a, Ensemble(p, sizes) as b:
        a.upload(packed)
        b.upload(packed)
        for _ in range(3):
            a.compute_derivatives()
            a.integrate(True)
        b.step(3)
        x, y = a.download(), b.download()
    for k in x:
        np.testing.assert_array_equal(x[k], y[k], err_msg=k)


def test_ensemble_deterministic():
    p = VARIANTS["solid"]()
    sizes = [2000, 700, 4097]
    packed = pack_states([sim_state(n, seed=500 + k) for k, n in enumerate(sizes)])
    out = []
    for _ in range(2):
        with Ensemble(p, sizes, make_options(accum="compensated")) as e:
            e.upload(packed)
            e.step(2)
            out.append(e.download())
    for k in out[0]:
        np.testing.assert_array_equal(out[0][k], out[1][k], err_msg=k)


def test_ensemble_close_to_single_contexts():
    """Each simulation of the batch vs the same simulation in its own context (both FP32)."""
    p = config0_params()
    sizes = [1024, 2500]
    states = [sim_state(n, seed=600 + k, rho0=0.239) for k, n in enumerate(sizes)]
    with Ensemble(p, sizes) as ens:
        ens.upload(pack_states(states))
        ens.compute_derivatives()
        got = ens.split(ens.download())
    for k, st in enumerate(states):
        with DeviceParticleBuffer(p, sizes[k]) as pb:
            pb.upload(st)
            pb.compute_derivatives()
            single = pb.download()
        for f in ("acc", "density"):
            scale = np.abs(single[f]).max()
            assert np.abs(got[k][f] - single[f]).max() <= 1e-5 * scale, f


@pytest.mark.parametrize("name", ["solid", "fluid", "nbody"])
def test_ensemble_diagnostics_vs_oracle(oracle, name):
    p = VARIANTS[name]()
    sizes = [800, 1600]
    states = [sim_state(n, seed=700 + k, rho0=p.rho0) for k, n in enumerate(sizes)]
    with Ensemble(p, sizes) as ens:
        ens.upload(pack_states(states))
        ens.compute_derivatives()
        d = ens.diagnostics(half_kick=0.5e-3)
    for k, st in enumerate(states):
        ref = copy_state(st)
        oracle.ts.current = oracle.ts.next = 0.0
        oracle.compute_derivatives(p, ref)
        o = oracle.diagnostics(p, ref, half_kick=0.5e-3)
        for f in ("e_grav", "mass"):
            assert abs(d[k][f] - o[f]) <= 1e-9 * max(abs(o[f]), 1e-30), (k, f, d[k][f], o[f])
        for f in ("e_kin", "e_int", "e_shear"):
            assert abs(d[k][f] - o[f]) <= 1e-5 * max(abs(o[f]), abs(o["e_kin"]), 1e-30), (k, f, d[k][f], o[f])


def test_ensemble_rejects_unsupported():
    base = ref_variants.params_dict(ref_variants.VARIANTS["solid_mc"])
    with pytest.raises(GsphError) as e:
        Ensemble(make_params(**base), [100, 200])
    assert e.value.code == -7
    with pytest.raises(GsphError) as e:
        Ensemble(config0_params(), [100, 0])
    assert e.value.code == -1
    with pytest.raises(GsphError) as e:
        Ensemble(config0_params(), [100], make_options(precision="double"))
    assert e.value.code == -7


def test_ensemble_autotune_keeps_results(oracle):
    p = VARIANTS["solid"]()
    sizes = [3000, 700]
    states = [sim_state(n, seed=800 + k) for k, n in enumerate(sizes)]
    with Ensemble(p, sizes) as ens:
        ens.upload(pack_states(states))
        shape = ens.autotune(1)
        assert shape["tile"] in (256, 512, 1024)
        ens.compute_derivatives()
        got = ens.split(ens.download())
        ens.step(2)
    for k, st in enumerate(states):
        ref, sens = fp32_sensitivity(oracle_derivs(oracle, p), st, trials=1)
        for f, tol in fields(p).items():
            check_within(got[k][f], ref[f], sens[f], tol, "autotuned sim %d %s" % (k, f))


def test_dependency_wait_runs_out_and_the_ensemble_recovers(oracle):
    """Failure detection without a GPU fault: the host makes one simulation's SPH items wait for a
    density item that does not exist (gsph_ensemble_inject_stall); with a 1 ms bound the device-side
    waits give up, set the timeout bit and return. compute_derivatives is asynchronous, so the next
    synchronising call (download) reports GSPH_E_TIMEOUT; after a fresh upload the same ensemble
    computes correct derivatives again."""
    import time
    from grasph2_b200._abi import GSPH_E_TIMEOUT
    p = VARIANTS["fluid"]()
    sizes = [700, 1500, 300]
    states = [sim_state(n, seed=400 + k, rho0=p.rho0) for k, n in enumerate(sizes)]
    with Ensemble(p, sizes, make_options(wait_limit_us=1000)) as ens:
        ens.upload(pack_states(states))
        ens.inject_stall(1)
        t0 = time.perf_counter()
        ens.compute_derivatives()
        with pytest.raises(GsphError) as exc:
            ens.download()
        elapsed = time.perf_counter() - t0
        assert exc.value.code == GSPH_E_TIMEOUT
        assert "gave up" in str(exc.value)
        assert elapsed < 5.0, elapsed  # every wait bounded by 1 ms; launch and report overhead only
        ens.upload(pack_states(states))  # the context stays usable
        ens.compute_derivatives()
        got = ens.split(ens.download())
    for k, st in enumerate(states):
        ref, sens = fp32_sensitivity(oracle_derivs(oracle, p), st, trials=1)
        for f, tol in fields(p).items():
            check_within(got[k][f], ref[f], sens[f], tol, "after timeout sim %d %s" % (k, f))
