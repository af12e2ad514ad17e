"""The learned surrogate's device pieces: features, the proposal update, snapshots, the fast energy, and
the end-to-end gain of the trained network over the extrapolation without it."""

import numpy as np
import pytest

from grasph2_b200 import ics
from grasph2_b200 import surrogate as S
from grasph2_b200.params import impact_smoothing_length, make_params
from grasph2_b200.sim import DeviceParticleBuffer
from helpers import f32_exact

pytestmark = pytest.mark.gpu


def impact_params(nb, ns):
    return make_params(switches=("SELF_GRAVITY", "SPH", "SOLIDS", "ARTIFICIAL_VISCOSITY", "PLASTICITY_MIESE"),
                       H=impact_smoothing_length(nb, 1.0, ns, 0.5), grav_eps=0.01, rho0=1.0, bulk=10.0, dbulk_dp=1.0,
                       soundspeed=10 ** 0.5, shear=5.0, Y=0.5, av_alpha=1.0, av_beta=2.0, fixed_dt=1e-4)


def solid_state(n, seed):
    rng = np.random.default_rng(seed)
    st = ics.uniform_sphere(n, radius=1.0, rho0=1.0, omega=(0, 0, 0.3), seed=seed)
    st["vel"] += 0.05 * rng.normal(size=(n, 3))
    st["density"][:] = 1.0 + 0.02 * rng.normal(size=n)
    M = rng.normal(size=(n, 3, 3)) * 0.05
    st["dstress"][:] = 0.5 * (M + M.transpose(0, 2, 1))
    return f32_exact(st)


def features_numpy(st, p):
    """The 32 features restated on the host in FP64 (brute force over all pairs)."""
    x, v, m = st["pos"], st["vel"], st["mass"]
    h, rho0 = p.H, p.rho0
    d = x[None, :, :] - x[:, None, :]  # d[i, j] = x_j - x_i
    r = np.sqrt((d * d).sum(-1))
    q = r / h
    w = np.where(q < 0.5, 6 * q ** 3 - 6 * q ** 2 + 1, 2 * (1 - q) ** 3)
    w = np.where((r > 0) & (q <= 1), w, 0.0) * (8.0 / (np.pi * h ** 3)) * m[None, :]
    e = d / h
    u = v[None, :, :] - v[:, None, :]
    S = st["dstress"].reshape(-1, 9)
    f = np.zeros((len(m), 32))
    f[:, 0:3] = v
    f[:, 3] = st["density"] / rho0 - 1
    f[:, 4:10] = S[:, [0, 4, 8, 1, 2, 5]]
    f[:, 10] = w.sum(1) / rho0
    f[:, 11:14] = (w[:, :, None] * e).sum(1) / rho0
    f[:, 14:17] = (w[:, :, None] * u).sum(1) / rho0
    ee = np.stack([e[..., 0] ** 2, e[..., 1] ** 2, e[..., 2] ** 2, e[..., 0] * e[..., 1], e[..., 0] * e[..., 2],
                   e[..., 1] * e[..., 2]], -1)
    f[:, 17:23] = (w[:, :, None] * ee).sum(1) / rho0
    f[:, 23:32] = (w[:, :, None] * (u[..., :, None] * e[..., None, :]).reshape(len(m), len(m), 9)).sum(1) / rho0
    return f


def test_features_vs_host():
    import torch
    p = impact_params(1800, 200)
    p.H = 0.35
    st = solid_state(2000, 1)
    with DeviceParticleBuffer(p, 2000) as pb:
        pb.upload(st)
        f = S.features(pb).cpu().numpy()
        mu = torch.arange(32, dtype=torch.float32, device="cuda") * 0.1
        sig = torch.full((32,), 2.0, device="cuda")
        fn = S.features(pb, mu, sig).cpu().numpy()
    want = features_numpy(st, p)
    for k in range(32):
        scale = max(np.abs(want[:, k]).max(), 1e-12)
        assert np.abs(f[:, k] - want[:, k]).max() <= 2e-5 * scale, k
    np.testing.assert_allclose(fn, (f - 0.1 * np.arange(32)) / 2.0, rtol=1e-6, atol=1e-6)


def test_apply_is_the_constant_derivative_leapfrog():
    import torch
    p = impact_params(1800, 200)
    st = solid_state(2000, 2)
    K = 8
    with DeviceParticleBuffer(p, 2000) as pb:
        pb.upload(st)
        pb.compute_derivatives()
        s0 = S._state(pb)
        S.snapshot(pb, 2, False)
        S.apply(pb, K)
        x = pb.download_pos64()
        got = pb.download(["vel", "dstress"])
        rng = np.random.default_rng(3)
        delta = torch.from_numpy(rng.normal(size=(2000, 13)).astype(np.float32)).cuda()
        omu = torch.from_numpy(rng.normal(size=13).astype(np.float32) * 1e-4).cuda()
        osig = torch.from_numpy(rng.uniform(1e-5, 1e-4, size=13).astype(np.float32)).cuda()
        S.snapshot(pb, 2, True)
        np.testing.assert_array_equal(pb.download_pos64(), s0["pos64"])
        S.apply(pb, K, delta, omu, osig)
        x2 = pb.download_pos64()
    kin = S.kinematic(s0, K, p.fixed_dt)
    np.testing.assert_allclose(x, kin["pos"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(got["vel"], kin["vel"], rtol=1e-6, atol=1e-7)
    d = omu.cpu().numpy()[None, :] + osig.cpu().numpy()[None, :] * delta.cpu().numpy()
    np.testing.assert_allclose(x2 - x, d[:, 0:3], rtol=1e-5, atol=1e-12)


def test_snapshot_restores_every_array():
    p = impact_params(1800, 200)
    st = solid_state(2000, 4)
    with DeviceParticleBuffer(p, 2000) as pb:
        pb.upload(st)
        pb.step(2)
        S.snapshot(pb, 0, False)
        a = pb.download()
        pb.step(3)
        S.snapshot(pb, 0, True)
        b = pb.download()
        pb.step(3)
        c = pb.download()
        S.snapshot(pb, 0, True)
        pb.step(3)
        d = pb.download()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
        np.testing.assert_array_equal(c[k], d[k], err_msg=k)


def test_fast_diagnostics_match_fp64():
    p = impact_params(1800, 200)
    st = solid_state(3000, 5)
    with DeviceParticleBuffer(p, 3000) as pb:
        pb.upload(st)
        pb.compute_derivatives()
        a = pb.diagnostics(5e-5)
        b = pb.diagnostics(5e-5, fast=True)
    assert abs(a["e_grav"] - b["e_grav"]) <= 1e-6 * abs(a["e_grav"])
    for k in ("e_kin", "e_int", "e_shear", "mass"):
        assert a[k] == b[k], k


def _trained(nb, seed=0):
    ns = nb // 8
    p = impact_params(nb, ns)
    rng = np.random.default_rng(seed)
    X, Y = [], []
    for tr in range(6):
        st = ics.two_sphere_impact(nb, ns, v_rel=rng.uniform(0.2, 1.0), y_offset=rng.uniform(0, 0.8), seed=100 + tr)
        with DeviceParticleBuffer(p, nb + ns) as pb:
            pb.upload(st)
            x, y = S.collect(pb, 12, 8, 4096, rng, every=2)
            X.append(x)
            Y.append(y)
    sur, _ = S.fit(np.concatenate(X), np.concatenate(Y), 8, steps=1500, batch=32768, lr=2e-3)
    return p, sur


def test_network_gains_over_the_extrapolation():
    """On a held-out impact, the trained network's proposals are closer to the plain solver than the
    constant-derivative extrapolation alone: energy error at least 5x lower, position error lower."""
    nb, ns = 7282, 910
    p, sur = _trained(nb)
    st = ics.two_sphere_impact(nb, ns, v_rel=0.6, y_offset=0.4, seed=999)
    res = {}
    for use in (False, True):
        with DeviceParticleBuffer(p, nb + ns) as pb:
            pb.upload(st)
            errs = []
            for w in range(12):
                if w % 3 == 0:
                    errs.append(S.window_errors(pb, sur, use))
                else:
                    pb.step(8)
        res[use] = np.array(errs)
    assert res[True][:, 1].mean() < 0.2 * res[False][:, 1].mean(), res
    assert res[True][:, 0].mean() < res[False][:, 0].mean(), res


def test_advance_rejects_back_to_the_plain_path():
    """With a zero tolerance every window is rejected and the result is exactly the plain integrator's."""
    nb, ns = 1800, 225
    p = impact_params(nb, ns)
    st = ics.two_sphere_impact(nb, ns, v_rel=0.5, y_offset=0.3, seed=7)
    sur = S.Surrogate(8)
    with DeviceParticleBuffer(p, nb + ns) as a, DeviceParticleBuffer(p, nb + ns) as b:
        a.upload(st)
        b.upload(st)
        r = S.advance(a, sur, 3, M=2, pos_tol=0.0, e_tol=0.0)
        b.step(3 * 2 * 8)
        x, y = a.download(), b.download()
    assert r["accepted"] == 0 and r["substeps"] == 48
    for k in x:
        np.testing.assert_array_equal(x[k], y[k], err_msg=k)


def test_state_compare_matches_full_energies():
    """The judge's O(N) comparison against full diagnostics of both states and host position norms."""
    nb, ns = 7282, 910
    p = impact_params(nb, ns)
    st = ics.two_sphere_impact(nb, ns, v_rel=0.6, y_offset=0.4, seed=31)
    sur = S.Surrogate(8)
    with DeviceParticleBuffer(p, nb + ns) as pb:
        pb.upload(st)
        pb.step(5)
        S.snapshot(pb, 1, False)
        x0 = pb.download_pos64()
        sur.propose(pb, use_net=False)
        S.snapshot(pb, 2, False)
        xp = pb.download_pos64()
        ep = S._energy(pb.diagnostics(0.0))
        S.snapshot(pb, 1, True)
        pb.step(8)
        xq = pb.download_pos64()
        eq = S._energy(pb.diagnostics(0.0))
        de, dx2, d02, _ = S.compare(pb, 2, 1)
    np.testing.assert_allclose(dx2, ((xp - xq) ** 2).sum(), rtol=1e-9)
    np.testing.assert_allclose(d02, ((xq - x0) ** 2).sum(), rtol=1e-9)
    # first-order gravitational energy change: agrees to a small fraction of the difference itself
    assert abs(de - (ep - eq)) <= 0.05 * abs(ep - eq) + 1e-9 * abs(eq), (de, ep - eq)


def test_surrogate_entry_points_reject_unsupported_contexts():
    from grasph2_b200.params import make_options
    from grasph2_b200.sim import GsphError
    p = impact_params(900, 100)
    st = solid_state(1000, 9)
    with DeviceParticleBuffer(p, 1000, make_options(cull=False)) as pb:
        pb.upload(st)
        with pytest.raises(GsphError) as e:
            S.features(pb)
        assert e.value.code == -7
    with DeviceParticleBuffer(p, 1000, make_options(precision="double")) as pb:
        with pytest.raises(GsphError) as e:
            S.apply(pb, 8)
        assert e.value.code == -7
        with pytest.raises(GsphError):
            S.snapshot(pb, 0, False)
    with DeviceParticleBuffer(p, 1000) as pb:
        pb.upload(st)
        with pytest.raises(GsphError) as e:
            S.snapshot(pb, 0, True)  # nothing saved yet
        assert e.value.code == -4
        with pytest.raises(GsphError):
            S.snapshot(pb, 9, False)  # no such slot


def _quiet_surrogate(K=8, seed=3):
    """A random network whose outputs are scaled to ~1e-7: proposals stay close to the extrapolation."""
    from grasph2_b200.mlp import init_params
    rng = np.random.default_rng(seed)
    return S.Surrogate(K, init_params(seed), rng.normal(size=32) * 0.1, rng.uniform(0.5, 2.0, 32),
                       np.zeros(13), np.full(13, 1e-7))


def test_native_window_loop_matches_the_primitives():
    """gsph_surrogate_advance with every window accepted equals the same window rule written out with
    the public primitives (snapshots, proposals, plain steps, state comparison), bit for bit."""
    nb, ns = 1800, 225
    p = impact_params(nb, ns)
    st = ics.two_sphere_impact(nb, ns, v_rel=0.5, y_offset=0.3, seed=11)
    sur = _quiet_surrogate()
    M, K, nwin = 3, sur.K, 2
    with DeviceParticleBuffer(p, nb + ns) as a, DeviceParticleBuffer(p, nb + ns) as b:
        a.upload(st)
        b.upload(st)
        r = S.advance(a, sur, nwin, M=M, pos_tol=1e30, e_tol=1e30)
        e_ref = S._energy(b.diagnostics(0.0, fast=True))
        want = []
        for _ in range(nwin):
            S.snapshot(b, 0, False)
            for _ in range(M - 1):
                sur.propose(b)
            S.snapshot(b, 1, False)
            sur.propose(b)
            S.snapshot(b, 2, False)
            S.snapshot(b, 1, True)
            b.step(K)
            de, dx2, d02, _ = S.compare(b, 2, 1)
            want.append((np.sqrt(dx2 / d02), abs(de) / abs(e_ref)))
        x, y = a.download(), b.download()
        assert np.array_equal(a.download_pos64(), b.download_pos64())
    assert r["accepted"] == nwin and r["substeps"] == nwin * M * K
    for k in x:
        np.testing.assert_array_equal(x[k], y[k], err_msg=k)
    np.testing.assert_allclose(np.array(r["errors"]), np.array(want), rtol=1e-12)


def test_surrogate_model_file_round_trip(tmp_path):
    sur = _quiet_surrogate(K=6, seed=5)
    f = str(tmp_path / "m.gsur")
    sur.save(f)
    back = S.Surrogate.load(f)
    assert back.K == 6
    np.testing.assert_array_equal(back.net.params(), sur.net.params())
    for k in sur.stats:
        np.testing.assert_array_equal(back.stats[k], sur.stats[k], err_msg=k)
    g = str(tmp_path / "m.npz")
    sur.save(g)
    again = S.Surrogate.load(g)
    np.testing.assert_array_equal(again.net.params(), sur.net.params())


def test_committed_model_files_agree():
    """The trained model ships as an npz (with its training summary) and as the native model file."""
    import os
    base = os.path.join(os.path.dirname(S.__file__), "data", "surrogate_impact_n262144")
    a, b = S.Surrogate.load(base + ".npz"), S.Surrogate.load(base + ".gsur")
    assert a.K == b.K == 8
    np.testing.assert_array_equal(a.net.params(), b.net.params())
    for k in a.stats:
        np.testing.assert_array_equal(a.stats[k], b.stats[k], err_msg=k)


def test_energy_adjust_changes_the_requested_energies():
    """gsph_energy_adjust: kinetic energy about the centre of mass and shear energy change by the requested
    amounts; momentum and positions do not change."""
    nb, ns = 7282, 910
    p = impact_params(nb, ns)
    st = solid_state(nb + ns, 21)
    st["vel"] += np.array([0.3, -0.1, 0.05])  # a bulk velocity, kept by the adjustment
    with DeviceParticleBuffer(p, nb + ns) as pb:
        pb.upload(st)
        d0 = pb.diagnostics(0.0)
        x0 = pb.download_pos64()
        P0, M = np.array(d0["momentum"]), d0["mass"]
        ekc = d0["e_kin"] - P0 @ P0 / (2 * M)
        dk, ds = -0.01 * ekc, -0.02 * d0["e_shear"]  # decreases: the limiter cannot clip
        S.energy_adjust(pb, dk, ds)
        d1 = pb.diagnostics(0.0)
        x1 = pb.download_pos64()
    np.testing.assert_array_equal(x0, x1)
    P1 = np.array(d1["momentum"])
    assert np.abs(P1 - P0).max() <= 1e-6 * np.abs(P0).max()
    assert abs((d1["e_kin"] - d0["e_kin"]) - dk) <= 1e-4 * abs(dk), (d1["e_kin"] - d0["e_kin"], dk)
    assert abs((d1["e_shear"] - d0["e_shear"]) - ds) <= 1e-4 * abs(ds), (d1["e_shear"] - d0["e_shear"], ds)
    assert d1["e_int"] == d0["e_int"]


def test_energy_correction_matches_the_primitives():
    """With the energy correction on, gsph_surrogate_advance equals the rule written out with the
    primitives: window 1 uncorrected, its judge's kinetic and shear parts update the estimates by
    gain x part, and every proposal of window 2 is followed by gsph_energy_adjust(-estimates)."""
    nb, ns = 1800, 225
    p = impact_params(nb, ns)
    st = ics.two_sphere_impact(nb, ns, v_rel=0.5, y_offset=0.3, seed=13)
    sur = _quiet_surrogate()
    M, K, gain = 3, sur.K, 0.5
    with DeviceParticleBuffer(p, nb + ns) as a, DeviceParticleBuffer(p, nb + ns) as b:
        a.upload(st)
        b.upload(st)
        sur.energy_correction(True, gain)
        r = S.advance(a, sur, 2, M=M, pos_tol=1e30, e_tol=1e30)
        got_bias = sur.energy_bias()
        sur.energy_correction(False)
        e_ref = S._energy(b.diagnostics(0.0, fast=True))
        bias = [0.0, 0.0]

        def propose():
            sur.propose(b)
            if bias != [0.0, 0.0]:
                S.energy_adjust(b, -bias[0], -bias[1])

        for _ in range(2):
            S.snapshot(b, 0, False)
            for _ in range(M - 1):
                propose()
            S.snapshot(b, 1, False)
            propose()
            S.snapshot(b, 2, False)
            S.snapshot(b, 1, True)
            b.step(K)
            c = S.compare(b, 2, 1, parts=True)
            bias[0] += gain * (c[4] / abs(e_ref)) * abs(e_ref)
            bias[1] += gain * (c[6] / abs(e_ref)) * abs(e_ref)
        x, y = a.download(), b.download()
    assert r["accepted"] == 2
    assert bias[0] != 0.0 and bias[1] != 0.0
    assert got_bias == tuple(bias)
    for k in x:
        np.testing.assert_array_equal(x[k], y[k], err_msg=k)
