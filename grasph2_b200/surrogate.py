"""The learned K-substep surrogate of the impact workload.

A proposal advances a context by K substeps at once: one computeDerivatives at the current state, the
32 neighbour-moment features of every particle (gsph_surrogate_features), the per-particle MLP on the
tensor cores (gsph_mlp_forward), and gsph_surrogate_apply, which adds the MLP's correction to the
fixed-step leapfrog extrapolated with the current derivatives held constant:

    x_K = x + K dt v + K(K+1)/2 dt^2 a + dx,   v_K = v + K dt a + dv,   rho_K = rho + drho,
    S_K = S + K dt dS/dt + dS                  (then the plasticity limiter)

(v is the stored half-step velocity). The MLP predicts (dx, dv, drho, dS) in units of their spread
over the training set. Training targets are the plain solver's own K-step results minus that
extrapolation, so "the method without the network" is the extrapolation alone (delta = 0).

advance() runs windows of M proposals; the plain integrator re-advances the last proposal of each
window from the same state as judge. The window is accepted when the proposal is within pos_tol of
the plain result in position (relative to the plain displacement over the K substeps) and within
e_tol in total energy; the state then continues from the plain result. Otherwise every proposal of
the window is discarded and the window is re-run with the plain integrator from its start.
"""

import ctypes
import math
import time

import numpy as np

from .mlp import MLP
from .sim import _stream_handle

NF, NO = 32, 13
OUT_NAMES = ["dx", "dy", "dz", "dvx", "dvy", "dvz", "drho", "dSxx", "dSyy", "dSzz", "dSxy", "dSxz", "dSyz"]


def _torch():
    import torch
    return torch


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def features(pb, mu=None, sig=None, out=None, stream=None):
    """Features of the current state (device tensor [n][32], caller's order)."""
    torch = _torch()
    if out is None:
        out = torch.empty(pb.n, NF, dtype=torch.float32, device="cuda")
    pb._check(pb.lib.gsph_surrogate_features(pb.handle, _p(mu), _p(sig), _p(out), _stream_handle(stream)))
    return out


def apply(pb, K, delta=None, omu=None, osig=None, stream=None):
    pb._check(pb.lib.gsph_surrogate_apply(pb.handle, _p(delta), _p(omu), _p(osig), int(K), _stream_handle(stream)))


def snapshot(pb, slot, restore, stream=None):
    pb._check(pb.lib.gsph_snapshot(pb.handle, int(slot), int(bool(restore)), _stream_handle(stream)))


def _sym6(m9):
    """9 row-major tensor components -> xx yy zz xy xz yz."""
    m9 = np.asarray(m9).reshape(len(m9), 9)
    return m9[:, [0, 4, 8, 1, 2, 5]]


def kinematic(s0, K, dt):
    """The constant-derivative K-substep extrapolation (host, float64), same formula as the apply kernel
    (whose time step is the float32 one of the integrator)."""
    dt = float(np.float32(dt))
    T, c2 = K * dt, 0.5 * K * (K + 1) * dt * dt
    return {"pos": s0["pos64"] + T * s0["vel"] + c2 * s0["acc"], "vel": s0["vel"] + T * s0["acc"],
            "density": s0["density"] + T * s0["density_dt"],
            "S": _sym6(s0["dstress"]) + T * _sym6(s0["dstress_dt"])}


def _state(pb):
    st = pb.download(["vel", "acc", "density", "density_dt", "dstress", "dstress_dt"])
    out = {k: np.asarray(v, dtype=np.float64) for k, v in st.items()}
    out["pos64"] = pb.download_pos64()
    return out


def targets(s0, sK, K, dt):
    """Plain K-step result minus the extrapolation, [n][13]."""
    kin = kinematic(s0, K, dt)
    return np.concatenate([sK["pos64"] - kin["pos"], sK["vel"] - kin["vel"], (sK["density"] - kin["density"])[:, None],
                           _sym6(sK["dstress"]) - kin["S"]], axis=1)


def collect(pb, nwin, K, rows, rng, every=1, stream=None):
    """Run nwin windows of K plain steps from the context's state; every `every`-th window gives the
    features at its start and the targets of `rows` random particles. Returns (X [m][32], Y [m][13])
    as float32 host arrays."""
    torch = _torch()
    dt = pb.params.fixed_dt
    Xs, Ys = [], []
    for w in range(nwin):
        if w % every:
            pb.step(K, stream)
            continue
        pb.compute_derivatives(stream)
        f = features(pb, stream=stream)
        s0 = _state(pb)
        pb.integrate(True, stream)
        if K > 1:
            pb.step(K - 1, stream)
        sK = _state(pb)
        idx = rng.choice(pb.n, size=min(rows, pb.n), replace=False)
        Xs.append(f[torch.from_numpy(idx).cuda()].cpu().numpy())
        Ys.append(targets(s0, sK, K, dt)[idx].astype(np.float32))
    return np.concatenate(Xs), np.concatenate(Ys)


class Surrogate:
    """MLP + standardisation of its inputs and outputs + the substep count K."""

    def __init__(self, K=8, params=None, in_mu=None, in_sig=None, out_mu=None, out_sig=None):
        torch = _torch()
        self.K = int(K)
        self.net = MLP(params)
        z = lambda k: np.zeros(k, np.float32)  # noqa: E731
        o = lambda k: np.ones(k, np.float32)  # noqa: E731
        self.stats = {"in_mu": in_mu if in_mu is not None else z(NF), "in_sig": in_sig if in_sig is not None else o(NF),
                      "out_mu": out_mu if out_mu is not None else z(NO),
                      "out_sig": out_sig if out_sig is not None else o(NO)}
        self.dev = {k: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32)).cuda() for k, v in self.stats.items()}
        self._feat = self._out = None

    def save(self, path, **meta):
        np.savez(path, params=self.net.params(), K=self.K, **self.stats, **meta)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(int(z["K"]), z["params"], z["in_mu"], z["in_sig"], z["out_mu"], z["out_sig"])

    def propose(self, pb, use_net=True, stream=None):
        """Advance pb by K substeps in one proposal."""
        torch = _torch()
        if self._feat is None or self._feat.shape[0] != pb.n:
            self._feat = torch.empty(pb.n, NF, dtype=torch.float32, device="cuda")
            self._out = torch.empty(pb.n, NO, dtype=torch.float32, device="cuda")
        pb.compute_derivatives(stream)
        if use_net:
            features(pb, self.dev["in_mu"], self.dev["in_sig"], self._feat, stream)
            self.net.forward(self._feat, self._out, pb.n, stream)
            apply(pb, self.K, self._out, self.dev["out_mu"], self.dev["out_sig"], stream)
        else:
            apply(pb, self.K, None, None, None, stream)


def fit(X, Y, K, steps=2000, batch=65536, lr=1e-3, seed=0, log_every=0, wout=None, clip=0.0, stream=None):
    """Train a Surrogate on (X, Y) with the device kernels (forward + backward on the tensor cores, Adam);
    wout weights the 13 standardised outputs in the loss (default 1); clip > 0 limits the standardised
    targets to +-clip (the heavy tails of the impact zone otherwise dominate single batches). Returns
    (surrogate, loss history)."""
    torch = _torch()
    from .mlp import init_params
    in_mu, in_sig = X.mean(0), X.std(0) + 1e-6
    out_mu, out_sig = Y.mean(0), Y.std(0) + 1e-30
    out_sig = np.maximum(out_sig, 1e-6 * out_sig.max())
    sur = Surrogate(K, init_params(seed), in_mu.astype(np.float32), in_sig.astype(np.float32),
                    out_mu.astype(np.float32), out_sig.astype(np.float32))
    Xd = ((torch.from_numpy(X).cuda() - sur.dev["in_mu"]) / sur.dev["in_sig"]).contiguous()
    Yd = ((torch.from_numpy(Y).cuda() - sur.dev["out_mu"]) / sur.dev["out_sig"]).contiguous()
    if clip > 0:
        Yd.clamp_(-clip, clip)
    w = torch.from_numpy(np.asarray(wout if wout is not None else np.ones(NO), dtype=np.float32)).cuda()
    g = torch.Generator(device="cuda").manual_seed(seed)
    m = X.shape[0]
    hist = []
    for step in range(steps):
        idx = torch.randint(0, m, (min(batch, m),), device="cuda", generator=g)
        xb, yb = Xd[idx].contiguous(), Yd[idx].contiguous()
        rate = lr * 0.5 * (1.0 + math.cos(math.pi * step / steps))  # cosine decay
        want = log_every and (step % log_every == 0 or step == steps - 1)
        r = sur.net.gradient(xb, yb, w, xb.shape[0], stream, want=bool(want))
        if want:
            hist.append((step, r[1]))
        sur.net.adam(lr=rate, stream=stream)
    return sur, hist


def compare(pb, slot_p, slot_0, stream=None):
    """gsph_state_compare: (E(P) - E(Q), sum |x_P - x_Q|^2, sum |x_Q - x_0|^2, local energy of Q)."""
    out = (ctypes.c_double * 4)()
    pb._check(pb.lib.gsph_state_compare(pb.handle, int(slot_p), int(slot_0), out, _stream_handle(stream)))
    return tuple(out)


def window_errors(pb, sur, use_net=True, e_ref=None, stream=None):
    """One proposal and the plain K steps from the same state; returns (position error, relative energy
    error). The position error is norm-wise over all particles, relative to the plain displacement:
    ||x_proposal - x_plain||_2 / ||x_plain - x_start||_2; the energy error is |E_proposal - E_plain| / |E|
    (gsph_state_compare, O(N) on the device; E from the fast diagnostics unless e_ref is given). The
    context ends on the plain result."""
    if e_ref is None:
        e_ref = _energy(pb.diagnostics(0.0, stream, fast=True))
    snapshot(pb, 1, False, stream)
    sur.propose(pb, use_net, stream)
    snapshot(pb, 2, False, stream)
    snapshot(pb, 1, True, stream)
    pb.step(sur.K, stream)
    de, dx2, d02, _ = compare(pb, 2, 1, stream)
    return float(math.sqrt(dx2 / d02)) if d02 > 0 else float("inf"), float(abs(de) / abs(e_ref))


def _energy(d):
    return d["e_kin"] + d["e_grav"] + d["e_int"] + d["e_shear"]


def advance(pb, sur, nwin, M=4, pos_tol=1e-3, e_tol=1e-4, use_net=True, stream=None):
    """nwin windows of M proposals (K substeps each), the last one judged against the plain integrator.
    Returns a dict: substeps advanced, wall seconds, accepted windows, per-window errors."""
    torch = _torch()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e_ref = _energy(pb.diagnostics(0.0, stream, fast=True))  # the scale of the energy criterion
    acc, errs = 0, []
    for _ in range(nwin):
        snapshot(pb, 0, False, stream)
        for _ in range(M - 1):
            sur.propose(pb, use_net, stream)
        ex, ee = window_errors(pb, sur, use_net, e_ref, stream)
        errs.append((ex, ee))
        if ex <= pos_tol and ee <= e_tol:
            acc += 1
        else:  # discard the window's proposals: plain integrator from the window's start
            snapshot(pb, 0, True, stream)
            pb.step(M * sur.K, stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    return {"substeps": nwin * M * sur.K, "wall_s": wall, "accepted": acc, "windows": nwin, "errors": errs}
