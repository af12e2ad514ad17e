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

Surrogate.energy_correction() turns on the judge-calibrated energy correction: the network's
proposals lose a little kinetic and shear energy against the plain integrator, the same way each
time, so every proposal is followed by gsph_energy_adjust with running estimates of that bias, which
every judged window updates from its own comparison.
"""

import ctypes
import math
import time

import numpy as np

from ._abi import SurrogateWindow, load_library
from .mlp import MLP
from .sim import GsphError, _stream_handle

NF, NO = 32, 13
NSTATS = 2 * NF + 2 * NO
OUT_NAMES = ["dx", "dy", "dz", "dvx", "dvy", "dvz", "drho", "dSxx", "dSyy", "dSzz", "dSxy", "dSxz", "dSyz"]


def _torch():
    import torch
    return torch


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _fp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


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
    """The native surrogate (gsph_surrogate_*): its MLP, the standardisation of the MLP's inputs and
    outputs, and the substep count K. `net` is a view of the surrogate's own MLP (train it in place)."""

    def __init__(self, K=8, params=None, in_mu=None, in_sig=None, out_mu=None, out_sig=None, _handle=None):
        torch = _torch()
        self.lib = load_library()
        if _handle is None:
            count = int(self.lib.gsph_mlp_param_count())
            arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float32).ravel()
                    for a in (params, in_mu, in_sig, out_mu, out_sig)]
            for a, k in zip(arrs, (count, NF, NF, NO, NO)):
                if a is not None and a.shape != (k,):
                    raise ValueError("surrogate arrays must have %d, %d, %d, %d and %d values" % (count, NF, NF, NO, NO))
            _handle = ctypes.c_void_p()
            rc = self.lib.gsph_surrogate_create(*[_fp(a) for a in arrs], int(K), ctypes.byref(_handle))
            if rc != 0:
                raise GsphError(rc, self.lib.gsph_last_error(None).decode())
        self._h = _handle
        self.K = int(self.lib.gsph_surrogate_substeps(self._h))
        self.net = MLP.borrow(self.lib.gsph_surrogate_mlp(self._h), self)
        st = np.empty(NSTATS, dtype=np.float32)
        self._check(self.lib.gsph_surrogate_stats(self._h, _fp(st)))
        self.stats = {"in_mu": st[:NF], "in_sig": st[NF:2 * NF], "out_mu": st[2 * NF:2 * NF + NO],
                      "out_sig": st[2 * NF + NO:]}
        self.dev = {k: torch.from_numpy(v.copy()).cuda() for k, v in self.stats.items()}

    def _check(self, rc):
        if rc != 0:
            raise GsphError(rc, self.lib.gsph_surrogate_last_error(self._h).decode())

    def close(self):
        if self._h:
            self.lib.gsph_surrogate_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def save(self, path, **meta):
        """`.gsur`: the native model file (gsph_surrogate_save); otherwise an npz with `meta` beside."""
        if str(path).endswith(".gsur"):
            self._check(self.lib.gsph_surrogate_save(self._h, str(path).encode()))
        else:
            np.savez(path, params=self.net.params(), K=self.K, **self.stats, **meta)

    @classmethod
    def load(cls, path):
        if str(path).endswith(".gsur"):
            lib = load_library()
            h = ctypes.c_void_p()
            rc = lib.gsph_surrogate_load(str(path).encode(), ctypes.byref(h))
            if rc != 0:
                raise GsphError(rc, lib.gsph_last_error(None).decode())
            return cls(_handle=h)
        z = np.load(path)
        return cls(int(z["K"]), z["params"], z["in_mu"], z["in_sig"], z["out_mu"], z["out_sig"])

    def propose(self, pb, use_net=True, stream=None):
        """Advance pb by K substeps in one proposal (gsph_surrogate_propose)."""
        self._check(self.lib.gsph_surrogate_propose(self._h, pb.handle, int(bool(use_net)), _stream_handle(stream)))

    def energy_correction(self, on=True, gain=1.0):
        """Judge-calibrated energy correction (gsph_surrogate_set_energy_correction); resets the estimates."""
        self._check(self.lib.gsph_surrogate_set_energy_correction(self._h, int(bool(on)), float(gain)))

    def energy_bias(self):
        """The running estimates of one proposal's kinetic and shear energy bias."""
        b = (ctypes.c_double * 2)()
        self._check(self.lib.gsph_surrogate_energy_bias(self._h, b))
        return b[0], b[1]

    def launch_count(self):
        c = ctypes.c_int64(0)
        self._check(self.lib.gsph_surrogate_launch_count(self._h, ctypes.byref(c)))
        return c.value


def fit(X, Y, K, steps=2000, batch=65536, lr=1e-3, seed=0, log_every=0, wout=None, clip=0.0, grad_clip=0.0,
        stream=None, eval_rows=65536):
    """Train a Surrogate on (X, Y) with the device kernels (forward + backward on the tensor cores, Adam);
    wout weights the 13 standardised outputs in the loss (default 1); clip > 0 limits the standardised
    targets to +-clip (the heavy tails of the impact zone otherwise dominate single batches); grad_clip > 0
    limits the global gradient norm of each Adam step. Returns (surrogate, loss history): every log_every
    steps (step, loss of that step's batch, loss on a fixed evaluation set of eval_rows samples drawn once
    with seed + 1). A batch loss follows its batch (a batch holding a few impact-zone samples can read
    30x the typical loss); the evaluation loss follows the model. The evaluation runs before the step's
    own gradient, which overwrites it, so training is the same with or without it."""
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
    if grad_clip > 0:
        sur.net.set_grad_clip(grad_clip)
    m = X.shape[0]
    hist = []
    if log_every:
        ge = torch.Generator(device="cuda").manual_seed(seed + 1)
        eidx = torch.randint(0, m, (min(eval_rows, m),), device="cuda", generator=ge)
        xe, ye = Xd[eidx].contiguous(), Yd[eidx].contiguous()
    for step in range(steps):
        idx = torch.randint(0, m, (min(batch, m),), device="cuda", generator=g)
        xb, yb = Xd[idx].contiguous(), Yd[idx].contiguous()
        rate = lr * 0.5 * (1.0 + math.cos(math.pi * step / steps))  # cosine decay
        want = log_every and (step % log_every == 0 or step == steps - 1)
        if want:
            le = sur.net.gradient(xe, ye, w, xe.shape[0], stream, want=True)[1]
        r = sur.net.gradient(xb, yb, w, xb.shape[0], stream, want=bool(want))
        if want:
            hist.append((step, r[1], le))
        sur.net.adam(lr=rate, stream=stream)
    return sur, hist


def compare(pb, slot_p, slot_0, stream=None, parts=False):
    """gsph_state_compare: (E(P) - E(Q), sum |x_P - x_Q|^2, sum |x_Q - x_0|^2, local energy of Q); with
    parts, gsph_state_compare_parts: the same followed by the kinetic, internal, shear and first-order
    gravitational parts of E(P) - E(Q)."""
    out = (ctypes.c_double * (8 if parts else 4))()
    f = pb.lib.gsph_state_compare_parts if parts else pb.lib.gsph_state_compare
    pb._check(f(pb.handle, int(slot_p), int(slot_0), out, _stream_handle(stream)))
    return tuple(out)


def energy_adjust(pb, d_kin, d_shear, stream=None):
    """gsph_energy_adjust: change the kinetic energy about the centre of mass and the shear energy."""
    pb._check(pb.lib.gsph_energy_adjust(pb.handle, float(d_kin), float(d_shear), _stream_handle(stream)))


def window_errors(pb, sur, use_net=True, e_ref=None, stream=None):
    """One proposal and the plain K steps from the same state (gsph_surrogate_judge); returns (position
    error, relative energy error). The position error is norm-wise over all particles, relative to the
    plain displacement: ||x_proposal - x_plain||_2 / ||x_plain - x_start||_2; the energy error is
    |E_proposal - E_plain| / |E| (gsph_state_compare, O(N) on the device; E from the fast diagnostics
    unless e_ref is given). The context ends on the plain result."""
    w = SurrogateWindow()
    sur._check(sur.lib.gsph_surrogate_judge(sur._h, pb.handle, int(bool(use_net)), float(e_ref or 0.0),
                                            ctypes.byref(w), _stream_handle(stream)))
    return w.pos_error, w.energy_error


def _energy(d):
    return d["e_kin"] + d["e_grav"] + d["e_int"] + d["e_shear"]


def advance(pb, sur, nwin, M=4, pos_tol=1e-3, e_tol=1e-4, use_net=True, stream=None):
    """nwin windows of M proposals (K substeps each), the last one judged against the plain integrator
    (gsph_surrogate_advance). Returns a dict: substeps advanced, wall seconds, accepted windows,
    per-window errors."""
    torch = _torch()
    wins = (SurrogateWindow * max(1, nwin))()
    acc = ctypes.c_int32(0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sur._check(sur.lib.gsph_surrogate_advance(sur._h, pb.handle, int(nwin), int(M), float(pos_tol), float(e_tol),
                                              int(bool(use_net)), wins, ctypes.byref(acc), _stream_handle(stream)))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    errs = [(wins[k].pos_error, wins[k].energy_error) for k in range(nwin)]
    parts = [tuple(wins[k].energy_parts) for k in range(nwin)]
    return {"substeps": nwin * M * sur.K, "wall_s": wall, "accepted": acc.value, "windows": nwin, "errors": errs,
            "energy_parts": parts, "accepted_mask": [bool(wins[k].accepted) for k in range(nwin)]}
