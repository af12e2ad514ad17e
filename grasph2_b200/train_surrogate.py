"""Train the learned surrogate of the impact workload on trajectories of the plain solver.

    python -m grasph2_b200.train_surrogate [--n 262144] [--trajectories 200] [--windows 32] [--every 4]
                                           [--rows 8192] [--steps 6000] [--out grasph2_b200/data/...npz]

Each trajectory is a two-sphere impact (radii 1 and 0.5, equal number density, N split 8:1) with a
seeded relative velocity in [0.2, 1.0] and y-offset in [0, 0.8], advanced by the plain solver for
windows x K substeps (K = 8); every `every`-th window contributes the features at its start and the
K-step targets of `rows` random particles. The MLP is then fitted on the device by the project's own
tensor-core forward/backward kernels and Adam. Writes the model (parameters, standardisation, K) as an
npz and as the native model file (.gsur, gsph_surrogate_load), and a summary of the run (collection and
training times, loss history) next to them.
"""

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "data", "surrogate_impact_n262144.npz")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--trajectories", type=int, default=200)
    ap.add_argument("--windows", type=int, default=32)
    ap.add_argument("--every", type=int, default=4)
    ap.add_argument("--rows", type=int, default=8192)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--clip", type=float, default=0.0, help="limit the standardised targets to +-clip (0: off)")
    ap.add_argument("--grad-clip", type=float, default=1.0, help="global gradient-norm clipping of Adam (0: off)")
    ap.add_argument("--K", type=int, default=8)
    ap.add_argument("--seed", type=int, default=20261207)
    ap.add_argument("--out", default=DEFAULT_OUT)
    a = ap.parse_args(argv)
    import torch
    sys.path.insert(0, os.path.dirname(HERE))
    from grasph2_b200 import ics
    from grasph2_b200 import surrogate as S
    from grasph2_b200.params import impact_params
    from grasph2_b200.sim import DeviceParticleBuffer

    nb = round(a.n * 8 / 9)
    ns = a.n - nb
    p = impact_params(nb, ns)
    rng = np.random.default_rng(a.seed)
    X, Y = [], []
    t0 = time.time()
    for tr in range(a.trajectories):
        v = rng.uniform(0.2, 1.0)
        off = rng.uniform(0.0, 0.8)
        st = ics.two_sphere_impact(nb, ns, v_rel=v, y_offset=off, seed=a.seed + 1 + tr)
        with DeviceParticleBuffer(p, a.n) as pb:
            pb.upload(st)
            x, y = S.collect(pb, a.windows, a.K, a.rows, rng, every=a.every)
        X.append(x)
        Y.append(y)
    X, Y = np.concatenate(X), np.concatenate(Y)
    t_collect = time.time() - t0
    t0 = time.time()
    sur, hist = S.fit(X, Y, a.K, steps=a.steps, batch=a.batch, lr=a.lr, seed=a.seed, log_every=max(1, a.steps // 20),
                      clip=a.clip, grad_clip=a.grad_clip)
    torch.cuda.synchronize()
    t_fit = time.time() - t0
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    meta = dict(n=a.n, trajectories=a.trajectories, windows=a.windows, every=a.every, rows=a.rows, steps=a.steps,
                batch=a.batch, lr=a.lr, clip=a.clip, grad_clip=a.grad_clip, seed=a.seed, samples=int(X.shape[0]), collect_s=t_collect, fit_s=t_fit,
                loss=[(int(s), float(l)) for s, l, _ in hist], eval_loss=[(int(s), float(e)) for s, _, e in hist])
    sur.save(a.out, meta=json.dumps(meta))
    sur.save(os.path.splitext(a.out)[0] + ".gsur")  # the native model file (gsph_surrogate_load)
    with open(os.path.splitext(a.out)[0] + ".json", "w") as f:
        json.dump(meta, f, indent=1)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
