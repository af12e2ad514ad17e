"""Host restatement of the device initial-condition generators (test infrastructure only): the same
counter-based draws (splitmix64) and formulas in numpy, for bit-level comparison of the draws and
float-rounding-level comparison of the particles."""

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x):
    with np.errstate(over="ignore"):
        x = (x + np.uint64(0x9E3779B97F4A7C15)) & M64
        x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & M64
        x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & M64
        return x ^ (x >> np.uint64(31))


def uniform(seed, k, i):
    with np.errstate(over="ignore"):
        base = splitmix64(np.uint64(seed) + np.uint64(k))
        x = splitmix64(base + np.asarray(i, dtype=np.uint64))
    return (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def direction(seed, k, i):
    ct = 2.0 * uniform(seed, k, i) - 1.0
    ph = 2.0 * np.pi * uniform(seed, k + 1, i)
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    return np.stack([st * np.cos(ph), st * np.sin(ph), ct], axis=1)


def uniform_sphere(n, radius, total_mass, rho0, omega, seed):
    i = np.arange(n, dtype=np.uint64)
    d = direction(seed, 1, i)
    r = radius * np.cbrt(uniform(seed, 0, i))
    x = r[:, None] * d
    w = np.asarray(omega, dtype=np.float64)
    return {"pos": x, "vel": np.cross(w[None, :], x), "mass": np.full(n, total_mass / n), "density": np.full(n, rho0)}


def plummer(n, a, M, G, seed):
    i = np.arange(n, dtype=np.uint64)
    u = np.clip(uniform(seed, 0, i), 1e-300, 1.0 - 1e-16)
    r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    x = r[:, None] * direction(seed, 1, i)
    q = np.zeros(n)
    done = np.zeros(n, dtype=bool)
    for t in range(1000):
        xx = uniform(seed, 3 + 2 * t, i)
        yy = 0.1 * uniform(seed, 4 + 2 * t, i)
        take = ~done
        q[take] = xx[take]
        done |= yy <= xx * xx * (1.0 - xx * xx) ** 3.5
        if done.all():
            break
    speed = q * np.sqrt(2.0 * G * M / np.sqrt(r * r + a * a))
    v = speed[:, None] * direction(seed, 2003, i)
    return {"pos": x, "vel": v, "mass": np.full(n, M / n)}


def rotation_matrix(axis, angle):
    """R = c I + (1 - c) a a^T + s [a]x for the unit axis a (ParticleSource::rotate,
    src/initialConditions/ParticleSource.h:128-148)."""
    a = np.asarray(axis, dtype=np.float64)
    a = a / np.linalg.norm(a)
    c, s = np.cos(angle), np.sin(angle)
    K = np.array([[0.0, -a[2], a[1]], [a[2], 0.0, -a[0]], [-a[1], a[0], 0.0]])
    return c * np.eye(3) + (1.0 - c) * np.outer(a, a) + s * K


def modify(state, ops, com=(0.0, 0.0, 0.0), vcom=(0.0, 0.0, 0.0)):
    """The modifier list (grasph2_b200.ics op_* tuples) applied to a host state in FP64, with the same
    counter-based draws as the device; returns (state, desired COM, desired velocity of the COM), the COM
    bookkeeping following ParticleSource.h:93-148."""
    st = {k: np.array(v, dtype=np.float64) for k, v in state.items()}
    n = st["pos"].shape[0] if "pos" in st else st["mass"].shape[0]
    i = np.arange(n, dtype=np.uint64)
    com = np.array(com, dtype=np.float64)
    vcom = np.array(vcom, dtype=np.float64)
    for kind, v, seed in ops:
        name, _, attr = kind.partition(":")
        if name == "move":
            st["pos"] += np.array(v)
            com += np.array(v)
        elif name == "rotate":
            R = rotation_matrix(v[:3], v[3])
            st["pos"] = st["pos"] @ R.T
            st["vel"] = st["vel"] @ R.T
            com = R @ com
            vcom = R @ vcom
        elif name in ("pos_noise", "random_vel"):
            key = "pos" if name == "pos_noise" else "vel"
            d = np.stack([2.0 * uniform(seed, c, i) - 1.0 for c in range(3)], axis=1)
            st[key] += v[0] * d
        elif name == "angular_vel":
            w = np.array(v)
            st["vel"] += np.cross(w[None, :], st["pos"])
            vcom += np.cross(w, com)
        elif name == "linear_vel":
            st["vel"] += np.array(v)
            vcom += np.array(v)
        elif name == "set_constant":
            st[attr].reshape(n, -1)[:] = np.array(v)[None, :]
    return st, com, vcom
