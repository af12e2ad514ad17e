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
