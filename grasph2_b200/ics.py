"""Seeded initial conditions for the named workloads.

The reference draws its spheres with mpUtils' random point pickers (UniformSphere.cu:39,
PlummerSphere.cu:39-88, not vendored); these generators produce the same distributions from
numpy's PCG64 so that the CUDA path and the oracle receive identical arrays:

* uniform sphere: radius R*U^(1/3), isotropic direction, equal masses, density = rest density
  (src/initialConditions/particleSources/UniformSphere.cu:35-44), optional rigid rotation
  v = omega x r (ParticleSource::addAngularVelocity);
* Plummer sphere: r = a (U^(-2/3) - 1)^(-1/2) (PlummerSphere.cu:41-51, no cutoff), speeds from
  the von Neumann rejection of g(q) = q^2 (1-q^2)^(7/2) with v = q sqrt(2GM / sqrt(r^2+a^2))
  (PlummerSphere.cu:60-88);
* centre-of-mass and centre-of-mass-velocity correction (InitGenerator.h:113-152).
"""

import math

import numpy as np

from .state import new_state


def _isotropic(rng, n):
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    return np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)


def uniform_sphere_positions(rng, n, radius):
    r = radius * rng.uniform(0.0, 1.0, n) ** (1.0 / 3.0)
    return _isotropic(rng, n) * r[:, None]


def _com_correct(state):
    m = state["mass"].astype(np.float64)
    for key in ("pos", "vel"):
        a = state[key].astype(np.float64)
        c = (m[:, None] * a).sum(0) / m.sum()
        state[key] = (a - c).astype(state[key].dtype)


def uniform_sphere(n, radius=1.0, total_mass=1.0, rho0=1.0, omega=(0.0, 0.0, 0.0), seed=0, dtype=np.float64,
                   com_correct=True):
    rng = np.random.Generator(np.random.PCG64(seed))
    st = new_state(n, dtype)
    x = uniform_sphere_positions(rng, n, radius)
    st["pos"][:] = x
    st["mass"][:] = total_mass / n
    st["density"][:] = rho0
    st["vel"][:] = np.cross(np.asarray(omega, dtype=np.float64)[None, :], x)
    if com_correct:
        _com_correct(st)
    return st


def two_sphere_impact(n_big=58254, n_small=7282, r_big=1.0, r_small=0.5, v_rel=0.5, y_offset=0.3, rho0=1.0,
                      seed=0, dtype=np.float64):
    """Two uniform spheres of equal number density: the big one at rest at the origin, the small
    one touching its surface with centre offset y_offset in y and moving +x at v_rel; then the
    centre-of-mass frame. Masses m = rho0 * V_total / N."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = n_big + n_small
    st = new_state(n, dtype)
    xb = uniform_sphere_positions(rng, n_big, r_big)
    xs = uniform_sphere_positions(rng, n_small, r_small)
    d = r_big + r_small
    xs += np.array([-math.sqrt(d * d - y_offset * y_offset), y_offset, 0.0])
    st["pos"][:n_big] = xb
    st["pos"][n_big:] = xs
    vol = 4.0 / 3.0 * math.pi * (r_big ** 3 + r_small ** 3)
    st["mass"][:] = rho0 * vol / n
    st["density"][:] = rho0
    st["vel"][n_big:, 0] = v_rel
    _com_correct(st)
    return st


def plummer_sphere(n, a=1.0, total_mass=1.0, G=1.0, seed=0, dtype=np.float64):
    rng = np.random.Generator(np.random.PCG64(seed))
    st = new_state(n, dtype)
    u = rng.uniform(0.0, 1.0, n)
    u = np.clip(u, 1e-300, 1.0 - 1e-16)
    r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    st["pos"][:] = _isotropic(rng, n) * r[:, None]
    q = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        x = rng.uniform(0.0, 1.0, todo.size)
        y = rng.uniform(0.0, 0.1, todo.size)
        ok = y <= x * x * (1.0 - x * x) ** 3.5
        q[todo[ok]] = x[ok]
        todo = todo[~ok]
    speed = q * np.sqrt(2.0 * G * total_mass / np.sqrt(r * r + a * a))
    st["vel"][:] = _isotropic(rng, n) * speed[:, None]
    st["mass"][:] = total_mass / n
    _com_correct(st)
    return st


def ensemble_sizes(count=512, lo=1024, hi=32768, seed=0):
    """Seeded log-uniform integer sizes in [lo, hi]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi + 1), count))).astype(np.int64).clip(lo, hi)


# ---- generators on the device (gsph_ic_*): torch CUDA tensors in the host layout ------------------
def _dev(n, k=None):
    import torch
    return torch.empty((n, k) if k else (n,), dtype=torch.float32, device="cuda")


def _com(lib, n, st):
    import ctypes
    import torch
    scratch = torch.empty(7 * 256, dtype=torch.float64, device="cuda")
    rc = lib.gsph_ic_com_correct(n, ctypes.c_void_p(st["pos"].data_ptr()), ctypes.c_void_p(st["vel"].data_ptr()),
                                 ctypes.c_void_p(st["mass"].data_ptr()), ctypes.c_void_p(scratch.data_ptr()), None)
    if rc != 0:
        raise RuntimeError(lib.gsph_last_error(None).decode())


def uniform_sphere_device(n, radius=1.0, total_mass=1.0, rho0=1.0, omega=(0.0, 0.0, 0.0), seed=0, com_correct=True):
    """Uniform sphere generated on the GPU (counter-based draws; see include/grasph2_b200.h)."""
    import ctypes
    from ._abi import load_library
    lib = load_library()
    st = {"pos": _dev(n, 3), "vel": _dev(n, 3), "mass": _dev(n), "density": _dev(n)}
    w = (ctypes.c_double * 3)(*omega)
    rc = lib.gsph_ic_uniform_sphere(n, radius, total_mass, rho0, w, seed, *(ctypes.c_void_p(st[k].data_ptr())
                                    for k in ("pos", "vel", "mass", "density")), None)
    if rc != 0:
        raise RuntimeError(lib.gsph_last_error(None).decode())
    if com_correct:
        _com(lib, n, st)
    return st


def plummer_sphere_device(n, a=1.0, total_mass=1.0, G=1.0, seed=0, com_correct=True):
    """Plummer sphere generated on the GPU."""
    import ctypes
    from ._abi import load_library
    lib = load_library()
    st = {"pos": _dev(n, 3), "vel": _dev(n, 3), "mass": _dev(n)}
    rc = lib.gsph_ic_plummer(n, a, total_mass, G, seed, *(ctypes.c_void_p(st[k].data_ptr())
                             for k in ("pos", "vel", "mass")), None)
    if rc != 0:
        raise RuntimeError(lib.gsph_last_error(None).decode())
    if com_correct:
        _com(lib, n, st)
    return st


# ---- particle-source modifiers on the device (gsph_ic_modify; ParticleSource.h:65-74) ---------------
def op_move(dx):
    """pos += dx (ParticleSource::move)"""
    return ("move", tuple(float(x) for x in dx), 0)


def op_rotate(axis, angle):
    """pos = R pos, vel = R vel about `axis` by `angle` radians (ParticleSource::rotate)"""
    return ("rotate", tuple(float(x) for x in axis) + (float(angle),), 0)


def op_positional_noise(strength, seed):
    """pos += uniform in [-strength, strength) per component (ParticleSource::addPositionalNoise)"""
    return ("pos_noise", (float(strength),), int(seed))


def op_angular_velocity(omega):
    """vel += omega x pos (ParticleSource::addAngularVelocity)"""
    return ("angular_vel", tuple(float(x) for x in omega), 0)


def op_linear_velocity(v):
    """vel += v (ParticleSource::addLinearVelocity)"""
    return ("linear_vel", tuple(float(x) for x in v), 0)


def op_random_velocity(strength, seed):
    """vel += uniform in [-strength, strength) per component (ParticleSource::addRandomVelocity)"""
    return ("random_vel", (float(strength),), int(seed))


def op_set_constant(attribute, value):
    """attribute (a state name, e.g. "density") = value for every particle (ParticleSource::setConstant)"""
    return ("set_constant:" + attribute, tuple(float(x) for x in np.atleast_1d(value)), 0)


_OP_KIND = {"move": 1, "rotate": 2, "pos_noise": 3, "angular_vel": 4, "linear_vel": 5, "random_vel": 6,
            "set_constant": 7}


def modify_device(st, ops, desired_com=(0.0, 0.0, 0.0), desired_vel_of_com=(0.0, 0.0, 0.0)):
    """Apply the modifiers `ops` (op_* tuples, in order) to the device state `st` (torch CUDA tensors in the
    host layout) on the GPU. Returns the desired centre of mass and its velocity after the ops (the
    reference's m_desiredCOM / m_desiredVelOfCOM), the targets of com_set_device."""
    import ctypes
    from ._abi import ATTR_BITS, GsphHostParticles, GsphIcOp, load_library
    lib = load_library()
    arr = (GsphIcOp * max(1, len(ops)))()
    for k, (kind, v, seed) in enumerate(ops):
        name, _, attr = kind.partition(":")
        arr[k].kind = _OP_KIND[name]
        arr[k].attr = ATTR_BITS[attr] if attr else 0
        arr[k].seed = seed
        for j, x in enumerate(v):
            arr[k].v[j] = x
    view = GsphHostParticles()
    for name, t in st.items():
        setattr(view, name, ctypes.cast(ctypes.c_void_p(t.data_ptr()), ctypes.POINTER(ctypes.c_float)))
    com = (ctypes.c_double * 3)(*desired_com)
    vcom = (ctypes.c_double * 3)(*desired_vel_of_com)
    rc = lib.gsph_ic_modify(st["mass"].shape[0] if "mass" in st else st["pos"].shape[0], arr, len(ops),
                            ctypes.byref(view), com, vcom, None)
    if rc != 0:
        raise RuntimeError(lib.gsph_last_error(None).decode())
    return tuple(com), tuple(vcom)


def com_set_device(st, com=None, vel_of_com=None):
    """Shift the device state's mass-weighted mean position / velocity to com / vel_of_com (None: leave)
    (the per-source correction of InitGenerator.h:113-152)."""
    import ctypes
    import torch
    from ._abi import load_library
    lib = load_library()
    scratch = torch.empty(7 * 256, dtype=torch.float64, device="cuda")
    c = (ctypes.c_double * 3)(*com) if com is not None else None
    v = (ctypes.c_double * 3)(*vel_of_com) if vel_of_com is not None else None
    rc = lib.gsph_ic_com_set(st["mass"].shape[0], ctypes.c_void_p(st["pos"].data_ptr()),
                             ctypes.c_void_p(st["vel"].data_ptr()), ctypes.c_void_p(st["mass"].data_ptr()), c, v,
                             ctypes.c_void_p(scratch.data_ptr()), None)
    if rc != 0:
        raise RuntimeError(lib.gsph_last_error(None).decode())


def two_sphere_impact_device(n_big=58254, n_small=7282, r_big=1.0, r_small=0.5, v_rel=0.5, y_offset=0.3, rho0=1.0,
                             seed=0):
    """The two-sphere impact assembled on the GPU as the reference's initial-condition generator would: two
    uniform sphere sources of equal number density, the small one moved to touch the big one's surface at
    y-offset `y_offset` and given velocity v_rel along x, each source's centre of mass and its velocity
    corrected to the desired values its modifiers imply (InitGenerator.h:113-152)."""
    import torch
    n = n_big + n_small
    vol_big = 4.0 / 3.0 * math.pi * r_big ** 3
    m = rho0 * vol_big / n_big
    st = {"pos": _dev(n, 3), "vel": _dev(n, 3), "mass": _dev(n), "density": _dev(n)}
    parts = []
    for (nk, rk, sk) in ((n_big, r_big, seed), (n_small, r_small, seed + 1)):
        part = uniform_sphere_device(nk, radius=rk, total_mass=m * nk, rho0=rho0, seed=sk, com_correct=False)
        parts.append(part)
    dx = -math.sqrt(max(0.0, (r_big + r_small) ** 2 - y_offset ** 2))
    for part, ops in ((parts[0], []),
                      (parts[1], [op_move((dx, y_offset, 0.0)), op_linear_velocity((v_rel, 0.0, 0.0))])):
        com, vcom = modify_device(part, ops)
        com_set_device(part, com, vcom)
    off = 0
    for part in parts:
        k = part["mass"].shape[0]
        for key in st:
            st[key][off:off + k] = part[key]
        off += k
    torch.cuda.synchronize()
    return st
