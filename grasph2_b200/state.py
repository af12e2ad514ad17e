"""Host particle state in the reference's attribute layout.

A state is a dict of numpy arrays, one per attribute of particle_bases
(src/particles/partice_attributes.h:91-106): pos (n,3), mass (n,), vel (n,3), acc (n,3),
balsara (n,), xvel (n,3), density (n,), density_dt (n,), dstress (n,3,3), dstress_dt (n,3,3),
maxvsig (n,). The tensors are row-major 3x3 as in the reference's tsv/h5 output
(src/ResultStorageManager.cu:141-149).
"""

import ctypes

import numpy as np

from ._abi import ATTRIBUTES

SHAPES = {"pos": (3,), "mass": (), "vel": (3,), "acc": (3,), "balsara": (), "xvel": (3,), "density": (),
          "density_dt": (), "dstress": (3, 3), "dstress_dt": (3, 3), "maxvsig": ()}


def new_state(n, dtype=np.float32):
    return {name: np.zeros((n,) + SHAPES[name], dtype=dtype) for name, _, _ in ATTRIBUTES}


def as_dtype(state, dtype):
    return {k: np.ascontiguousarray(v, dtype=dtype) for k, v in state.items()}


def copy_state(state):
    return {k: v.copy() for k, v in state.items()}


def pointer_struct(state, struct_type, ctype):
    """Fill a ctypes struct of per-attribute pointers (GsphHostParticles / OracleParticles)
    with the arrays of `state`. Arrays must be C-contiguous of the matching dtype."""
    s = struct_type()
    for name, _, _ in ATTRIBUTES:
        a = state.get(name)
        if a is None:
            continue
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("attribute %s is not C-contiguous" % name)
        setattr(s, name, a.ctypes.data_as(ctypes.POINTER(ctype)))
    return s


def state_size(state):
    return int(state["mass"].shape[0])
