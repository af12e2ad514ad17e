"""HDF5 snapshots (gsph_h5_*): the reference's STORE_HDF5 layout -- one float dataset per attribute, named
as the attribute, shape {N, components} (src/ResultStorageManager.cu:191-227) -- through the system's
libhdf5, loaded at run time. Without libhdf5 (this image has none) the calls must fail cleanly with
GSPH_E_UNSUPPORTED, as the reference falls back when HDF5_AVAILABLE is unset (CMakeLists.txt:123-130);
with it, a file round-trips exactly."""

import numpy as np
import pytest

from grasph2_b200 import _abi
from grasph2_b200.sim import GsphError, h5_available, read_h5, write_h5


def _state(n, seed):
    rng = np.random.default_rng(seed)
    return {"pos": rng.normal(size=(n, 3)).astype(np.float32), "mass": rng.uniform(size=n).astype(np.float32),
            "vel": rng.normal(size=(n, 3)).astype(np.float32), "density": rng.uniform(1, 2, n).astype(np.float32),
            "dstress": rng.normal(size=(n, 3, 3)).astype(np.float32)}


def test_h5_unavailable_fails_cleanly(tmp_path):
    if h5_available():
        pytest.skip("libhdf5 is installed: the round trip below covers it")
    with pytest.raises(GsphError) as e:
        write_h5(tmp_path / "x.h5", _state(10, 1))
    assert e.value.code == _abi.GSPH_E_UNSUPPORTED
    assert "libhdf5" in str(e.value)
    with pytest.raises(GsphError) as e:
        read_h5(tmp_path / "x.h5")
    assert e.value.code == _abi.GSPH_E_UNSUPPORTED


def test_h5_round_trip(tmp_path):
    if not h5_available():
        pytest.skip("libhdf5 is not installed")
    st = _state(1000, 2)
    names = ("pos", "mass", "vel", "density", "dstress")
    write_h5(tmp_path / "s.h5", st, names)
    back = read_h5(tmp_path / "s.h5", names)
    for k in names:
        np.testing.assert_array_equal(back[k], st[k], err_msg=k)
