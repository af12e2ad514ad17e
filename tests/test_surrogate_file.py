"""The native surrogate model file (gsph_surrogate_load): malformed files and arguments are rejected
with GSPH_E_INVALID before any device work, so these run without a GPU."""

import ctypes

import numpy as np
import pytest

from grasph2_b200 import _abi


@pytest.fixture(scope="module")
def lib():
    return _abi.load_library()


def _file(path, magic=b"GSPHSUR1", K=8, count=None, nparams=None, nstats=90, extra=b""):
    lib = _abi.load_library()
    n = int(lib.gsph_mlp_param_count())
    with open(path, "wb") as f:
        f.write(magic)
        f.write(np.array([K, n if count is None else count], dtype="<i4").tobytes())
        f.write(np.zeros(n if nparams is None else nparams, dtype="<f4").tobytes())
        f.write(np.ones(nstats, dtype="<f4").tobytes())
        f.write(extra)


@pytest.mark.parametrize("case", ["magic", "count", "short", "trailing"])
def test_malformed_model_files_are_rejected(lib, tmp_path, case):
    f = str(tmp_path / "bad.gsur")
    kw = {"magic": dict(magic=b"GSPHSUR0"), "count": dict(count=1000), "short": dict(nstats=89),
          "trailing": dict(extra=b"\0")}[case]
    _file(f, **kw)
    h = ctypes.c_void_p()
    assert lib.gsph_surrogate_load(f.encode(), ctypes.byref(h)) == -1
    assert not h.value
    assert b"not a surrogate model file" in lib.gsph_last_error(None)


def test_missing_file_and_bad_arguments(lib, tmp_path):
    h = ctypes.c_void_p()
    assert lib.gsph_surrogate_load(str(tmp_path / "none.gsur").encode(), ctypes.byref(h)) == -1
    assert lib.gsph_surrogate_create(None, None, None, None, None, 0, ctypes.byref(h)) == -1  # K < 1
    sig = np.ones(32, dtype=np.float32)
    sig[7] = 0.0
    fp = sig.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    assert lib.gsph_surrogate_create(None, None, fp, None, None, 8, ctypes.byref(h)) == -1  # sigma must be > 0
    assert not h.value
    assert lib.gsph_surrogate_propose(None, None, 1, None) == -1
    assert lib.gsph_surrogate_substeps(None) == 0
