"""The C-ABI library: it loads, exports every entry point include/grasph2_b200.h declares, its struct
layouts match the ctypes mirror, and the host-only entry points validate their arguments.
CPU only: nothing here launches a kernel."""

import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from grasph2_b200 import _abi
from grasph2_b200.params import make_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "grasph2_b200.h")


@pytest.fixture(scope="session")
def lib():
    from grasph2_b200 import build
    build.build()
    return _abi.load_library()


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gsph_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_expected_entry_points():
    fns = declared_functions()
    for f in ("gsph_create", "gsph_destroy", "gsph_upload", "gsph_download", "gsph_compute_derivatives",
              "gsph_integrate", "gsph_step", "gsph_current_timestep", "gsph_diagnostics", "gsph_last_error"):
        assert f in fns


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (gsph_[a-z0-9_]+)", out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    for f in declared_functions():
        getattr(lib, f)


def test_ctypes_signatures_cover_header():
    assert sorted(_abi._SIGNATURES) == declared_functions()


def test_struct_layouts_match_c():
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "grasph2_b200.h"
int main(void){
  printf("%zu %zu %zu %zu %zu\n", sizeof(gsph_params), sizeof(gsph_options), sizeof(gsph_host_particles),
         sizeof(gsph_diag), sizeof(gsph_device_view));
  printf("%zu %zu %zu %zu\n", offsetof(gsph_params, H), offsetof(gsph_params, const_acc),
         offsetof(gsph_params, box_reflectiveness), offsetof(gsph_diag, mass));
  return 0;}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "l")
        subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(x) for x in lines[0].split()]
    assert sizes == [ctypes.sizeof(_abi.GsphParams), ctypes.sizeof(_abi.GsphOptions),
                     ctypes.sizeof(_abi.GsphHostParticles), ctypes.sizeof(_abi.GsphDiag),
                     ctypes.sizeof(_abi.GsphDeviceView)]
    offs = [int(x) for x in lines[1].split()]
    assert offs == [_abi.GsphParams.H.offset, _abi.GsphParams.const_acc.offset,
                    _abi.GsphParams.box_reflectiveness.offset, _abi.GsphDiag.mass.offset]


def test_reference_defaults_are_valid(lib):
    p = _abi.GsphParams()
    assert lib.gsph_params_reference_defaults(ctypes.byref(p)) == 0
    buf = ctypes.create_string_buffer(200)
    assert lib.gsph_params_validate(ctypes.byref(p), buf, 200) == 0
    assert p.flags & _abi.FLAG_BITS["SOLIDS"] and p.flags & _abi.FLAG_BITS["PLASTICITY_MC"]
    assert abs(p.H - 0.1 * 2 ** (-14 / 3) * 2.5) < 1e-15
    ref = make_params()  # python defaults mirror settings.h too
    assert ref.flags == p.flags and abs(ref.soundspeed - p.soundspeed) < 1e-9 * p.soundspeed


@pytest.mark.parametrize("field,value,needle", [
    ("H", 0.0, "H must be positive"),
    ("flags", 1 << 20, "unknown flag"),
    ("dimension", 4, "dimension"),
    ("grav_eps", -1.0, "grav_eps"),
])
def test_validate_rejects(lib, field, value, needle):
    p = make_params()
    setattr(p, field, value)
    buf = ctypes.create_string_buffer(200)
    assert lib.gsph_params_validate(ctypes.byref(p), buf, 200) == _abi.GSPH_E_INVALID
    assert needle in buf.value.decode()


def test_validate_rejects_two_plasticity_models(lib):
    p = make_params(switches=("SPH", "SOLIDS", "PLASTICITY_MIESE", "PLASTICITY_MC"))
    buf = ctypes.create_string_buffer(200)
    assert lib.gsph_params_validate(ctypes.byref(p), buf, 200) == _abi.GSPH_E_INVALID
    assert "plasticity" in buf.value.decode()


def test_null_arguments_are_errors(lib):
    assert lib.gsph_destroy(None) == _abi.GSPH_E_INVALID
    assert lib.gsph_compute_derivatives(None, None) == _abi.GSPH_E_INVALID
    assert lib.gsph_integrate(None, 1, None) == _abi.GSPH_E_INVALID
    assert lib.gsph_step(None, 1, None) == _abi.GSPH_E_INVALID
    assert lib.gsph_upload(None, 1, None, None) == _abi.GSPH_E_INVALID
    assert lib.gsph_size(None, None) == _abi.GSPH_E_INVALID
    out = ctypes.c_void_p()
    assert lib.gsph_create(None, None, 10, ctypes.byref(out)) == _abi.GSPH_E_INVALID
    assert b"NULL" in lib.gsph_last_error(None)
    p = make_params()
    assert lib.gsph_create(ctypes.byref(p), None, 0, ctypes.byref(out)) == _abi.GSPH_E_INVALID
    o = _abi.GsphOptions()
    o.accum = 7
    assert lib.gsph_create(ctypes.byref(p), ctypes.byref(o), 10, ctypes.byref(out)) == _abi.GSPH_E_INVALID
    assert b"accum" in lib.gsph_last_error(None)
    o = _abi.GsphOptions()
    o.j_tile = 100
    assert lib.gsph_create(ctypes.byref(p), ctypes.byref(o), 10, ctypes.byref(out)) == _abi.GSPH_E_INVALID


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_create_without_gpu_fails_cleanly(lib):
    p = make_params()
    out = ctypes.c_void_p()
    rc = lib.gsph_create(ctypes.byref(p), None, 100, ctypes.byref(out))
    assert rc == _abi.GSPH_E_CUDA and not out.value
    assert b"CUDA" in lib.gsph_last_error(None)
