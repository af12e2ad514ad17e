"""The C++ adapter (include/grasph2_b200.hpp) driving the library the way the reference's main loop
drives its own hot path: compiled with g++ against libgrasph2_b200.so and run on the GPU."""

import os
import subprocess
import tempfile

import pytest

from grasph2_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.gpu
def test_cpp_adapter_main_loop():
    assert os.path.exists(_abi.LIB_PATH)
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "adapter_check")
        subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "adapter_check.cpp"), "-L", os.path.dirname(_abi.LIB_PATH),
                        "-lgrasph2_b200", "-Wl,-rpath," + os.path.dirname(_abi.LIB_PATH), "-o", exe], check=True)
        model = os.path.join(ROOT, "grasph2_b200", "data", "surrogate_impact_n262144.gsur")
        assert os.path.exists(model), model
        r = subprocess.run([exe, d, model], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "ADAPTER OK" in r.stdout
