"""tsv snapshot files byte for byte against GraSPH2's own writer and reader (CPU).

oracle/_ref/libref_io.so is the reference's ResultStorageManager::printTextFile with its attributePrinter
(src/ResultStorageManager.cu:102-186) and its TextFile particle source
(src/initialConditions/particleSources/TextFile.h:43-170), compiled unchanged for the host
(oracle/ref_io_driver.cpp). The library's side is the C++ adapter (include/grasph2_b200.hpp:
snapshotFileName, printTextFile, readTextFile), driven by tests/cpp/tsv_check.cpp. The async device
writer (gsph_writer_*) is checked against the same reference bytes in test_gpu_writer.py.
"""

import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_IO = os.path.join(ROOT, "oracle", "_ref", "libref_io.so")

if not os.path.exists(REF_IO):
    pytest.skip("the reference's tsv writer (oracle/_ref/libref_io.so) is not built", allow_module_level=True)

_fp = ctypes.POINTER(ctypes.c_float)


def ref_io():
    L = ctypes.CDLL(REF_IO)
    L.refio_print_text.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int64, _fp, _fp, _fp,
                                   _fp, ctypes.c_double]
    L.refio_read_text.argtypes = [ctypes.c_char_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), _fp, _fp, _fp, _fp]
    return L


def particles(n, seed):
    """Values across the magnitudes a snapshot holds: positions of order 1 with some far out, masses
    down to 1e-9 (printed as 0.0000000 in fixed notation), signed velocities, densities up to 1e5."""
    rng = np.random.default_rng(seed)
    pos = rng.normal(size=(n, 3)).astype(np.float32)
    pos[::97] *= 1.0e4
    mass = (10.0 ** rng.uniform(-9, 0, n)).astype(np.float32)
    vel = rng.normal(scale=0.3, size=(n, 3)).astype(np.float32)
    vel[::13] = -vel[::13]
    density = (10.0 ** rng.uniform(-3, 5, n)).astype(np.float32)
    density[7] = 0.0
    return pos, mass, vel, density


def ptr(a):
    return np.ascontiguousarray(a, dtype=np.float32).ctypes.data_as(_fp)


@pytest.fixture(scope="module")
def tsv_check(tmp_path_factory):
    d = tmp_path_factory.mktemp("tsvbin")
    exe = os.path.join(str(d), "tsv_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "tsv_check.cpp"), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("time", [0.0, 0.05, 1.25, 123.456789])
def test_snapshot_file_equals_the_reference_byte_for_byte(tmp_path, tsv_check, time):
    n = 1000
    pos, mass, vel, density = particles(n, seed=int(time * 1000) + 1)
    ref_dir = tmp_path / "ref"
    our_dir = tmp_path / "ours"
    ref_dir.mkdir()
    our_dir.mkdir()
    L = ref_io()
    keep = [np.ascontiguousarray(a) for a in (pos, mass, vel, density)]
    rc = L.refio_print_text((str(ref_dir) + "/").encode(), b"graSPH2_", b"2026-12-03_18-40", n,
                            *[ptr(a) for a in keep], time)
    assert rc == 0
    ref_files = os.listdir(ref_dir)
    assert len(ref_files) == 1
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        for a in keep:
            f.write(a.tobytes())
    r = subprocess.run([tsv_check, "write", str(our_dir) + "/", "graSPH2_", "2026-12-03_18-40", repr(time), str(n),
                        str(inp)], capture_output=True, text=True, check=True)
    ours = r.stdout.strip()
    assert os.path.basename(ours) == ref_files[0]  # <prefix><start>_<time, fixed 7 digits>.tsv
    a = open(ref_dir / ref_files[0], "rb").read()
    b = open(ours, "rb").read()
    assert a == b
    assert a.count(b"\n") == n


def test_reader_equals_the_reference_value_for_value(tmp_path, tsv_check):
    """Both readers on the same file (the reference's own output, blank lines added) give the same float32
    bits: each token is parsed as a double and rounded to float, as TextFile does."""
    n = 2000
    pos, mass, vel, density = particles(n, seed=9)
    L = ref_io()
    keep = [np.ascontiguousarray(a) for a in (pos, mass, vel, density)]
    assert L.refio_print_text((str(tmp_path) + "/").encode(), b"p_", b"t", n, *[ptr(a) for a in keep], 0.5) == 0
    (name,) = [f for f in os.listdir(tmp_path) if f.endswith(".tsv")]
    path = tmp_path / name
    lines = open(path).read().split("\n")
    lines.insert(10, "   ")
    lines.insert(500, "")
    open(path, "w").write("\n".join(lines))
    got = {k: np.zeros(s, np.float32) for k, s in (("pos", 3 * n), ("mass", n), ("vel", 3 * n), ("density", n))}
    cnt = ctypes.c_int64(0)
    assert L.refio_read_text(str(path).encode(), n, ctypes.byref(cnt), *[ptr(got[k]) for k in
                                                                          ("pos", "mass", "vel", "density")]) == 0
    assert cnt.value == n
    out = tmp_path / "out.bin"
    subprocess.run([tsv_check, "read", str(path), str(out)], check=True)
    raw = open(out, "rb").read()
    assert np.frombuffer(raw[:8], np.int64)[0] == n
    ours = np.frombuffer(raw[8:], np.float32)
    want = np.concatenate([got["pos"], got["mass"], got["vel"], got["density"]])
    np.testing.assert_array_equal(ours.view(np.uint32), want.view(np.uint32))
