"""Asynchronous snapshot writer: files equal synchronous downloads of the same states."""

import numpy as np
import pytest

from grasph2_b200 import ics
from grasph2_b200.params import config0_params
from grasph2_b200.sim import DeviceParticleBuffer, SnapshotWriter

pytestmark = pytest.mark.gpu


def read_tsv(path):
    return np.loadtxt(path, delimiter="\t", usecols=range(8), dtype=np.float64)


def test_async_snapshots_match_downloads(tmp_path):
    p = config0_params()
    n = 3000
    st = ics.uniform_sphere(n, rho0=0.239, omega=(0, 0, 0.1), seed=5)
    want = []
    with DeviceParticleBuffer(p, n) as pb:
        pb.upload(st)
        with SnapshotWriter(pb, depth=2) as w:
            for k in range(4):
                pb.step(3)
                w.write(tmp_path / ("snap_%d.tsv" % k))
                d = pb.download(["pos", "mass", "vel", "density"])
                want.append(np.concatenate([d["pos"], d["mass"][:, None], d["vel"], d["density"][:, None]], 1))
            assert w.flush() == 4
    for k in range(4):
        got = read_tsv(tmp_path / ("snap_%d.tsv" % k))
        # the tsv holds digits10 + 1 = 7 significant decimal digits of each float
        np.testing.assert_allclose(got, want[k], rtol=2e-6, atol=1e-7)


def test_writer_reports_a_failed_file(tmp_path):
    p = config0_params()
    st = ics.uniform_sphere(500, rho0=0.239, seed=6)
    with DeviceParticleBuffer(p, 500) as pb:
        pb.upload(st)
        w = SnapshotWriter(pb, depth=1)
        w.write(tmp_path / "missing_dir" / "x.tsv")
        w.write(tmp_path / "ok.tsv")  # the single slot frees once the first job has failed
        with pytest.raises(Exception):
            w.flush()
        with pytest.raises(Exception):
            w.close()
    assert (tmp_path / "ok.tsv").exists()


def test_async_snapshot_bytes_equal_the_reference_writer(tmp_path):
    """The file the device writer produces is byte for byte the one GraSPH2's own printTextFile
    (oracle/_ref/libref_io.so) writes from the same downloaded state."""
    import ctypes
    import os
    ref_io = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                          "libref_io.so")
    if not os.path.exists(ref_io):
        pytest.skip("oracle/_ref/libref_io.so is not built")
    fp = ctypes.POINTER(ctypes.c_float)
    L = ctypes.CDLL(ref_io)
    L.refio_print_text.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int64, fp, fp, fp, fp,
                                   ctypes.c_double]
    p = config0_params()
    n = 2048
    st = ics.uniform_sphere(n, rho0=0.239, omega=(0, 0, 0.1), seed=8)
    with DeviceParticleBuffer(p, n) as pb:
        pb.upload(st)
        pb.step(2)
        with SnapshotWriter(pb, depth=1) as w:
            w.write(tmp_path / "ours.tsv")
            assert w.flush() == 1
        d = pb.download(["pos", "mass", "vel", "density"])
    arrs = [np.ascontiguousarray(d[k], dtype=np.float32) for k in ("pos", "mass", "vel", "density")]
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    assert L.refio_print_text((str(ref_dir) + "/").encode(), b"s_", b"t", n,
                              *[a.ctypes.data_as(fp) for a in arrs], 0.0) == 0
    (name,) = os.listdir(ref_dir)
    assert open(ref_dir / name, "rb").read() == open(tmp_path / "ours.tsv", "rb").read()
