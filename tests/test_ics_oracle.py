"""Host restatement of the device IC generators: the draw function's known answer and distributions."""

import numpy as np

import ics_oracle as O


def test_splitmix64_known_answer():
    # splitmix64 from state 0 (Steele, Lea & Flood 2014; the reference implementation's first output)
    assert int(O.splitmix64(np.uint64(0))) == 0xE220A8397B1DCDAF


def test_uniform_draws_are_uniform():
    u = O.uniform(5, 2, np.arange(200000, dtype=np.uint64))
    assert 0.0 <= u.min() and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 3e-3 and abs(u.var() - 1.0 / 12.0) < 2e-3


def test_plummer_radii_follow_the_mass_profile():
    n = 50000
    st = O.plummer(n, 1.0, 1.0, 1.0, 3)
    r = np.sort(np.linalg.norm(st["pos"], axis=1))
    m = r ** 3 / (1.0 + r * r) ** 1.5  # enclosed mass fraction of a Plummer sphere with a = 1
    assert np.abs(m - np.arange(1, n + 1) / n).max() < 0.01
