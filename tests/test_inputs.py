"""Synthetic inputs and the reference's text formats (src/fileio.h)."""
import os

import numpy as np
import pytest

from mlfma_b200 import inputs


@pytest.mark.parametrize("level", [0, 1, 2, 3])
def test_icosphere_counts_and_closure(level):
    m = inputs.make_icosphere(level, radius=2.0)
    assert m.faces.shape[0] == 20 * 4 ** level
    assert m.vertices.shape[0] == 10 * 4 ** level + 2
    assert m.rwgs.shape[0] == 30 * 4 ** level
    np.testing.assert_allclose(np.linalg.norm(m.vertices, axis=1), 2.0, rtol=1e-14)
    for v0, v1, tp, tm in m.rwgs[:: max(1, m.n // 50)]:
        assert {v0, v1} <= set(m.faces[tp]) and {v0, v1} <= set(m.faces[tm]) and tp != tm


def test_icosphere_level5_edge_length():
    m = inputs.make_icosphere(5, radius=2.0)
    assert m.n == 30720 and m.faces.shape[0] == 20480
    e = np.linalg.norm(m.vertices[m.rwgs[:, 0]] - m.vertices[m.rwgs[:, 1]], axis=1)
    assert 0.06 < e.min() and e.max() < 0.09


def test_dipoles_seeded_and_in_box():
    a, b = inputs.make_dipoles(1000, side=4.0, seed=1), inputs.make_dipoles(1000, side=4.0, seed=1)
    np.testing.assert_array_equal(a.pos, b.pos)
    assert np.abs(a.pos).max() <= 2.0
    np.testing.assert_array_equal(a.mom, np.tile([1.0, 0, 0], (1000, 1)))


def test_text_formats_round_trip(tmp_path):
    d = inputs.make_dipoles(20, seed=3)
    p = tmp_path / "dip.txt"
    inputs.write_dipoles(str(p), d)
    d2 = inputs.read_dipoles(str(p))
    np.testing.assert_array_equal(d.pos, d2.pos)
    m = inputs.make_icosphere(1)
    inputs.write_rwg(str(tmp_path / "mesh"), m)
    m2 = inputs.read_rwg(str(tmp_path / "mesh"))
    np.testing.assert_array_equal(m.rwgs, m2.rwgs)
    np.testing.assert_array_equal(m.vertices, m2.vertices)
    pw = inputs.PlaneWave(amplitude=2.0, pol=(0, 1, 0), khat=(1, 0, 0), wavenum=3.0)
    inputs.write_planewave(str(tmp_path / "pw.txt"), pw)
    assert inputs.read_planewave(str(tmp_path / "pw.txt")) == pw


def test_readers_raise_like_the_reference(tmp_path):
    with pytest.raises(RuntimeError, match="Unable to find file"):
        inputs.read_planewave(str(tmp_path / "missing.txt"))
    (tmp_path / "bad.txt").write_text("1 2 3\n")
    with pytest.raises(RuntimeError, match="Unable to parse line"):
        inputs.read_planewave(str(tmp_path / "bad.txt"))
