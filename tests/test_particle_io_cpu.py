"""Particle files and manifests (ao_read_particles / ao_read_manifest), on CPU.

Formats of the reference's tests/particle_io.hpp and benchmark drivers: text
rows of four numbers (charge-x-y-z or x-y-z-charge) or ESC, blank and '#'
rows skipped; binary xyz frames with NaN for an escaped particle.
"""
import numpy as np
import pytest

from adaptive_trees_b200 import io
from adaptive_trees_b200._capi import AoError


def test_text_layouts_comments_and_escaped(tmp_path):
    f = tmp_path / "snap.dat"
    f.write_text("# charge x y z\n\n1.0 0.1 0.2 0.3\n  -1 +0.4 5e-1 0.6  # trailing comment\nESC\n"
                 "0.5 1e-3 2E-3 3e-3\n")
    x, y, z = io.read_particles(f, "cxyz")
    assert np.array_equal(x, [0.1, 0.4, io.ESCAPED, 1e-3])
    assert np.array_equal(y, [0.2, 0.5, io.ESCAPED, 2e-3])
    assert np.array_equal(z, [0.3, 0.6, io.ESCAPED, 3e-3])
    x, y, z = io.read_particles(f, io.XYZ_CHARGE)
    assert np.array_equal(x[:2], [1.0, -1.0]) and np.array_equal(z[:2], [0.2, 0.5])


def test_binary_frames_and_manifest(tmp_path):
    pts = np.array([[0.1, 0.2, 0.3], [np.nan, 0, 0], [0.7, 0.8, 0.9]])
    (tmp_path / "frames").mkdir()
    pts.tofile(tmp_path / "frames" / "f0.bin")
    (tmp_path / "frames" / "f1.dat").write_text("0 0.11 0.21 0.31\nESC\n0 0.71 0.81 0.91\n")
    m = tmp_path / "set.manifest"
    m.write_text("# dataset manifest\ndataset toy\nslots 3\nbox 0 1 0 1 0 1\n"
                 "frame 0 100 bin frames/f0.bin\nframe 1 101 cxyz frames/f1.dat\n")
    man = io.read_manifest(m)
    assert man["dataset"] == "toy" and man["slots"] == 3 and man["box"] == (0, 1, 0, 1, 0, 1)
    assert [f["id"] for f in man["frames"]] == [100, 101]
    x, y, z = io.read_frame(man["frames"][0])
    assert np.array_equal(x, [0.1, io.ESCAPED, 0.7]) and np.array_equal(z, [0.3, io.ESCAPED, 0.9])
    x, _, _ = io.read_frame(man["frames"][1])
    assert np.array_equal(x, [0.11, io.ESCAPED, 0.71])


def test_errors(tmp_path):
    bad = tmp_path / "bad.dat"
    bad.write_text("1 2 3\n")
    with pytest.raises(AoError, match="four numbers"):
        io.read_particles(bad)
    with pytest.raises(AoError, match="cannot open"):
        io.read_particles(tmp_path / "missing.dat")
    (tmp_path / "odd.bin").write_bytes(b"\0" * 10)
    with pytest.raises(AoError, match="xyz doubles"):
        io.read_particles(tmp_path / "odd.bin", io.BINARY_XYZ)
    (tmp_path / "empty.manifest").write_text("dataset x\n")
    with pytest.raises(AoError):
        io.read_manifest(tmp_path / "empty.manifest")
