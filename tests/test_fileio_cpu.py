"""Output files and surface geometry against the reference (CPU, no GPU needed).

* The writers of oscars_b200.fileio, given the values the reference wrote, reproduce the reference's
  ofile / bofile bytes exactly (tests/golden/files.npz, written by the reference build: flux and
  power density on rectangles and point surfaces in 2 and 3 dimensions, a spectrum, trajectories in
  the default and a custom column format).
* calculate_trajectory(ofile=, bofile=, oformat=) through a host-only context writes the same bytes
  as the reference (the host trajectory is bit-identical to the reference's).
* x0x1x2 rectangles and rotated / translated point surfaces give the reference's positions bit for
  bit (golden fixtures of those cases).
"""
import os

import numpy as np
import pytest

from cases import CASES, FILE_CASES, run_case

from oscars_b200 import fileio
from oscars_b200.sr import sr as SR

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FILES = np.load(os.path.join(GOLDEN, "files.npz"))
POINT_CASES = {"flux_rect_dim2": 2, "flux_rect_dim3": 3, "pd_rect": 2, "pd_points": 3}


def _golden_bytes(name, kind):
    return bytes(FILES[name + "/" + kind])


@pytest.mark.parametrize("name", sorted(POINT_CASES))
def test_point_files_byte_identical(name, tmp_path):
    pos, val, dim = FILES[name + "/pos"], FILES[name + "/val"], POINT_CASES[name]
    t, b = tmp_path / "o.txt", tmp_path / "o.bin"
    fileio.write_points_text(str(t), pos, val, dim)
    fileio.write_points_binary(str(b), pos, val, dim)
    assert t.read_bytes() == _golden_bytes(name, "txt")
    assert b.read_bytes() == _golden_bytes(name, "bin")


def test_spectrum_files_byte_identical(tmp_path):
    E, F = FILES["spectrum/pos"], FILES["spectrum/val"]
    t, b = tmp_path / "s.txt", tmp_path / "s.bin"
    fileio.write_spectrum_text(str(t), E, F)
    fileio.write_spectrum_binary(str(b), E, F)
    assert t.read_bytes() == _golden_bytes("spectrum", "txt")
    assert b.read_bytes() == _golden_bytes("spectrum", "bin")


@pytest.mark.parametrize("name", ["traj_default", "traj_format"])
def test_trajectory_files_byte_identical(name, tmp_path):
    setup, call, kw = FILE_CASES[name]
    t, b = tmp_path / "t.txt", tmp_path / "t.bin"
    s = SR(device=-1)
    res = run_case(s, setup + [(call, dict(kw, ofile=str(t), bofile=str(b)))])
    a = np.array([[p[0]] + p[1] + p[2] + p[3] for p in res], dtype=np.float64).T
    assert np.array_equal(a, FILES[name + "/traj"])
    assert t.read_bytes() == _golden_bytes(name, "txt")
    assert b.read_bytes() == _golden_bytes(name, "bin")


def test_trajectory_format_errors(tmp_path):
    a = FILES["traj_default/traj"]
    with pytest.raises(ValueError, match="format specifier not recognized"):
        fileio.write_trajectory_text(str(tmp_path / "x.txt"), a, "T Q")
    with pytest.raises(ValueError, match="at least one element"):
        fileio.write_trajectory_binary(str(tmp_path / "x.bin"), a, "   ")


@pytest.mark.parametrize("name", ["flux_x0x1x2", "flux_x0x1x2_dim2", "pd_x0x1x2"])
def test_x0x1x2_positions_bit_exact(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    last, kw = CASES[name][-1]
    xyz, _, x12 = SR(device=-1)._rectangle(kw["npoints"], kw.get("plane", "XY"), kw.get("width"), kw["x0x1x2"],
                                           kw.get("rotations"), kw.get("translation"), kw.get("normal", 0),
                                           last.startswith("calculate_power"))
    pos = (xyz if kw.get("dim", 2) == 3 else x12).reshape(-1, 3)
    assert np.array_equal(pos, g["pos"])


@pytest.mark.parametrize("name", ["pd_points", "pd_points_directional", "pd_points_inverted"])
def test_point_surface_positions_bit_exact(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    kw = CASES[name][-1][1]
    xyz, _ = SR(device=-1)._surface_points(kw["points"], kw.get("rotations"), kw.get("translation"),
                                           kw.get("normal", 0) == -1)
    assert np.array_equal(xyz.reshape(-1, 3), g["pos"])


def test_surface_argument_errors():
    s = SR(device=-1)
    with pytest.raises(ValueError, match="'x0x1x2' must have 3 XYZ points"):
        s._rectangle([5, 5], "XY", None, [[0, 0, 30], [1, 0, 30]], None, None, 0, False)
    with pytest.raises(ValueError, match=">= 2 in each direction"):
        s._rectangle([1, 5], "XY", None, [[0, 0, 30], [1, 0, 30], [0, 1, 30]], None, None, 0, False)
    with pytest.raises(ValueError, match="Incorrect format in 'points'"):
        s._surface_points([[[0, 0, 30]]], None, None, False)
    with pytest.raises(ValueError, match="Point or Normal does not have 3 elements"):
        s._surface_points([[[0, 0], [0, 0, 1]]], None, None, False)
