"""STL meshes on the host: the product's reader and container against the reference.

The facets and centres that oscars_b200.stl builds from the committed meshes (tests/golden/stl/) are
compared bit for bit with the vertices the reference returned in every STL golden fixture, the
print_stl text with the reference's printer output, and the mesh file written for stlofile with the
bytes the reference wrote (stl_files.npz; its 80-byte header is partly uninitialised there, so only
the reference's text at its start is compared).  No GPU: the contexts are host-only.
"""
import os

import numpy as np
import pytest

from cases import CASES, STL_DIR, run_case, stl_file

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
STL_CASES = sorted(k for k, v in CASES.items() if v[-1][0] == "calculate_power_density_stl")


def _host_sr():
    from oscars_b200.sr import sr
    return sr(gpu=1, device=-1)


@pytest.mark.parametrize("name", STL_CASES)
def test_facets_match_reference_vertices(name):
    s = _host_sr()
    run_case(s, [c for c in CASES[name] if c[0] == "add_stl"])
    facets, centers = s._stl.facets()
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    assert np.array_equal(facets[:, 0:9].reshape(-1, 3, 3), g["pos"])
    from oracle.oracle import read_stl
    adds = [kw for c, kw in CASES[name] if c == "add_stl"]
    ref_c = np.vstack([read_stl(stl_file(kw["ifile"]), kw.get("scale", 1), kw.get("translation", [0, 0, 0]))[1]
                       for kw in adds])
    assert np.array_equal(centers, ref_c)


def test_print_stl_matches_reference_text(capsys):
    s = _host_sr()
    run_case(s, [c for c in CASES["stl_shadow"] if c[0] == "add_stl"])
    s.print_stl()
    out = capsys.readouterr().out
    expect = ("*STL Information*\nTSTLContainer has 2 STL Objects\n"
              "Name:             plate\nFilenName:        %s\nScale:            1\nRotations:        (0, 0, 0)\n"
              "Translation:      (0, 0, 20)\nNTriangles:       32\n\n"
              "Name:             shield\nFilenName:        %s\nScale:            0.001\nRotations:        (0, 0, 0)\n"
              "Translation:      (0, 0, 10)\nNTriangles:       2\n\n\n") % (stl_file("plate.stl"), stl_file("shield_mm.stl"))
    assert out == expect


def test_stl_output_file_matches_reference_bytes(tmp_path):
    s = _host_sr()
    run_case(s, [c for c in CASES["stl_shadow"] if c[0] == "add_stl"])
    path = str(tmp_path / "out.stl")
    s._stl.write_stl(path)
    data = open(path, "rb").read()
    g = np.load(os.path.join(GOLDEN, "stl_files.npz"))
    assert data[:37] == bytes(g["head"])
    assert data[80:] == bytes(g["body"])


def test_names_removal_and_errors(tmp_path):
    s = _host_sr()
    s.add_stl(stl_file("plate.stl"), name="a")
    with pytest.raises(ValueError, match="stl with this name already exists"):
        s.add_stl(stl_file("plate.stl"), name="a")
    s.add_stl(stl_file("shield_mm.stl"), scale=0.001)   # default name _stl1
    assert [m.name for m in s._stl.meshes] == ["a", "_stl1"] and len(s._stl) == 34
    s.remove_stl("a")
    assert [m.name for m in s._stl.meshes] == ["_stl1"]
    s.clear_stl()
    assert len(s._stl) == 0
    with pytest.raises(ValueError, match="cannot be opened"):
        s.add_stl(str(tmp_path / "missing.stl"))
    with pytest.raises(ValueError, match="Incorrect format in 'translation'"):
        s.add_stl(stl_file("plate.stl"), translation=[0, 0])
    with pytest.raises(ValueError, match="No particle beam defined"):
        s.calculate_power_density_stl([0, 0, 0])
    s.set_particle_beam(type="electron", energy_GeV=3, x0=[0, 0, 0], d0=[0, 0, 1], current=0.5)
    with pytest.raises(ValueError, match="'quantity' must be: 'power density', 'precision', 'level', or blank"):
        s.calculate_power_density_stl([0, 0, 0], quantity="flux")
    assert s.calculate_power_density_stl([0, 0, 0]) == []  # no facets: nothing to compute


def test_committed_meshes_are_the_generated_ones(tmp_path, monkeypatch):
    """The meshes under stl/ are what cases.write_stl_files() writes."""
    import cases
    monkeypatch.setattr(cases, "STL_DIR", str(tmp_path))
    cases.write_stl_files()
    for f in sorted(os.listdir(STL_DIR)):
        assert open(os.path.join(STL_DIR, f), "rb").read() == open(str(tmp_path / f), "rb").read()
