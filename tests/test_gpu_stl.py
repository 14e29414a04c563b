"""Power density on STL facets on the GPU (k_stl_level) against the oracle.

The golden STL cases (a plate, the plate partly shadowed by a shield, a tilted mesh with stored
normals of length 2 and a zero normal, its level-capped variant, the precision of the shadowed case,
a 3-particle beam) run through test_gpu_parity.py like every golden case.  Here a seeded mesh with
many mutually shadowing facets (a plate behind randomly placed small triangles, some of them tilted
edge-on) is compared with the CPU oracle at the parity tolerance (1e-9 of the peak value) with
identical stop levels, for power density, precision and level.
"""
import numpy as np
import pytest

from cases import BEAM, UND_SHORT, traj

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _mesh(path, seed=11):
    """A 6 x 6 plate (72 facets) in z = 0 plus 24 small triangles between z = -18 and -12 m in front of
    it (2 to 8 m from the source once the mesh is translated to z = 20 m), normals as written by the generator."""
    from cases import _grid_plate, _write_stl
    rng = np.random.default_rng(seed)
    tris = _grid_plate(6, 6, -0.012, 0.012, -0.012, 0.012, (0.0, 0.0, 1.0))
    for _ in range(24):
        c = np.array([rng.uniform(-0.005, 0.005), rng.uniform(-0.005, 0.005), rng.uniform(-18, -12)])
        p = [tuple(c + rng.normal(0, 0.0015, 3) * np.array([1, 1, 0.0 if rng.uniform() < 0.7 else 200]))
             for _ in range(3)]
        tris.append(((0.0, 0.0, -1.0), p[0], p[1], p[2]))
    _write_stl(path, tris)


def _run(obj, path, **kw):
    for name, a in [UND_SHORT, BEAM] + traj(5001, -0.5, 0.5):
        if name == "set_ctstartstop":
            obj.set_ctstartstop(a["start"], a["stop"])
        elif name == "set_npoints_trajectory":
            obj.set_npoints_trajectory(a["n"])
        else:
            getattr(obj, name)(**a)
    obj.add_stl(path, translation=[0, 0, 20])
    res = obj.calculate_power_density_stl([0, 0, 0], max_level=11, **kw)
    return np.array([r[1] for r in res]), np.array([r[0] for r in res])


@pytest.mark.parametrize("quantity", ["power density", "precision", "level"])
def test_random_shadowing_mesh_matches_oracle(tmp_path, quantity):
    from oracle.oracle import OracleSR
    from oscars_b200.sr import sr
    path = str(tmp_path / "mesh.stl")
    _mesh(path)
    a, pa = _run(sr(gpu=1), path, quantity=quantity)
    o = OracleSR()
    b, pb = _run(o, path, quantity=quantity)
    assert np.array_equal(pa, pb)
    nan = np.isnan(b)
    assert np.array_equal(np.isnan(a), nan)
    if quantity == "level":
        assert np.array_equal(a, b)
    else:
        err = float(np.max(np.abs(a[~nan] - b[~nan])) / np.max(np.abs(b[~nan])))
        print("%s: peak-normalised error %.3e" % (quantity, err))
        assert err <= TOL


def test_shadowed_facets_lose_power(tmp_path):
    """Facets of the plate behind the small triangles receive less than without them."""
    from cases import _grid_plate, _write_stl
    from oscars_b200.sr import sr
    path = str(tmp_path / "mesh.stl")
    _mesh(path)
    plate = str(tmp_path / "plate.stl")
    _write_stl(plate, _grid_plate(6, 6, -0.012, 0.012, -0.012, 0.012, (0.0, 0.0, 1.0)))
    with_shields, _ = _run(sr(gpu=1), path)
    alone, _ = _run(sr(gpu=1), plate)
    ratio = with_shields[:72] / alone
    assert np.all(ratio <= 1 + 1e-12) and np.any(ratio < 0.999)
