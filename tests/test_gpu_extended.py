"""Extended levels on the GPU: the levels above max_level, which the reference evaluates on the fly on
their own time grid (spacing T / (2^L - 1), src/TParticleTrajectoryInterpolatedPoints.cc:32-55), held
in device memory like the memory levels, up to level 27 (past the reference's memory limit of 26).

* the deep spectrum of cases.DEEP_LEVELS (memory levels 0..12, extended 13..27, 2^28 samples per
  entry) against the reference's own values (deep_levels.npz) at 1e-9 of the peak, in FP64; the
  mixed path against FP64 at 1e-4;
* the level cache switching between the memory grid and an extended split on one object (flux and
  power density), each result against its golden fixture;
* the mixed path on extended levels against FP64 at a fixed level, and the mixed power density;
* a level above 30 refused.
The golden extended-level cases (flux_und_extended, spec_und_extended, pd_und_extended) also run in
test_gpu_parity.py and through the reference's own seam in test_gpu_seam.py.
"""
import os

import numpy as np
import pytest

from cases import CASES, DEEP_LEVELS, E1_U, UND_SETUP, carried_levels, run_case

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-9
TOL_MIXED = 1e-4

pytestmark = pytest.mark.gpu


def _sr():
    from oscars_b200.sr import sr
    return sr(gpu=1)


def _flat(res):
    return (np.array([r[0] for r in res], dtype=np.float64), np.array([r[1] for r in res], dtype=np.float64))


def _peak_rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _with(calls, **extra):
    last, kw = calls[-1]
    return calls[:-1] + [(last, dict(kw, **extra))]


def test_deep_levels_fp64_match_the_reference():
    g = np.load(os.path.join(GOLDEN, "deep_levels.npz"))
    pos, val = _flat(run_case(_sr(), _with(DEEP_LEVELS, gpu=1)))
    assert np.array_equal(pos, g["pos"])
    assert _peak_rel(val, g["val"]) <= TOL, _peak_rel(val, g["val"])
    _, lev = _flat(run_case(_sr(), _with(DEEP_LEVELS, gpu=1, quantity="level")))
    assert np.all(lev == -1)  # precision 0: no entry converges, every one ran to level 27


def test_deep_levels_mixed_against_fp64():
    _, f = _flat(run_case(_sr(), _with(DEEP_LEVELS, gpu=1)))
    _, m = _flat(run_case(_sr(), _with(DEEP_LEVELS, gpu=1, compute="mixed")))
    assert _peak_rel(m, f) <= TOL_MIXED, _peak_rel(m, f)


@pytest.mark.parametrize("pair", [("flux_und_extended", "flux_und_41"), ("pd_und_extended", "pd_und_41")])
def test_level_cache_follows_the_level_grid(pair):
    """One object, one trajectory: extended split, memory grid, extended split again.  Each call must
    match its own fixture, so the cached levels of the other grid are never reused."""
    ext, mem = pair
    s = _sr()
    run_case(s, CASES[ext][:-1])
    for name in (ext, mem, ext):
        g = np.load(os.path.join(GOLDEN, name + ".npz"))
        last, kw = CASES[name][-1]
        pos, val = _flat(getattr(s, last)(**dict(kw, gpu=1)))
        assert np.array_equal(pos, g["pos"])
        assert _peak_rel(val, g["val"]) <= TOL, (name, _peak_rel(val, g["val"]))
        _, lev = _flat(getattr(s, last)(**dict(kw, gpu=1, quantity="level")))
        assert np.array_equal(carried_levels(lev), g["level"]), name


def test_mixed_extended_levels_against_fp64():
    calls = UND_SETUP + [("calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[21, 21], width=[0.01, 0.01],
                                                           translation=[0, 0, 30], precision=0, max_level=9,
                                                           max_level_extended=13, gpu=1))]
    _, f = _flat(run_case(_sr(), calls))
    _, m = _flat(run_case(_sr(), _with(calls, compute="mixed")))
    assert _peak_rel(m, f) <= TOL_MIXED, _peak_rel(m, f)


def test_mixed_power_density_on_extended_levels():
    """The mixed power density on an extended split (levels 10..12 on their own grid): the records and
    their beta-difference maxima follow the split, so values match FP64 and the stop levels agree."""
    name = "pd_und_extended"
    last, kw = CASES[name][-1]
    out = {}
    for compute in ("fp64", "mixed"):
        s = _sr()
        run_case(s, CASES[name][:-1])
        out[compute] = (_flat(getattr(s, last)(**dict(kw, gpu=1, compute=compute)))[1],
                        _flat(getattr(s, last)(**dict(kw, gpu=1, compute=compute, quantity="level")))[1])
    assert _peak_rel(out["mixed"][0], out["fp64"][0]) <= TOL_MIXED
    assert np.mean(out["mixed"][1] == out["fp64"][1]) >= 0.97


def test_level_above_30_refused():
    s = _sr()
    run_case(s, UND_SETUP)
    with pytest.raises(ValueError, match="max_level_extended above 30"):
        s.calculate_spectrum(obs=[0, 0, 30], energy_points_eV=[E1_U], precision=0, max_level=12, max_level_extended=31,
                             gpu=1)
