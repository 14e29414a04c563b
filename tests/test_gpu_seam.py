"""The reference's own oscars.sr with gpu=1, computing on this library.

OSCARS sends gpu=1 requests through the seam of include/OSCARSSR_Cuda.h (OSCARSSR::Calculate*GPU,
src/OSCARSSR.cc:2429, 3125, 4428).  oscars_b200/seam builds the reference's `sr` extension from its
own sources with that seam served by liboscars_b200 (the reference's host code draws particles and
integrates trajectories; this library's FP64 kernels integrate the radiation).  Every golden
radiation case is replayed through that build with gpu=1 and compared with the golden values, which
the reference's CPU path produced: peak-normalised error <= 1e-9 and identical stop-level maps.  The
build must have been made beforehand (make -C oscars_b200/seam REF=<OSCARS sources>); the GPU box
only receives the built files.  The reference runs in a child process, because the CPU reference
build the other tests load is also a package named `oscars`.

Excluded: the directional power-density cases (normal != 0) -- the seam's power-density function
carries no `Directional` argument (include/OSCARSSR_Cuda.h:56-63), so a directional request is
answered non-directionally by the reference's GPU path and by this seam alike.  The STL power-density
cases -- the reference has no GPU path for them: its Python entry parses `gpu` with the format letter
'O' into an int (src/OSCARSSR_Python.cc:7027), so gpu=1 is refused as "'gpu' must be 0 or 1", and
OSCARSSR::CalculatePowerDensitySTL throws on its GPU branch (src/OSCARSSR.cc:3209).  The
extended-level cases (max_level_extended above max_level) -- the reference hands its GPU functions
one level, max(max_level_extended, max_level) (src/OSCARSSR.cc:4424-4440, 2425-2436), so its GPU
path has no extended levels: the seam answers on the memory grid up to that level, as the
reference's GPU path does, which is not what its CPU path (the fixture) computes.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from cases import CASES, carried_levels

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "oscars_b200", "seam", "_build")
GOLDEN = os.path.join(ROOT, "tests", "golden")
TOL = 1e-9
def _extended(kw):
    """Whether a call reaches extended levels (src/OSCARSSR.cc:4108-4109)."""
    ml = kw.get("max_level", -2)
    return kw.get("max_level_extended", 0) > (ml if -1 <= ml <= 26 else 26)


NAMES = sorted(k for k, v in CASES.items() if v[-1][0] not in ("calculate_trajectory", "calculate_power_density_stl")
               and not (v[-1][0].startswith("calculate_power_density") and v[-1][1].get("normal", 0) != 0)
               and not _extended(v[-1][1]))


@pytest.fixture(scope="module")
def seam_results(tmp_path_factory):
    if not os.path.isdir(os.path.join(BUILD, "oscars")):
        pytest.fail("the seam build is missing: make -C oscars_b200/seam REF=<OSCARS sources>")
    out = str(tmp_path_factory.mktemp("seam") / "seam.npz")
    env = dict(os.environ, PYTHONPATH="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "seam_worker.py"), BUILD, out] + NAMES,
                       capture_output=True, text=True, env=env, timeout=1200)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    return dict(np.load(out))


def test_seam_build_is_the_one_loaded_and_sees_the_gpu(seam_results):
    assert str(seam_results["module"]).startswith(BUILD)
    assert int(seam_results["ngpu"]) >= 1  # CheckGPU() through the seam: gpu=1 requests go to the GPU


@pytest.mark.parametrize("name", NAMES)
def test_golden_case_through_reference_gpu_seam(seam_results, name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    pos, val = seam_results[name + "/pos"], seam_results[name + "/val"]
    assert np.array_equal(pos.reshape(g["pos"].shape), g["pos"])
    if CASES[name][-1][1].get("quantity") == "level":
        assert np.array_equal(carried_levels(val), g["val"])
    else:
        # NaN where the golden values are NaN (a trajectory that repeats its start time, as the
        # reference's adaptive Cash-Karp trajectory does), the finite values within TOL
        nan = np.isnan(g["val"])
        assert np.array_equal(np.isnan(val), nan), "%s: NaN pattern differs" % name
        if not nan.all():
            ref, got = g["val"][~nan], val[~nan]
            err = float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300))
            assert err <= TOL, "%s: peak-normalised error %.3e" % (name, err)
    if "level" in g.files and name + "/level" in seam_results:
        lev = carried_levels(seam_results[name + "/level"])
        assert np.array_equal(lev, g["level"]), "stop levels differ at %d entries" % int(np.sum(lev != g["level"]))
