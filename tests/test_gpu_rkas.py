"""Radiation on RKAS trajectories on the GPU.

The reference's RKAS trajectory holds its start time twice (the forward and the backward sweep both
store t0), so the spline through it has a 0 / 0 at that knot and every radiation result on it is NaN,
with no entry converging (golden case spec_rkas, replayed by test_gpu_parity.py).  The same holds
here for both arithmetic paths, and a mixed-precision multi-particle request with RKAS selected takes
the host integrator (not the device RK4 of the batched path), so it is NaN too.
"""
import numpy as np
import pytest

from cases import BEAM, BEAM_GAUSS, UND_SHORT, run_case, traj

pytestmark = pytest.mark.gpu


def _sr(beam, method):
    from oscars_b200.sr import sr
    s = sr(gpu=1)
    run_case(s, [UND_SHORT, beam] + traj(5001, -0.5, 0.5))
    s.set_trajectory_calculation(method)
    return s


@pytest.mark.parametrize("compute", ["fp64", "mixed"])
def test_spectrum_on_rkas_trajectory_is_nan_and_unconverged(compute):
    s = _sr(BEAM, "RKAS")
    r = s.calculate_spectrum(obs=[0, 0, 30], energy_range_eV=[400, 500], npoints=3, max_level=10, compute=compute)
    assert all(np.isnan(v) for _, v in r)
    assert np.array_equal(s.last_levels, [-1, -1, -1])


def test_mixed_beam_with_rkas_uses_the_host_integrator():
    kw = dict(energy_eV=458.9458, npoints=[3, 3], width=[0.002, 0.002], translation=[0, 0, 30], nparticles=2,
              max_level=10, compute="mixed", return_numpy=True)
    s = _sr(BEAM_GAUSS, "RKAS")
    s.set_seed(3)
    _, v = s.calculate_flux_rectangle(**kw)
    assert np.all(np.isnan(v))
    s = _sr(BEAM_GAUSS, "RK4")
    s.set_seed(3)
    _, v = s.calculate_flux_rectangle(**kw)
    assert np.all(np.isfinite(v)) and np.all(v > 0)
