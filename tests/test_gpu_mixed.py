"""Mixed-precision path (compute='mixed') against the plain FP64 GPU path.

Tolerance: peak-normalised relative error max_i |F_i - F64_i| / max_i |F64_i| <= 1e-4, at a fixed
level (precision=0, max_level=L) so that both paths integrate exactly the same samples.  The FP64
path itself matches the reference to <= 1e-9 (test_gpu_parity.py).  Each case is normalised by its
own peak, so small grids away from the axis test the path where the flux is weak, not only near the
on-axis maximum.  The cases span the region the mixed path accepts (mixed_geometry_ok): observer
angles up to min(1e-2, 20/gamma), correction phases (w/c) rho^2 / (2 Rz) up to 3e4 rad, harmonics
up to the 7th, the 2-3 keV end of the 100-3000 eV spectrum off axis; outside it the path refuses.
Power density (no phase: every direction is accepted) on the 201 x 201 grid, on points with normals
(directional and not), on a side wall at large angles, adaptively and for a seeded beam.
"""
import math

import numpy as np
import pytest

from cases import E1_EPU, E1_U, EPU_SETUP, UND_SETUP, run_case

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _sr():
    from oscars_b200.sr import sr
    return sr(gpu=1)


def _vals(res):
    return np.array([r[1] for r in res], dtype=np.float64)


def _pair(setup, call, kw):
    out = []
    for compute in ("fp64", "mixed"):
        s = _sr()
        run_case(s, setup)
        out.append(_vals(getattr(s, call)(**dict(kw, compute=compute))))
    return out


def _err(a, ref):
    return float(np.max(np.abs(a - ref)) / np.max(np.abs(ref)))


def test_flux_201x201_fixed_level_12():
    f64, mx = _pair(UND_SETUP, "calculate_flux_rectangle",
                    dict(energy_eV=E1_U, npoints=[201, 201], width=[0.01, 0.01], translation=[0, 0, 30],
                         precision=0, max_level=12))
    e = _err(mx, f64)
    print("flux 201x201 L=12 mixed vs fp64: %.3e" % e)
    assert e <= TOL


def test_spectrum_2000_fixed_level_13():
    f64, mx = _pair(UND_SETUP, "calculate_spectrum",
                    dict(obs=[0, 0, 30], energy_range_eV=[100, 3000], npoints=2000, precision=0, max_level=13))
    e = _err(mx, f64)
    print("spectrum 2000 L=13 mixed vs fp64: %.3e" % e)
    assert e <= TOL


@pytest.mark.parametrize("pol", ["lh", "lv", "cl", "cr"])
def test_polarized_flux_epu(pol):
    f64, mx = _pair(EPU_SETUP, "calculate_flux_rectangle",
                    dict(energy_eV=E1_EPU, npoints=[41, 41], width=[0.008, 0.008], translation=[0, 0, 30],
                         precision=0, max_level=11, polarization=pol))
    assert _err(mx, f64) <= TOL


def test_off_axis_beam_frame():
    """Tilted, displaced beam: the mixed path works in the particle's own frame."""
    setup = [("add_bfield_undulator", dict(bfield=[0, 0.5, 0], period=[0, 0.0, 0.05], nperiods=21, phase=-math.pi / 2,
                                           translation=[0.001, 0, 0])),
             ("set_particle_beam", dict(type="electron", energy_GeV=3, x0=[0.001, -0.0005, -1.2], d0=[0.0003, 0.0001, 1],
                                        current=0.5)),
             ("set_ctstartstop", dict(start=-0.2, stop=2.4)), ("set_npoints_trajectory", dict(n=12001))]
    f64, mx = _pair(setup, "calculate_flux_rectangle",
                    dict(energy_eV=2 * E1_U, npoints=[31, 31], width=[0.006, 0.006], translation=[0.01, 0.003, 30],
                         precision=0, max_level=11))
    assert _err(mx, f64) <= TOL


def test_adaptive_mode_close_to_fp64():
    """Adaptive stop levels may differ where a level's relative change sits at the threshold."""
    out, lev = [], []
    for compute in ("fp64", "mixed"):
        s = _sr()
        run_case(s, UND_SETUP)
        out.append(_vals(s.calculate_flux_rectangle(energy_eV=E1_U, npoints=[101, 101], width=[0.01, 0.01],
                                                    translation=[0, 0, 30], compute=compute)))
        lev.append(s.last_levels.copy())
    frac = float(np.mean(lev[0] != lev[1]))
    print("adaptive: %.4f of entries stop at another level; error %.3e" % (frac, _err(out[1], out[0])))
    # flips happen at low-flux entries where |E| << sum |terms|, so the peak-normalised error stays small
    assert frac <= 0.03
    assert _err(out[1], out[0]) <= 1e-4


HBAR_C_EVM = 1.973269804e-7  # hbar c [eV m]: w / c = E / (hbar c)
GAMMA_3GEV = 3.0 / 0.51099895e-3


def _setup_energy(energy_GeV):
    und, beam = UND_SETUP[0], dict(UND_SETUP[1][1], energy_GeV=energy_GeV)
    return [und, ("set_particle_beam", beam)] + UND_SETUP[2:]


@pytest.mark.parametrize("theta_gamma", [2, 5])
def test_small_off_axis_grids_at_e1(theta_gamma):
    """3 x 3 grids 0.2 mm wide at 20 m, centred theta_gamma / gamma off axis: the flux there is a
    fraction of the on-axis peak, and the phase correction is 3e3 .. 2e4 rad."""
    x = theta_gamma / GAMMA_3GEV * 20
    f64, mx = _pair(UND_SETUP, "calculate_flux_rectangle",
                    dict(energy_eV=E1_U, npoints=[3, 3], width=[0.0002, 0.0002], translation=[x, 0, 20],
                         precision=0, max_level=13))
    e = _err(mx, f64)
    print("off-axis grid theta*gamma=%d: mixed vs fp64 %.3e" % (theta_gamma, e))
    assert e <= TOL


@pytest.mark.parametrize("harmonic", [3, 5, 7])
@pytest.mark.parametrize("corr_phase", [1e4, 2.7e4])
def test_harmonics_up_to_the_correction_phase_limit(harmonic, corr_phase):
    """15 x 15 grid at 20 m whose corner reaches the given correction phase at the h-th harmonic
    (the guard accepts up to 3e4 rad; the trajectory ends 1.5 m downstream of the origin)."""
    E = harmonic * E1_U
    rho = math.sqrt(corr_phase * 2 * (20 - 1.5) / (E / HBAR_C_EVM))
    w = 2 * rho / math.sqrt(2)
    f64, mx = _pair(UND_SETUP, "calculate_flux_rectangle",
                    dict(energy_eV=E, npoints=[15, 15], width=[w, w], translation=[0, 0, 20], precision=0,
                         max_level=13))
    e = _err(mx, f64)
    print("harmonic %d, corner correction phase %.1e rad (grid %.1f mm): mixed vs fp64 %.3e"
          % (harmonic, corr_phase, w * 1e3, e))
    assert e <= TOL


@pytest.mark.parametrize("obs", [[0.006, 0.002, 30], [0.0095, 0.0, 30]])
def test_off_axis_spectrum_2_to_3_keV(obs):
    """The high-energy end of the 100-3000 eV spectrum at observers 6-10 mm off axis at 30 m
    (correction phases 1e4 and 2.4e4 rad at 3 keV)."""
    f64, mx = _pair(UND_SETUP, "calculate_spectrum",
                    dict(obs=obs, energy_range_eV=[2000, 3000], npoints=201, precision=0, max_level=13))
    e = _err(mx, f64)
    print("spectrum 2-3 keV at %s: mixed vs fp64 %.3e" % (obs, e))
    assert e <= TOL


@pytest.mark.parametrize("angle,energy_eV", [(0.5e-2, 12.8), (0.9e-2, 5.0)])
def test_wide_angles_at_low_beam_energy(angle, energy_eV):
    """A 0.5 GeV beam (gamma 978): the angle limit is 1e-2 itself.  3 x 3 grids 4 mm wide at 20 m,
    centred at rho / Rz = 0.5e-2 and 0.9e-2, at energies that keep the correction phase near 2e4 rad."""
    f64, mx = _pair(_setup_energy(0.5), "calculate_flux_rectangle",
                    dict(energy_eV=energy_eV, npoints=[3, 3], width=[0.004, 0.004], translation=[angle * 20, 0, 20],
                         precision=0, max_level=12))
    e = _err(mx, f64)
    print("0.5 GeV, rho/Rz = %.1e at %.1f eV: mixed vs fp64 %.3e" % (angle, energy_eV, e))
    assert e <= TOL


def test_angles_beyond_the_limit_are_refused():
    """30 / gamma at 3 GeV (above 20 / gamma) and 1.2e-2 at 0.5 GeV (above 1e-2) are refused."""
    cases = [(UND_SETUP, 30 / GAMMA_3GEV * 20, 10.0), (_setup_energy(0.5), 0.012 * 20, 2.0)]
    for setup, x, E in cases:
        s = _sr()
        run_case(s, setup)
        with pytest.raises(ValueError, match="compute='mixed' needs observers near the beam axis"):
            s.calculate_flux_rectangle(energy_eV=E, npoints=[1, 1], width=[1e-4, 1e-4], translation=[x, 0, 20],
                                       compute="mixed")


def test_far_off_axis_observer_is_rejected():
    s = _sr()
    run_case(s, UND_SETUP)
    with pytest.raises(ValueError, match="compute='mixed' needs observers near the beam axis"):
        s.calculate_spectrum(obs=[3, 0, 30], energy_range_eV=[100, 200], npoints=3, compute="mixed")


def test_refusal_reported_once_through_every_entry_point():
    """The device entry queues its work and returns: a refused observer is reported by the next
    osc_last_stats, once (the error word is cleared), and the next valid request runs; the host
    entry with page-locked or pageable buffers reports it from the call itself."""
    import ctypes
    import torch
    from oscars_b200 import _lib
    from oscars_b200._lib import RadOpts
    s = _sr()
    run_case(s, UND_SETUP)
    o = RadOpts(precision=0.01, max_level=-2, max_level_extended=0, nparticles=0, quantity=0, precision_mode=1)
    o.horizontal[:] = [1, 0, 0]
    o.propagation[:] = [0, 0, 1]
    bad = np.array([[3.0, 0.0, 30.0], [0.0, 0.0, 30.0]])
    good = np.array([[0.0, 0.0, 30.0], [1e-4, 0.0, 30.0]])
    d_out = torch.zeros(2, dtype=torch.float64, device="cuda")
    d_lvl = torch.zeros(2, dtype=torch.int32, device="cuda")
    sm = ctypes.c_longlong()

    def dev_call(obs):
        d_obs = torch.tensor(obs, device="cuda")
        s._ctx.call("osc_flux_device", ctypes.c_void_p(d_obs.data_ptr()), 2, E1_U, ctypes.byref(o),
                    ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_lvl.data_ptr()), None)
        torch.cuda.synchronize()

    dev_call(bad)
    with pytest.raises(ValueError, match="compute='mixed' needs observers near the beam axis"):
        s._ctx.call("osc_last_stats", ctypes.byref(sm), None)
    s._ctx.call("osc_last_stats", ctypes.byref(sm), None)  # reported once
    dev_call(good)
    s._ctx.call("osc_last_stats", ctypes.byref(sm), None)
    assert sm.value > 0 and np.all(d_out.cpu().numpy() > 0)
    for pinned in (True, False):
        obs = torch.from_numpy(bad.copy())
        out = torch.zeros(2, dtype=torch.float64)
        if pinned:
            obs, out = obs.pin_memory(), out.pin_memory()
        with pytest.raises(ValueError, match="compute='mixed' needs observers near the beam axis"):
            s._ctx.call("osc_flux", _lib.dptr(obs.numpy()), 2, E1_U, ctypes.byref(o), _lib.dptr(out.numpy()), None,
                        None)
    ok = np.zeros(2)
    s._ctx.call("osc_flux", _lib.dptr(np.ascontiguousarray(good)), 2, E1_U, ctypes.byref(o), _lib.dptr(ok), None, None)
    assert np.allclose(ok, d_out.cpu().numpy(), rtol=0, atol=0)


def _variants(kind):
    import ctypes
    s = _sr()
    v, n = ctypes.c_int(), ctypes.c_int()
    s._ctx.call("osc_get_variant", kind, ctypes.byref(v), ctypes.byref(n))
    return n.value


@pytest.mark.parametrize("variant", range(4))
def test_every_mixed_variant_matches_fp64(variant):
    """Each compiled mixed kernel (pair records, 1/2/4 sample groups per CTA) on a flux grid with many
    spans per entry (level 13, fixed) and on a spectrum past the prefilled levels."""
    if variant >= _variants(2):
        pytest.skip("variant not compiled")
    flux = dict(energy_eV=E1_U, npoints=[41, 41], width=[0.008, 0.008], translation=[0, 0, 30], precision=0,
                max_level=13)
    spec = dict(obs=[0.0005, 0.0002, 30], energy_range_eV=[100, 3000], npoints=300, precision=0, max_level=16)
    for call, kw in (("calculate_flux_rectangle", flux), ("calculate_spectrum", spec)):
        out = {}
        for compute in ("fp64", "mixed"):
            s = _sr()
            if compute == "mixed":
                s._ctx.call("osc_set_variant", 2, variant)
            run_case(s, UND_SETUP)
            out[compute] = _vals(getattr(s, call)(**dict(kw, compute=compute)))
        e = _err(out["mixed"], out["fp64"])
        print("variant %d %s: mixed vs fp64 %.3e" % (variant, call, e))
        assert e <= TOL


# ---- power density ------------------------------------------------------------------------------
def test_power_density_201x201_fixed_level_12():
    f64, mx = _pair(UND_SETUP, "calculate_power_density_rectangle",
                    dict(npoints=[201, 201], width=[0.01, 0.01], translation=[0, 0, 30], precision=0, max_level=12))
    e = _err(mx, f64)
    print("power density 201x201 L=12 mixed vs fp64: %.3e" % e)
    assert e <= TOL


def test_power_density_adaptive_levels():
    kw = dict(npoints=[41, 41], width=[0.02, 0.02], translation=[0, 0, 30])
    f64, mx = _pair(UND_SETUP, "calculate_power_density_rectangle", kw)
    assert _err(mx, f64) <= TOL
    l64, lmx = _pair(UND_SETUP, "calculate_power_density_rectangle", dict(kw, quantity="level"))
    same = float(np.mean(l64 == lmx))
    print("power density adaptive: %.3e, levels equal at %.4f of the entries" % (_err(mx, f64), same))
    assert same >= 0.97


@pytest.mark.parametrize("normal", [1, -1, 0])
def test_power_density_points_with_normals(normal):
    """Points on a 30 m arc with tilted normals (directional for normal = +-1), and the same points
    with normals that half of the samples see from behind."""
    from cases import ARC_POINTS, ARC_POINTS_MIXED
    for pts in (ARC_POINTS, ARC_POINTS_MIXED):
        f64, mx = _pair(UND_SETUP, "calculate_power_density", dict(points=pts, normal=normal, precision=0, max_level=11))
        if not np.any(f64):  # every point sees the trajectory from behind its surface
            assert not np.any(mx)
            continue
        e = _err(mx, f64)
        print("power density points normal=%d mixed vs fp64: %.3e" % (normal, e))
        assert e <= TOL


def test_power_density_side_wall_at_large_angles():
    """A wall 0.1 m beside the beam from z = -1 m to 3 m (angles up to 90 degrees and beyond) whose
    normal points along the direction of view: no near-axis observer, each case normalised by its own
    peak."""
    zs = np.linspace(-1.0, 3.0, 41)
    ys = np.linspace(-0.05, 0.05, 5)
    pts = [[[0.1, float(y), float(z)], [1.0, 0.0, 0.0]] for z in zs for y in ys]  # N1 . normal > 0: seen
    for normal in (0, 1):
        f64, mx = _pair(UND_SETUP, "calculate_power_density", dict(points=pts, normal=normal, precision=0, max_level=12))
        e = _err(mx, f64)
        print("side wall normal=%d mixed vs fp64: %.3e" % (normal, e))
        assert e <= TOL
        # far from the axis the values are tiny but must keep their relative accuracy too
        far = np.abs(f64) > 0
        rel = np.max(np.abs(mx[far] - f64[far]) / np.abs(f64[far]))
        assert rel <= 1e-3, rel


def test_power_density_beam_mixed_matches_fp64():
    from cases import BEAM_GAUSS, EPU_X, EPU_Y, traj
    setup = [EPU_Y, EPU_X, BEAM_GAUSS] + traj(16001) + [("set_seed", dict(seed=11))]
    f64, mx = _pair(setup, "calculate_power_density_rectangle",
                    dict(npoints=[21, 21], width=[0.01, 0.01], translation=[0, 0, 30], nparticles=6, precision=0,
                         max_level=11))
    e = _err(mx, f64)
    print("power density beam (6 particles) mixed vs fp64: %.3e" % e)
    assert e <= TOL
