"""Parity cases shared by the golden-fixture generator and the tests.

Each case is a list of ``(method, kwargs)`` calls made on an object with the ``oscars.sr`` API
(the reference build, the CPU oracle, or ``oscars_b200.sr``); the last call's return value is the
result under test.  Workloads are seeded synthetic stand-ins for the reference's own examples:
a 41-period planar undulator (B0 = 0.5 T, 50 mm period) and a 30-period elliptical configuration
(By = 0.6 T cos, Bx = 0.4 T sin, 57 mm period), both with a 3 GeV electron beam.
"""
import math

E1_U = 458.9458        # first harmonic of the planar undulator [eV]
E1_EPU = 179.2558      # first harmonic of the elliptical configuration [eV]

UND = ("add_bfield_undulator", dict(bfield=[0, 0.5, 0], period=[0, 0, 0.05], nperiods=41, phase=-math.pi / 2))
EPU_Y = ("add_bfield_undulator", dict(bfield=[0, 0.6, 0], period=[0, 0, 0.057], nperiods=30, phase=-math.pi / 2))
EPU_X = ("add_bfield_undulator", dict(bfield=[0.4, 0, 0], period=[0, 0, 0.057], nperiods=30, phase=0))
BEAM = ("set_particle_beam", dict(type="electron", energy_GeV=3, x0=[0, 0, 0], d0=[0, 0, 1], current=0.5))
BEAM_GAUSS = ("set_particle_beam", dict(type="electron", energy_GeV=3, x0=[0, 0, 0], d0=[0, 0, 1], current=0.5,
                                        sigma_energy_GeV=0.003, beta=[1.5, 0.8], alpha=[0, 0],
                                        emittance=[0.9e-9, 8e-12]))


def traj(n=20001, a=-1.5, b=1.5):
    return [("set_ctstartstop", dict(start=a, stop=b)), ("set_npoints_trajectory", dict(n=n))]


UND_SETUP = [UND, BEAM] + traj()
EPU_SETUP = [EPU_Y, EPU_X, BEAM] + traj(16001)

CASES = {
    # trajectory of the planar undulator (checked through a subsample plus whole-array sums)
    "traj_und": UND_SETUP + [("calculate_trajectory", {})],
    # single-electron spectrum, 2000 energies over 100-3000 eV, adaptive levels
    "spec_und_2000": UND_SETUP + [("calculate_spectrum", dict(obs=[0, 0, 30], energy_range_eV=[100, 3000], npoints=2000))],
    # polarization projections off axis
    "spec_pol_lh": UND_SETUP + [("calculate_spectrum", dict(obs=[0.001, 0.0005, 30], energy_range_eV=[400, 500], npoints=40, polarization="lh"))],
    "spec_pol_lv": UND_SETUP + [("calculate_spectrum", dict(obs=[0.001, 0.0005, 30], energy_range_eV=[400, 500], npoints=40, polarization="lv"))],
    "spec_pol_cl": UND_SETUP + [("calculate_spectrum", dict(obs=[0.001, 0.0005, 30], energy_range_eV=[400, 500], npoints=40, polarization="circular-left"))],
    "spec_pol_cr": UND_SETUP + [("calculate_spectrum", dict(obs=[0.001, 0.0005, 30], energy_range_eV=[400, 500], npoints=40, polarization="cr"))],
    "spec_pol_angle": UND_SETUP + [("calculate_spectrum", dict(obs=[0.001, 0.0005, 30], energy_range_eV=[400, 500], npoints=40, angle=0.3))],
    # explicit energy list and a fixed level (precision 0 never converges: every point runs to 10)
    "spec_points_fixed": UND_SETUP + [("calculate_spectrum", dict(obs=[0, 0, 30], energy_points_eV=[200.0, 458.9458, 917.8916, 1376.8374], precision=0, max_level=10))],
    # flux on a 41x41 XY rectangle at E1
    "flux_und_41": UND_SETUP + [("calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[41, 41], width=[0.01, 0.01], translation=[0, 0, 30]))],
    "flux_und_fixed": UND_SETUP + [("calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[11, 11], width=[0.01, 0.01], translation=[0, 0, 30], precision=0, max_level=11))],
    "flux_und_lowlevel": UND_SETUP + [("calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[7, 7], width=[0.01, 0.01], translation=[0, 0, 30], max_level=6))],
    "flux_und_level": UND_SETUP + [("calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[21, 21], width=[0.01, 0.01], translation=[0, 0, 30], quantity="level"))],
    "flux_und_dim3_yz": UND_SETUP + [("calculate_flux_rectangle", dict(energy_eV=3 * E1_U, npoints=[9, 13], plane="XZ", width=[0.004, 0.006], rotations=[0, 0, 0.1], translation=[0, 0.0005, 30], dim=3, polarization="lv"))],
    # power density on the same rectangles
    "pd_und_41": UND_SETUP + [("calculate_power_density_rectangle", dict(npoints=[41, 41], width=[0.01, 0.01], translation=[0, 0, 30]))],
    "pd_und_directional": UND_SETUP + [("calculate_power_density_rectangle", dict(npoints=[11, 11], width=[0.02, 0.02], translation=[0, 0, 30], normal=1))],
    "pd_und_fixed": UND_SETUP + [("calculate_power_density_rectangle", dict(npoints=[9, 9], width=[0.01, 0.01], translation=[0, 0, 30], precision=0, max_level=10, quantity="precision"))],
    # elliptical configuration (two crossed undulators)
    "spec_epu_cl": EPU_SETUP + [("calculate_spectrum", dict(obs=[0, 0, 30], energy_range_eV=[100, 800], npoints=120, polarization="cl"))],
    "flux_epu_21": EPU_SETUP + [("calculate_flux_rectangle", dict(energy_eV=E1_EPU, npoints=[21, 21], width=[0.008, 0.008], translation=[0, 0, 30]))],
    # seeded Gaussian beam, several particles (checks the mt19937 / polar-normal sampling path)
    "flux_epu_multi": [EPU_Y, EPU_X, BEAM_GAUSS] + traj(16001) + [("set_seed", dict(seed=17)),
                       ("calculate_flux_rectangle", dict(energy_eV=E1_EPU, npoints=[7, 7], width=[0.008, 0.008], translation=[0, 0, 30], nparticles=4))],
    "pd_epu_multi": [EPU_Y, EPU_X, BEAM_GAUSS] + traj(16001) + [("set_seed", dict(seed=3)),
                     ("calculate_power_density_rectangle", dict(npoints=[7, 7], width=[0.01, 0.01], translation=[0, 0, 30], nparticles=3))],
    # tapered, time-dependent, displaced undulator; positron beam off axis; short trajectory
    "spec_taper_time": [("add_bfield_undulator", dict(bfield=[0, 0.7, 0], period=[0, 0, 0.03], nperiods=20, taper=0.02, frequency=1e6, frequency_phase=0.3, time_offset=1e-9, translation=[0, 0, 0.1])),
                        ("set_particle_beam", dict(type="positron", energy_GeV=2.5, x0=[0.0002, 0, -1], d0=[0.0001, 0, 1], current=0.4)),
                        ] + traj(8001, -1.0, 1.2) + [("calculate_spectrum", dict(obs=[0.002, 0.001, 25], energy_range_eV=[50, 1500], npoints=64))],
    "epu_field_spec": [("add_bfield_epu", dict(period=[0, 0, 0.04], nperiods=25, bfieldA=[0, 0.5, 0], bfieldB=[0.5, 0, 0], phase=1.2)), BEAM] + traj(12001, -1.0, 1.0)
                      + [("calculate_spectrum", dict(obs=[0, 0, 20], energy_range_eV=[200, 2000], npoints=60, polarization="cr"))],
}


def run_case(obj, calls):
    """Replay ``calls`` on ``obj`` and return the last call's result."""
    out = None
    for name, kw in calls:
        if name == "set_ctstartstop":
            out = obj.set_ctstartstop(kw["start"], kw["stop"])
        elif name == "set_npoints_trajectory":
            out = obj.set_npoints_trajectory(kw["n"])
        elif name == "set_seed":
            out = obj.set_seed(kw["seed"])
        else:
            out = getattr(obj, name)(**kw)
    return out
