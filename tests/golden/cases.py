"""Parity cases shared by the golden-fixture generator and the tests.

Each case is a list of ``(method, kwargs)`` calls made on an object with the ``oscars.sr`` API
(the reference build, the CPU oracle, or ``oscars_b200.sr``); the last call's return value is the
result under test.  Workloads are seeded synthetic stand-ins for the reference's own examples:
a 41-period planar undulator (B0 = 0.5 T, 50 mm period) and a 30-period elliptical configuration
(By = 0.6 T cos, Bx = 0.4 T sin, 57 mm period), both with a 3 GeV electron beam.
"""
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = os.path.join(HERE, "fields")

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
UND_SHORT = ("add_bfield_undulator", dict(bfield=[0, 0.5, 0], period=[0, 0, 0.05], nperiods=11, phase=-math.pi / 2))
UND_SHORT_SETUP = [UND_SHORT, BEAM] + traj(5001, -0.5, 0.5)
STL_PD = ("calculate_power_density_stl", dict(farfield_origin=[0, 0, 0], max_level=12))
# Levels past the reference's memory limit of 26: memory levels 0..12, extended levels 13..27 (2^28
# samples per entry; precision 0 never converges, so every entry runs to 27).  Its fixture
# (deep_levels.npz) takes the reference a few minutes and is not replayed on the oracle.
DEEP_LEVELS = UND_SHORT_SETUP + [("calculate_spectrum", dict(obs=[0, 0, 20], energy_points_eV=[458.9458, 1600.0], precision=0,
                                                             max_level=12, max_level_extended=27))]
EPU_SETUP = [EPU_Y, EPU_X, BEAM] + traj(16001)


# ---- grid fields and per-half-period undulator amplitudes --------------------------------------
def write_field_files():
    """Write the field files under fields/ (deterministic; the committed copies are what the tests
    and fixtures read).  und1d.txt: 'OSCARS1D Z By Bx' samples on an irregular z grid; grid3d.txt:
    an 'OSCARS' 3 x 3 x 241 grid; halfscale_41.txt: 82 half-period amplitude factors 1 + delta,
    delta ~ N(0, 0.005)."""
    import numpy as np
    os.makedirs(FIELDS, exist_ok=True)
    rng = np.random.default_rng(20240607)
    n = 1001
    z = -1.2 + 2.4 * np.arange(n) / (n - 1)
    z[1:-1] += rng.uniform(-0.3, 0.3, n - 2) * 2.4 / (n - 1)
    env = 0.5 * (np.tanh((z + 1.05) / 0.02) - np.tanh((z - 1.05) / 0.02))
    by = 0.5 * np.cos(2 * np.pi * z / 0.05) * env
    bx = 0.04 * np.sin(2 * np.pi * z / 0.05) * env
    with open(os.path.join(FIELDS, "und1d.txt"), "w") as f:
        f.write("# OSCARS1D Z By Bx test field (irregular z, tanh ends)\n")
        for i in rng.permutation(n):  # unsorted on purpose: the reader sorts
            f.write("%.15g, %.15g %.15g\n" % (z[i], by[i], bx[i]))
    nx, ny, nz = 3, 3, 241
    with open(os.path.join(FIELDS, "grid3d.txt"), "w") as f:
        f.write("# OSCARS 3D grid test field\n-0.002\n0.002\n%d\n-0.002\n0.002\n%d\n-0.96\n0.008\n%d\n" % (nx, ny, nz))
        for ix in range(nx):
            for iy in range(ny):
                for iz in range(nz):
                    zz = -0.96 + 0.008 * iz
                    env = 0.5 * (1 - math.cos(math.pi * iz / (nz - 1)))
                    f.write("%.10g %.10g %.10g\n" % (0.01 * (ix - 1) * env, 0.4 * math.cos(2 * math.pi * zz / 0.05)
                                                      * (1 + 0.05 * (iy - 1)) * env, 0.002 * (iz - 120) / 120))
    d = rng.normal(0.0, 0.005, 82)
    with open(os.path.join(FIELDS, "halfscale_41.txt"), "w") as f:
        for v in 1 + d:
            f.write("%.17g\n" % v)


def field_file(name):
    return os.path.join(FIELDS, name)


# ---- STL meshes (binary STL: 80-byte header, triangle count, 50-byte records N A B C attribute) ----
STL_DIR = os.path.join(HERE, "stl")


def stl_file(name):
    return os.path.join(STL_DIR, name)


def _write_stl(path, tris):
    """tris: list of (normal, A, B, C) 3-vectors, written as float32."""
    import struct
    with open(path, "wb") as f:
        f.write(b"parity mesh".ljust(80, b"\0"))
        f.write(struct.pack("<I", len(tris)))
        for n, a, b, c in tris:
            f.write(struct.pack("<12fH", *(list(n) + list(a) + list(b) + list(c)), 0))


def _grid_plate(nx, ny, x0, x1, y0, y1, normal, z_of=lambda x, y: 0.0, normal_of=None):
    tris = []
    for i in range(nx):
        for j in range(ny):
            xa, xb = x0 + (x1 - x0) * i / nx, x0 + (x1 - x0) * (i + 1) / nx
            ya, yb = y0 + (y1 - y0) * j / ny, y0 + (y1 - y0) * (j + 1) / ny
            p00, p10 = (xa, ya, z_of(xa, ya)), (xb, ya, z_of(xb, ya))
            p01, p11 = (xa, yb, z_of(xa, yb)), (xb, yb, z_of(xb, yb))
            k = 2 * (i * ny + j)
            tris.append((normal_of(k) if normal_of else normal, p00, p10, p11))
            tris.append((normal_of(k + 1) if normal_of else normal, p00, p11, p01))
    return tris


def write_stl_files():
    """Write the meshes under stl/ (deterministic; the committed copies are what the tests and the
    fixtures read).  plate.stl: 20 mm x 20 mm in the XY plane, 4 x 4 squares as 32 triangles, normal
    +z.  shield_mm.stl: a 6 mm x 3.3 mm rectangle in millimetres (2 triangles, normal -z), used with
    scale 0.001; at 10 m in front of the plate at 20 m its upper edge shadows the facets centred at
y = 6.67 mm from part of the 1 m trajectory only.  tilted.stl: 3 x 3 squares of 12 mm, tilted 30 degrees about x, stored normals of
    length 2 (as some exporters write them) and one zero normal."""
    os.makedirs(STL_DIR, exist_ok=True)
    _write_stl(stl_file("plate.stl"), _grid_plate(4, 4, -0.01, 0.01, -0.01, 0.01, (0.0, 0.0, 1.0)))
    _write_stl(stl_file("shield_mm.stl"), _grid_plate(1, 1, -3.0, 3.0, 0.0, 3.3, (0.0, 0.0, -1.0)))
    t = math.radians(30)
    nrm = (0.0, -2 * math.sin(t), 2 * math.cos(t))
    _write_stl(stl_file("tilted.stl"), _grid_plate(3, 3, -0.006, 0.006, -0.006, 0.006, nrm,
                                                   z_of=lambda x, y: y * math.tan(t),
                                                   normal_of=lambda k: (0.0, 0.0, 0.0) if k == 7 else nrm))


def halfscale_41():
    with open(field_file("halfscale_41.txt")) as f:
        return [float(v) for v in f.read().split()]


def halfscale_function(bfield, period, nperiods, phase, half_period_scale):
    """An undulator with per-half-period amplitude factors as a Python field function (for the
    reference's add_bfield_function): TField3D_IdealUndulator::GetF's operations in the same order
    (src/TField3D_IdealUndulator.cc:113-152), the full-strength region's half-period k scaled by
    half_period_scale[k].  No rotation, translation, taper or time dependence."""
    mag = math.sqrt(period[0] * period[0] + period[1] * period[1] + period[2] * period[2])
    pu = [period[0] / mag, period[1] / mag, period[2] / mag]
    lam = mag
    L = mag * (nperiods + 2)
    shift = phase * mag / (2.0 * math.pi)
    two_pi = 2.0 * math.pi
    hs = list(half_period_scale)
    amp = [float(v) for v in bfield]

    def field(x, y, z, t):
        d = (x - 0.0) * pu[0] + (y - 0.0) * pu[1] + (z - 0.0) * pu[2]
        tc = 1 + d * 0.0
        if d > L / 2. + shift or d < -L / 2. + shift:
            return [0.0, 0.0, 0.0]
        s = math.sin(two_pi * (d - shift) / lam)
        if d < -L / 2. + shift + lam or d > L / 2. + shift - lam:
            k = 0.25 if (d < -L / 2. + shift + lam / 2. or d > L / 2. + shift - lam / 2.) else 0.75
            return [a * k * s * tc for a in amp]
        i = int((d - (-L / 2. + shift + lam)) / (lam / 2.))
        i = 0 if i < 0 else (len(hs) - 1 if i >= len(hs) else i)
        return [a * s * tc * hs[i] for a in amp]
    return field


GRID1D = ("add_bfield_file", dict(ifile="und1d.txt", iformat="OSCARS1D Z By Bx", translation=[0, 0, 0.01],
                                  scale=[1, 1.02, 1]))
GRID3D = ("add_bfield_file", dict(ifile="grid3d.txt", iformat="OSCARS", rotations=[0, 0, 0.002],
                                  translation=[0.0001, 0, 0], scale=[1, 1, 1, 1, 1.1, 1]))
HALFSCALE = ("add_bfield_halfscale", dict(bfield=[0, 0.5, 0], period=[0, 0, 0.05], nperiods=41, phase=-math.pi / 2))

# A rectangle 8 mm x 6 mm near z = 30 m, slightly skewed and tilted, given by three corners.
X0X1X2 = [[-0.004, -0.003, 30.0], [0.004, -0.0025, 30.002], [-0.0038, 0.003, 29.998]]


def _arc_points(flip_every=0):
    """7 x 5 points on a cylinder of radius 30 m about the y axis (angles -0.25 .. 0.25 mrad, y within
    +-3 mm), normals pointing at the origin; with flip_every = k every k-th normal points away."""
    pts = []
    for i in range(7):
        phi = -2.5e-4 + 5e-4 * i / 6
        for j in range(5):
            y = -0.003 + 0.006 * j / 4
            n = [-math.sin(phi), 0.0, -math.cos(phi)]
            if flip_every and (5 * i + j) % flip_every == 0:
                n = [-v for v in n]
            pts.append([[30 * math.sin(phi), y, 30 * math.cos(phi)], n])
    return pts


ARC_POINTS = _arc_points()
ARC_POINTS_MIXED = _arc_points(3)

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
    # extended levels: above max_level the reference evaluates each level on the fly on its own time
    # grid (spacing T / (2^L - 1), not nested with the lower levels), up to max_level_extended
    "flux_und_extended": UND_SETUP + [("calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[7, 7], width=[0.01, 0.01], translation=[0, 0, 30], precision=0.001, max_level=9, max_level_extended=13))],
    "spec_und_extended": UND_SETUP + [("calculate_spectrum", dict(obs=[0.0005, 0, 30], energy_range_eV=[400, 500], npoints=20, precision=0.01, max_level=9, max_level_extended=13))],
    "pd_und_extended": UND_SETUP + [("calculate_power_density_rectangle", dict(npoints=[7, 7], width=[0.01, 0.01], translation=[0, 0, 30], precision=0.001, max_level=9, max_level_extended=12))],
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
    # grid fields from the reference's text formats (TField3D_Grid)
    "grid1d_traj": [GRID1D, BEAM] + traj(16001) + [("calculate_trajectory", {})],
    "grid1d_flux": [GRID1D, BEAM] + traj(16001) + [("calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[11, 11], width=[0.008, 0.008], translation=[0, 0, 30], precision=0, max_level=11))],
    "grid1d_spec": [GRID1D, BEAM] + traj(16001) + [("calculate_spectrum", dict(obs=[0.0005, 0, 30], energy_range_eV=[300, 600], npoints=40))],
    "grid3d_traj": [GRID3D, BEAM] + traj(12001, -1.2, 1.2) + [("calculate_trajectory", {})],
    "grid3d_flux": [GRID3D, BEAM] + traj(12001, -1.2, 1.2) + [("calculate_flux_rectangle", dict(energy_eV=516.0, npoints=[9, 9], width=[0.006, 0.006], translation=[0, 0, 30]))],
    "grid3d_pd": [GRID3D, BEAM] + traj(12001, -1.2, 1.2) + [("calculate_power_density_rectangle", dict(npoints=[9, 9], width=[0.01, 0.01], translation=[0, 0, 30]))],
    # 41-period undulator with 82 half-period amplitude factors (the field-tuning configuration)
    "halfscale_traj": [HALFSCALE, BEAM] + traj() + [("calculate_trajectory", {})],
    "halfscale_flux": [HALFSCALE, BEAM] + traj() + [("calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[11, 11], width=[0.002, 0.002], translation=[0, 0, 30], precision=0, max_level=11))],
    # rectangles given by three points (x0x1x2), rotated and translated, and arbitrary point surfaces
    "flux_x0x1x2": UND_SETUP + [("calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[9, 7], x0x1x2=X0X1X2, rotations=[0.001, -0.002, 0.0005], translation=[0.0005, -0.0002, 0.1], dim=3))],
    "flux_x0x1x2_dim2": UND_SETUP + [("calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[9, 7], x0x1x2=X0X1X2))],
    "pd_x0x1x2": UND_SETUP + [("calculate_power_density_rectangle", dict(npoints=[9, 9], x0x1x2=[[-0.005, -0.005, 30], [0.005, -0.005, 30], [-0.005, 0.005, 30]], normal=1))],
    "pd_points": UND_SETUP + [("calculate_power_density", dict(points=ARC_POINTS, rotations=[0.0, 0.001, 0.0], translation=[0.0, 0.0005, 0.0]))],
    "pd_points_directional": UND_SETUP + [("calculate_power_density", dict(points=ARC_POINTS_MIXED, normal=1))],
    "pd_points_inverted": UND_SETUP + [("calculate_power_density", dict(points=ARC_POINTS, normal=-1))],
    # several beams picked by weight for every particle, predefined beams, Twiss given with gamma and
    # a lattice reference point, and the ideal particle of a named beam
    "flux_two_beams": [EPU_Y, EPU_X,
                       ("add_particle_beam", dict(type="electron", name="a", energy_GeV=3, x0=[0, 0, 0], d0=[0, 0, 1],
                                                  current=0.5, sigma_energy_GeV=0.003, beta=[1.5, 0.8],
                                                  emittance=[0.9e-9, 8e-12], weight=1)),
                       ("add_particle_beam", dict(type="electron", name="b", energy_GeV=3.01, x0=[0.0002, 0, 0],
                                                  d0=[0.0001, 0, 1], current=0.5, sigma_energy_GeV=0.002,
                                                  beta=[3.0, 1.2], alpha=[0.5, -0.2], emittance=[2e-9, 2e-11],
                                                  weight=2))] + traj(16001) +
                      [("set_seed", dict(seed=5)),
                       ("calculate_flux_rectangle", dict(energy_eV=E1_EPU, npoints=[7, 7], width=[0.008, 0.008],
                                                         translation=[0, 0, 30], nparticles=6))],
    "traj_predefined_beam": [UND,
                             ("add_particle_beam", dict(beam="NSLSII-LONGSTRAIGHT", name="ls", x0=[0, 0, -0.2],
                                                        d0=[0.0002, 0, 1], energy_GeV=3.05))] +
                            traj(20001) + [("set_seed", dict(seed=9)), ("set_new_particle", dict(particle="")),
                                           ("calculate_trajectory", {})],
    "pd_predefined_and_twiss": [UND,
                                ("add_particle_beam", dict(beam="nsls2", name="n", weight=1)),
                                ("add_particle_beam", dict(type="positron", name="p", energy_GeV=3, current=0.4,
                                                           sigma_energy_GeV=0.001, beta=[2.0, 1.0], gamma=[0.6, 1.1],
                                                           emittance=[1e-9, 1e-11], lattice_reference=[0, 0, -1],
                                                           weight=3))] + traj() +
                               [("set_seed", dict(seed=13)),
                                ("calculate_power_density_rectangle", dict(npoints=[7, 7], width=[0.01, 0.01],
                                                                           translation=[0, 0, 30], nparticles=4))],
    "traj_named_beam_ideal": [UND,
                              ("add_particle_beam", dict(type="electron", name="first", energy_GeV=3, current=0.5)),
                              ("add_particle_beam", dict(type="electron", name="second", energy_GeV=2.5,
                                                         x0=[0.001, 0, 0], d0=[0, 0.0003, 1], current=0.3,
                                                         alpha=[0.4, 0.1], gamma=[1.0, 2.0], emittance=[1e-9, 1e-11],
                                                         distribution="kv"))] + traj(20001) +
                             [("set_new_particle", dict(beam="second", particle="ideal")), ("calculate_trajectory", {})],
    # adaptive Cash-Karp trajectories (RKAS): the 11-period undulator at the default precision, the
    # elliptical configuration at 1e-7; a spectrum on an RKAS trajectory (the reference's RKAS
    # trajectory holds the start time twice, so its spline and every radiation result are NaN)
    "traj_rkas": [UND_SHORT, BEAM] + traj(5001, -0.5, 0.5) + [("set_trajectory_calculation", dict(method="RKAS")),
                                                             ("calculate_trajectory", {})],
    "traj_rkas_epu": [EPU_Y, EPU_X, BEAM] + traj(16001, -1.0, 1.0) +
                     [("set_trajectory_calculation", dict(method="rkas", precision=1e-7)), ("calculate_trajectory", {})],
    "spec_rkas": [UND_SHORT, BEAM] + traj(5001, -0.5, 0.5) +
                 [("set_trajectory_calculation", dict(method="RKAS")),
                  ("calculate_spectrum", dict(obs=[0, 0, 30], energy_range_eV=[400, 500], npoints=3, max_level=10))],
    # power density on STL facets (11-period undulator, 1 m trajectory, levels up to 12): a plate in
    # the beam, the plate partly shadowed by a shield (millimetre file, scale 0.001), a tilted plate
    # with stored normals of length 2 and one zero normal (also capped at level 10, where facets that
    # do not stop report the previous facet's level), the precision of the shadowed case, and a
    # 3-particle beam on the plate
    "stl_plate": UND_SHORT_SETUP + [("add_stl", dict(ifile="plate.stl", translation=[0, 0, 20])), STL_PD],
    "stl_shadow": UND_SHORT_SETUP + [("add_stl", dict(ifile="plate.stl", translation=[0, 0, 20], name="plate")),
                                     ("add_stl", dict(ifile="shield_mm.stl", scale=0.001, translation=[0, 0, 10],
                                                      name="shield")), STL_PD],
    "stl_tilted": UND_SHORT_SETUP + [("add_stl", dict(ifile="tilted.stl", translation=[0, 0.002, 25],
                                                      rotations=[0.3, 0, 0])),
                                     ("calculate_power_density_stl", dict(farfield_origin=[0, 0, 0], max_level=12,
                                                                          precision=0.0005))],
    "stl_tilted_capped": UND_SHORT_SETUP + [("add_stl", dict(ifile="tilted.stl", translation=[0, 0.002, 25])),
                                            ("calculate_power_density_stl", dict(farfield_origin=[0, 0, 0], max_level=10,
                                                                                 precision=0.0005))],
    "stl_shadow_precision": UND_SHORT_SETUP + [("add_stl", dict(ifile="plate.stl", translation=[0, 0, 20])),
                                               ("add_stl", dict(ifile="shield_mm.stl", scale=0.001,
                                                                translation=[0, 0, 10])),
                                               ("calculate_power_density_stl", dict(farfield_origin=[0, 0, 0],
                                                                                    max_level=12,
                                                                                    quantity="precision"))],
    "stl_beam": [UND_SHORT, BEAM_GAUSS, ("set_seed", dict(seed=7))] + traj(5001, -0.5, 0.5) +
                [("add_stl", dict(ifile="plate.stl", translation=[0, 0, 20])),
                 ("calculate_power_density_stl", dict(farfield_origin=[0, 0, 0], max_level=12, nparticles=3))],
}


def carried_levels(levels):
    """Stop levels as the reference's single-thread point loop reports them with quantity='level':
    Result_Level is declared outside the loop (src/OSCARSSR.cc:4160), so an entry that did not
    converge (-1 here) repeats the level of the last entry before it that did (-1 before any).  The
    golden fixtures come from nthreads=1 runs; this library reports -1 for every such entry."""
    import numpy as np
    out = np.array(levels, dtype=np.float64)
    carry = -1.0
    for i in range(out.size):
        if out.flat[i] == -1:
            out.flat[i] = carry
        else:
            carry = out.flat[i]
    return out


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
        elif name == "add_stl":
            kw = dict(kw, ifile=stl_file(kw["ifile"]))
            out = obj.add_stl(**kw)
        elif name == "add_bfield_file":
            kw = dict(kw, ifile=field_file(kw["ifile"]))
            out = obj.add_bfield_file(**kw)
        elif name == "add_bfield_halfscale":
            hs = halfscale_41()
            if hasattr(obj, "add_bfield_function"):  # the reference: the same field as a Python function
                out = obj.add_bfield_function(halfscale_function(kw["bfield"], kw["period"], kw["nperiods"],
                                                                 kw["phase"], hs))
            else:
                out = obj.add_bfield_undulator(half_period_scale=hs, **kw)
        else:
            out = getattr(obj, name)(**kw)
    return out


# ---- differentiable tuning: the small configuration of the gradient fixtures -------------------
ADJ_LEVEL = 10
ADJ_FD_STEPS = (1e-6, 1e-3, 3e-3)   # central-difference steps of the gradient fixture


def richardson(fd_h, fd_rh, r):
    """Extrapolate central differences at steps h and r h to remove the O(h^2) term."""
    return (r * r * fd_h - fd_rh) / (r * r - 1)


def adjoint_config():
    """41-period undulator (B0 = 0.5 T, 50 mm) with 82 half-period factors; 5 x 5 observers over
    1 mm x 1 mm at z = 30 m; 8 energies over E1 +- 5 %; fixed level 10.  Loss = sum (F(s) - F(1))^2
    at s = the factors of halfscale_41.txt."""
    import numpy as np
    from oracle.oracle import rectangle
    obs, _, _ = rectangle("XY", 5, 5, 0.001, 0.001, [0.0, 0.0, 0.0], [0.0, 0.0, 30.0], 0)
    energies = np.linspace(0.95 * E1_U, 1.05 * E1_U, 8)
    return obs, energies, ADJ_LEVEL


# ---- output files: (setup, call, kwargs) whose ofile / bofile the reference wrote (files.npz) ------
FILE_CASES = {
    "flux_rect_dim2": (UND_SETUP, "calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[11, 9], width=[0.01, 0.008], translation=[0, 0, 30])),
    "flux_rect_dim3": (UND_SETUP, "calculate_flux_rectangle", dict(energy_eV=E1_U, npoints=[11, 9], width=[0.01, 0.008], translation=[0, 0, 30], dim=3)),
    "pd_rect": (UND_SETUP, "calculate_power_density_rectangle", dict(npoints=[9, 9], width=[0.01, 0.01], translation=[0, 0, 30])),
    "pd_points": (UND_SETUP, "calculate_power_density", dict(points=ARC_POINTS, normal=-1)),
    "spectrum": (UND_SETUP, "calculate_spectrum", dict(obs=[0, 0, 30], energy_range_eV=[100, 3000], npoints=60)),
    "traj_default": ([UND, BEAM] + traj(301), "calculate_trajectory", {}),
    "traj_format": ([UND, BEAM] + traj(301), "calculate_trajectory", dict(oformat="t x bx BPY")),
}
