"""``oscars_b200.sr`` -- drop-in for the ``oscars.sr`` calls of the radiation hot path.

Same method names, keyword names, defaults, return shapes and ValueError messages as the reference
CPython extension (src/OSCARSSR_Python.cc); the arithmetic runs in liboscars_b200.so: the FP64 RK4
trajectory and spline on the host (bit-identical to the reference), the level-ladder radiation sums
on the B200.  Argument preprocessing that the reference binding does in its own layer (rotations of
field vectors, the default horizontal direction, polarization strings, energy grids) is restated
here with the binding's file:line.

Extensions, all keyword-only and off by default:
  ``compute='fp64'|'mixed'``   arithmetic of the radiation sums (see include/oscars_b200.h)
  ``return_numpy=True``        return (positions, values) arrays instead of nested lists
  ``shard=(rank, count)``      this process's share of a multi-particle request (particles with
                               index % count == rank, weight 1/N): the shares add up to the whole
  ``half_period_scale=...``    (add_bfield_undulator) per-half-period amplitude factors
  ``add_bfield_grid(...)``     a grid field from memory (the file readers are add_bfield_file)
"""
from __future__ import annotations

import ctypes
import math
import sys

import numpy as np

from . import _lib, fileio
from .stl import StlContainer
from ._lib import BeamDesc, Context, FieldDesc, RadOpts, dptr, i32ptr

_ANGLE_UNSET = 112188979912321.0  # binding sentinel for "angle not given" (:5662)
_PREDEFINED_BEAMS = {"NSLSII": 1, "NSLS2": 1, "NSLS-II": 1,
                     "NSLSII-LONGSTRAIGHT": 2, "NSLS2-LONGSTRAIGHT": 2, "NSLS-II-LONGSTRAIGHT": 2,
                     "NSLSII-SHORTSTRAIGHT": 3, "NSLS2-SHORTSTRAIGHT": 3, "NSLS-II-SHORTSTRAIGHT": 3}
_PARTICLES = {"electron": 0, "anti-positron": 0, "positron": 1, "anti-electron": 1, "muon": 2,
              "anti-muon": 3, "proton": 4, "anti-proton": 5, "pi+": 6, "pi-": 7, "custom": 8}
_NOT_CONVERGED = "Not all points converged to desired precision.  Can try increasing 'max_level_extended'\n"


def _vec3(v, name):
    try:
        v = [float(x) for x in v]
    except TypeError:
        raise ValueError("Incorrect format in '%s'" % name)
    if len(v) != 3:
        raise ValueError("Incorrect format in '%s'" % name)
    return v


def _vec2(v, name):
    v = [float(x) for x in v]
    if len(v) != 2:
        raise ValueError("Incorrect format in '%s'" % name)
    return v


def _rotate_xyz(v, r):
    """TVector3D::RotateSelfXYZ (src/TVector3D.cc): about X, then Y, then Z."""
    x, y, z = v
    s, c = math.sin(r[0]), math.cos(r[0])
    y, z = c * y - s * z, s * y + c * z
    s, c = math.sin(r[1]), math.cos(r[1])
    z, x = c * z - s * x, s * z + c * x
    s, c = math.sin(r[2]), math.cos(r[2])
    x, y = c * x - s * y, s * x + c * y
    return [x, y, z]


def _polarization(polarization, angle):
    """Binding defaults (src/OSCARSSR_Python.cc:5889-5899) and the string match of
    src/OSCARSSR.cc:4129-4150."""
    if polarization == "all" and angle != _ANGLE_UNSET:
        raise ValueError("cannot specify 'all' and 'angle'.  This is to save you")
    pol = polarization if len(polarization) else ("linear" if angle != _ANGLE_UNSET else "all")
    p = pol.lower().replace(" ", "-")
    if "all" in p:
        return 0
    if "linear-horizontal" in p or "lh" in p:
        return 1
    if "linear-vertical" in p or "lv" in p:
        return 2
    if p == "linear":
        return 3
    if "circular-left" in p or "cl" in p:
        return 4
    if "circular-right" in p or "cr" in p:
        return 5
    raise ValueError("Polarization requested not recognized")


def _quantity(q, pd=False):
    Q = q.upper()
    if (pd and Q in ("POWER DENSITY", "POWERDENSITY")) or (not pd and Q == "FLUX"):
        return 0
    if Q == "PRECISION":
        return 1
    if Q == "LEVEL":
        return 2
    raise ValueError("'quantity' must be: '%s', 'precision', 'level', or blank" % ("power density" if pd else "flux"))


def _compute_mode(compute):
    if compute in ("fp64", "plain", 0):
        return 0
    if compute in ("mixed", 1):
        return 1
    raise ValueError("'compute' must be 'fp64' or 'mixed'")


class sr:
    """GPU implementation of the ``oscars.sr.sr`` radiation calls."""

    def __init__(self, nthreads=0, gpu=0, device=None):
        if gpu not in (0, 1):
            raise ValueError("global gpu settign must be 0 or 1")
        ndev = _lib.device_count()
        self._dev = device if device is not None else (0 if ndev > 0 else -1)
        self._ctx = Context(self._dev)
        self._gpu_global = 1
        self._nthreads_global = nthreads if nthreads > 0 else 2
        self._nbeams = 0
        self._stl = StlContainer()

    # ---- global settings ------------------------------------------------------------------------
    def set_gpu_global(self, gpu):
        if gpu not in (0, 1):
            raise ValueError("global gpu settign must be 0 or 1")
        self._gpu_global = 1  # every radiation call of this build runs on the GPU

    def check_gpu(self):
        return _lib.device_count()

    def set_nthreads_global(self, n):
        self._nthreads_global = int(n)

    def set_seed(self, seed):
        self._ctx.call("osc_set_seed", int(float(seed)))

    def version(self):
        return _lib.lib().osc_version().decode()

    # ---- fields (src/OSCARSSR_Python.cc:1309-1420, 1479-1630) ------------------------------------
    def clear_bfields(self):
        self._ctx.call("osc_clear_fields")

    def add_bfield_undulator(self, bfield, period, nperiods, phase=0, rotations=[], translation=[], taper=0,
                             frequency=0, frequency_phase=0, time_offset=0, name="", *, half_period_scale=None):
        """``half_period_scale`` (this build's extension): 2 * nperiods amplitude factors, one per
        half-period of the full-strength region between the end poles."""
        f = _vec3(bfield, "bfield")
        p = _vec3(period, "period")
        r = _vec3(rotations, "rotations") if len(rotations) else [0.0, 0.0, 0.0]
        t = _vec3(translation, "translation") if len(translation) else [0.0, 0.0, 0.0]
        if len(name) > 0 and name[0] == "_":
            raise ValueError("'name' cannot begin with '_'.  This is reserved for internal use.  Please pick a different name")
        d = FieldDesc(kind=0, nperiods=int(nperiods), phase=float(phase), taper=float(taper),
                      frequency=float(frequency), frequency_phase=float(frequency_phase),
                      time_offset=float(time_offset))
        d.bfield[:] = _rotate_xyz(f, r)
        d.period[:] = _rotate_xyz(p, r)
        d.center[:] = t
        if half_period_scale is not None:
            hs = np.ascontiguousarray(np.asarray(half_period_scale, dtype=np.float64).ravel())
            d.half_period_scale = dptr(hs)
            d.n_half_periods = int(hs.size)
        self._ctx.call("osc_add_field", ctypes.byref(d))

    def add_bfield_file(self, ifile="", bifile="", iformat="", rotations=[], translation=[], scale=[], frequency=0,
                        frequency_phase=0, time_offset=0, name=""):
        """Grid field from a file (src/OSCARSSR_Python.cc:526-625); formats 'OSCARS' and
        'OSCARS1D <columns>' (e.g. 'OSCARS1D Z Bx By Bz')."""
        if len(ifile) and len(bifile):
            raise ValueError("cannot specify both 'ifile' and 'bifile'")
        if len(ifile) and not len(iformat):
            raise ValueError("'iformat' is blank")
        try:
            r = _vec3(rotations, "rotations") if len(rotations) else [0.0, 0.0, 0.0]
        except ValueError:
            raise ValueError("Incorrect format in 'rotations'")
        try:
            t = _vec3(translation, "translation") if len(translation) else [0.0, 0.0, 0.0]
        except ValueError:
            raise ValueError("Incorrect format in 'translation'")
        if len(name) > 0 and name[0] == "_":
            raise ValueError("'name' cannot begin with '_'.  This is reserved for internal use.  Please pick a different name")
        path, fmt = (bifile, "BINARY") if len(bifile) else (ifile, iformat)
        sc = np.ascontiguousarray(np.asarray(list(scale), dtype=np.float64))
        R, T = np.array(r), np.array(t)
        try:
            self._ctx.call("osc_add_field_file", path.encode(), fmt.encode(), dptr(R), dptr(T),
                           dptr(sc) if sc.size else None, int(sc.size), float(frequency), float(frequency_phase),
                           float(time_offset))
        except ValueError as e:
            raise ValueError("Could not import magnetic field.  Check 'ifile' and 'iformat' are correct (%s)" % e)

    def add_bfield_grid(self, values, npoints, start, step, rotations=[], translation=[], frequency=0,
                        frequency_phase=0, time_offset=0, name=""):
        """Grid field from memory (this build's extension): ``values`` has shape
        (nx, ny, nz, 3) or (nx * ny * nz, 3) in the reference's order (x slowest, z fastest);
        interpolation and conventions as add_bfield_file."""
        n = [int(v) for v in npoints]
        if len(n) != 3:
            raise ValueError("'npoints' must have 3 entries [nx, ny, nz]")
        v = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(-1, 3))
        if v.shape[0] != n[0] * n[1] * n[2]:
            raise ValueError("'values' must hold nx * ny * nz field vectors")
        d = FieldDesc(kind=2, frequency=float(frequency), frequency_phase=float(frequency_phase),
                      time_offset=float(time_offset))
        d.grid_n[:] = n
        d.grid_start[:] = _vec3(start, "start")
        d.grid_step[:] = _vec3(step, "step")
        d.grid_values = dptr(v)
        d.rotations[:] = _vec3(rotations, "rotations") if len(rotations) else [0.0, 0.0, 0.0]
        d.center[:] = _vec3(translation, "translation") if len(translation) else [0.0, 0.0, 0.0]
        self._ctx.call("osc_add_field", ctypes.byref(d))

    def add_bfield_epu(self, period, nperiods, bfieldA=[], bfieldB=[], phase=0, rotations=[], translation=[],
                       taper=0, frequency=0, frequency_phase=0, time_offset=0, name=""):
        if len(bfieldA) == 0 and len(bfieldB) == 0:
            raise ValueError("Must define at least one of 'bfieldA', 'bfieldB'")
        fa = _vec3(bfieldA, "bfieldA") if len(bfieldA) else [0.0, 0.0, 0.0]
        fb = _vec3(bfieldB, "bfieldB") if len(bfieldB) else [0.0, 0.0, 0.0]
        p = _vec3(period, "period")
        r = _vec3(rotations, "rotations") if len(rotations) else [0.0, 0.0, 0.0]
        t = _vec3(translation, "translation") if len(translation) else [0.0, 0.0, 0.0]
        d = FieldDesc(kind=1, nperiods=int(nperiods), phase=float(phase), taper=float(taper),
                      frequency=float(frequency), frequency_phase=float(frequency_phase),
                      time_offset=float(time_offset))
        d.bfield[:] = _rotate_xyz(fa, r)
        d.bfield_b[:] = _rotate_xyz(fb, r)
        d.period[:] = _rotate_xyz(p, r)
        d.center[:] = t
        self._ctx.call("osc_add_field", ctypes.byref(d))

    def get_bfield(self, x, t=0, name=""):
        X = np.array(_vec3(x, "x"))
        out = np.zeros(3)
        self._ctx.call("osc_get_bfield", dptr(X), float(t), dptr(out))
        return list(map(float, out))

    # ---- beam (src/OSCARSSR_Python.cc:3561-3576, 3699-4100) --------------------------------------
    def clear_particle_beams(self):
        self._ctx.call("osc_clear_beams")
        self._nbeams = 0

    def set_particle_beam(self, **kw):
        self.clear_particle_beams()
        self.add_particle_beam(**kw)

    def add_particle_beam(self, type="electron", name="", energy_GeV=-1, d0=None, x0=None, beam="",
                          sigma_energy_GeV=0, t0=0, current=0, weight=1, rotations=None, translation=None,
                          horizontal_direction=None, beta=None, alpha=None, gamma=None, emittance=None, eta=None,
                          lattice_reference=None, mass=0, charge=0, ctstartstop=None, distribution=""):
        predefined = 0
        if beam:  # TParticleBeam::SetPredefinedBeam (src/TParticleBeam.cc:135-206)
            predefined = _PREDEFINED_BEAMS.get(beam.upper(), -1)
            if predefined < 0:
                raise ValueError("Error in predefined beam name / definition")
        elif type not in _PARTICLES:
            raise ValueError("invalid argument in adding particle beam.  possibly 'name' already exists")
        pos = _vec3(x0, "x0") if x0 is not None else [0.0, 0.0, 0.0]
        if energy_GeV != -1 and energy_GeV < 0:
            raise ValueError("We do not currently support negative energy beams.  Please change 'energy_GeV' to >= 0")
        dr = _vec3(d0, "d0") if d0 is not None else [0.0, 0.0, 1.0]
        rot = _vec3(rotations, "rotations") if rotations is not None else [0.0, 0.0, 0.0]
        tr = _vec3(translation, "translation") if translation is not None else [0.0, 0.0, 0.0]
        if horizontal_direction is not None:
            hd = _vec3(horizontal_direction, "horizontal_direction")
        else:  # -Direction.Orthogonal() of the un-rotated direction (include/TVector3D.h:132-142)
            ax, ay, az = (-v if v < 0.0 else v for v in dr)
            if ax < ay:
                o = [0.0, dr[2], -dr[1]] if ax < az else [dr[1], -dr[0], 0.0]
            else:
                o = [-dr[2], 0.0, dr[0]] if ay < az else [dr[1], -dr[0], 0.0]
            hd = [-o[0], -o[1], -o[2]]
        pos = _rotate_xyz(pos, rot)
        dr = _rotate_xyz(dr, rot)
        pos = [pos[0] + tr[0], pos[1] + tr[1], pos[2] + tr[2]]
        if type == "custom" and (mass == 0 or charge == 0):
            raise ValueError("'mass' or 'charge' is zero")
        d = BeamDesc(particle=_PARTICLES.get(type, 0), charge=float(charge), mass=float(mass),
                     energy_GeV=float(energy_GeV), t0=float(t0), current=float(current),
                     sigma_energy_GeV=float(sigma_energy_GeV), predefined=predefined, has_d0=int(d0 is not None),
                     weight=float(weight))
        d.x0[:] = pos
        d.d0[:] = dr
        d.horizontal[:] = hd
        if emittance is not None:
            d.emittance[:] = _vec2(emittance, "emittance")
            d.has_emittance = 1
        if beta is not None:
            d.beta[:] = _vec2(beta, "beta")
            d.has_beta = 1
        if alpha is not None:
            d.alpha[:] = _vec2(alpha, "alpha")
            d.has_alpha = 1
        if gamma is not None:
            d.gamma[:] = _vec2(gamma, "gamma")
            d.has_gamma = 1
        if lattice_reference is not None:
            d.lattice_reference[:] = _vec3(lattice_reference, "lattice_reference")
            d.has_lattice_reference = 1
        if eta is not None:
            d.eta[:] = _vec2(eta, "gamma")
        dist = {"": -1, "filament": 1, "gaussian": 2, "kv": 3}
        if distribution.lower() not in dist:
            raise ValueError("Unknown beam distribution name: " + distribution)
        d.distribution = dist[distribution.lower()]
        if ctstartstop is not None:
            d.ctstartstop[:] = _vec2(ctstartstop, "ctstartstop")
            d.has_ctstartstop = 1
        self._ctx.call("osc_add_beam", ctypes.byref(d), str(name).encode())
        self._nbeams += 1

    def set_new_particle(self, beam="", particle=""):
        """A new particle from the named beam, or from a beam picked by weight (beam=""): the ideal one
        (particle='ideal') or a random one (src/OSCARSSR.cc:510-524)."""
        self._ctx.call("osc_set_new_particle_of_beam", str(beam).encode(), int(particle.lower() == "ideal"))

    def _particle(self):
        x0, b0 = np.zeros(3), np.zeros(3)
        t0, g = ctypes.c_double(), ctypes.c_double()
        self._ctx.call("osc_get_particle", dptr(x0), dptr(b0), ctypes.byref(t0), ctypes.byref(g))
        return x0, b0, t0.value, g.value

    def beam_particles(self, n, shard=(0, 1)):
        """The particles a request with nparticles = n draws (same random sequence), restricted to
        shard (rank, count): array (k, 6) of x0 [m] and beta0."""
        rank, count = int(shard[0]), int(shard[1])
        out = np.zeros(6 * ((int(n) + count - 1) // count + 1))
        k = ctypes.c_longlong()
        self._ctx.call("osc_beam_particles", int(n), rank, count, dptr(out), ctypes.byref(k))
        return out[:6 * k.value].reshape(k.value, 6)

    def get_particle_x0(self):
        return list(map(float, self._particle()[0]))

    def get_particle_beta0(self):
        return list(map(float, self._particle()[1]))

    # ---- trajectory ------------------------------------------------------------------------------
    def set_ctstartstop(self, start, stop):
        self._ctx.call("osc_set_ctstartstop", float(start), float(stop))

    def _ctss(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._ctx.call("osc_get_ctstartstop", ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def get_ctstart(self):
        return self._ctss()[0]

    def get_ctstop(self):
        return self._ctss()[1]

    def set_npoints_trajectory(self, npoints):
        self._ctx.call("osc_set_npoints_trajectory", int(npoints))

    def set_trajectory_calculation(self, method, precision=-1):
        """'RK4' (fixed step, the default) or 'RKAS' (adaptive Cash-Karp steps at `precision`, default
        1e-6), src/OSCARSSR_Python.cc:5115-5146."""
        self._ctx.call("osc_set_trajectory_calculation", str(method).encode(), float(precision))

    def print_trajectory(self):
        m, p = ctypes.c_int(), ctypes.c_double()
        self._ctx.call("osc_get_trajectory_calculation", ctypes.byref(m), ctypes.byref(p))
        sys.stdout.write("*Trajectory Calculation Globals*\nMethod:    %s\nPrecision: %s\n\n"
                         % ("RKAS" if m.value == 1 else "RK4", "%g" % p.value))

    def get_npoints_trajectory(self):
        n = ctypes.c_longlong()
        self._ctx.call("osc_get_npoints_trajectory", ctypes.byref(n))
        return n.value

    def trajectory_array(self):
        """(10, n) array: t, x, y, z, beta_x, beta_y, beta_z, a_x/c, a_y/c, a_z/c."""
        n = ctypes.c_longlong()
        self._ctx.call("osc_get_trajectory", None, 0, ctypes.byref(n))
        out = np.zeros(10 * n.value)
        self._ctx.call("osc_get_trajectory", dptr(out), out.size, ctypes.byref(n))
        return out.reshape(10, n.value)

    def get_trajectory(self):
        a = self.trajectory_array()
        return [[float(a[0, i]), a[1:4, i].tolist(), a[4:7, i].tolist(), a[7:10, i].tolist()] for i in range(a.shape[1])]

    def calculate_trajectory(self, ofile="", bofile="", oformat=""):
        self._ctx.call("osc_calculate_trajectory")
        if ofile or bofile:  # TParticleTrajectoryPoints::WriteToFile / WriteToFileBinary formats
            a = self.trajectory_array()
            if ofile:
                fileio.write_trajectory_text(ofile, a, oformat)
            if bofile:
                fileio.write_trajectory_binary(bofile, a, oformat)
        return self.get_trajectory()

    # ---- radiation -------------------------------------------------------------------------------
    def _check_gpu(self, gpu, nthreads):
        if gpu not in (0, 1, -1):
            raise ValueError("'gpu' must be 0 or 1")
        if nthreads < 0:
            raise ValueError("'nthreads' must be > 0")
        if nthreads > 0 and gpu == 1:
            raise ValueError("gpu is 1 and nthreads > 0.  Both are not currently allowed.")
        if gpu == 0:
            raise ValueError("gpu=0 selects the reference's CPU path; this build computes on the GPU only")

    def _opts(self, polarization, angle, horizontal_direction, propogation_direction, precision, max_level,
              max_level_extended, nparticles, quantity, compute, shard=None):
        o = RadOpts()
        if shard is not None:  # (rank, count): this process's share of a multi-particle request
            rank, count = int(shard[0]), int(shard[1])
            if count < 1 or not 0 <= rank < count:
                raise ValueError("'shard' must be (rank, count) with 0 <= rank < count")
            o.shard_rank, o.shard_count = rank, count
        o.polarization = _polarization(polarization, angle)
        o.angle = float(angle)
        o.horizontal[:] = _vec3(horizontal_direction, "translation") if horizontal_direction else [1.0, 0.0, 0.0]
        o.propagation[:] = _vec3(propogation_direction, "translation") if propogation_direction else [0.0, 0.0, 1.0]
        o.precision = float(precision)
        o.max_level = int(max_level)
        o.max_level_extended = int(max_level_extended)
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        o.nparticles = int(nparticles)
        o.quantity = quantity
        o.precision_mode = _compute_mode(compute)
        return o

    def _report(self, nnc):
        if nnc.value > 0:
            sys.stderr.write(_NOT_CONVERGED)

    @staticmethod
    def _energies(npoints, energy_range_eV, energy_points_eV):
        """TSpectrumContainer::Init (src/TSpectrumContainer.cc:57-112) and the binding's default
        point count (src/OSCARSSR_Python.cc:5817-5822)."""
        if energy_points_eV is not None:
            if len(energy_points_eV) == 0:
                raise ValueError("Number of points to calculate is zero.  Check input.")
            return np.array([float(e) for e in energy_points_eV])
        e0 = e1 = 0.0
        if energy_range_eV is not None:
            if len(energy_range_eV) != 2:
                raise ValueError("'energy_range_eV' must be a list of length 2")
            e0, e1 = float(energy_range_eV[0]), float(energy_range_eV[1])
        if npoints < 1:
            npoints = abs(int(e1 - e0) + 1) if abs(e1 - e0) + 1 > 100 else 100
        if npoints == 1:
            return np.array([e0])
        return np.array([e0 + (e1 - e0) / (npoints - 1) * float(i) for i in range(npoints)])

    def calculate_spectrum(self, obs, npoints=0, energy_range_eV=None, energy_points_eV=None, points_eV=None,
                           polarization="", angle=_ANGLE_UNSET, horizontal_direction=None, propogation_direction=None,
                           precision=0.01, max_level=-2, max_level_extended=0, nparticles=0, nthreads=0, gpu=-1,
                           ngpu=None, quantity="flux", ofile="", bofile="", *, compute="fp64", return_numpy=False,
                           shard=None):
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        if points_eV is not None:
            energy_points_eV = points_eV
        E = self._energies(npoints, energy_range_eV, energy_points_eV)
        O = np.array(_vec3(obs, "obs"))
        self._check_gpu(gpu, nthreads)
        q = _quantity(quantity)
        o = self._opts(polarization, angle, horizontal_direction, propogation_direction, precision, max_level,
                       max_level_extended, nparticles, q, compute, shard)
        out = np.zeros(E.size)
        lv = np.zeros(E.size, dtype=np.int32)
        nnc = ctypes.c_longlong()
        self._ctx.call("osc_spectrum", dptr(O), dptr(E), E.size, ctypes.byref(o), dptr(out), i32ptr(lv), ctypes.byref(nnc))
        self.last_levels = lv
        self._report(nnc)
        if ofile:
            fileio.write_spectrum_text(ofile, E, out)
        if bofile:
            fileio.write_spectrum_binary(bofile, E, out)
        if return_numpy:
            return E, out
        return [[float(E[i]), float(out[i])] for i in range(E.size)]

    def _rectangle(self, npoints, plane, width, x0x1x2, rotations, translation, normal, pd):
        if len(npoints) != 2:
            raise ValueError("'npoints' must be [int, int]")
        nx1, nx2 = int(npoints[0]), int(npoints[1])
        if nx1 <= 0 or nx2 <= 0:
            raise ValueError("an entry in 'npoints' is <= 0")
        r = np.array(_vec3(rotations, "rotations") if rotations else [0.0, 0.0, 0.0])
        t = np.array(_vec3(translation, "translation") if translation else [0.0, 0.0, 0.0])
        w1, w2 = (0.010, 0.010) if pd else (0.0, 0.0)
        if width is not None and len(width) == 2:
            w1, w2 = float(width[0]), float(width[1])
        if abs(normal) > 1:
            raise ValueError("'normal' must be -1, 0, or 1")
        n = nx1 * nx2
        if x0x1x2 is not None:  # the three-point form (src/OSCARSSR_Python.cc:6633-6658, 8146-8172)
            if len(x0x1x2) != 3:
                raise ValueError("'x0x1x2' must have 3 XYZ points defined correctly")
            pts = np.array([_vec3(p, "x0x1x2") for p in x0x1x2], dtype=np.float64).ravel()
            xyz, nrm, x12 = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n)
            rc = _lib.lib().osc_surface_x0x1x2(nx1, nx2, dptr(pts), dptr(r), dptr(t), int(normal), dptr(xyz), dptr(nrm),
                                               dptr(x12))
            if rc != 0:
                raise ValueError(_lib.lib().osc_last_error(None).decode())
            return xyz, nrm, x12
        if w1 <= 0 or w2 <= 0:
            raise ValueError("'width' must be > 0" if pd else "'width' must be given as [w1, w2] with both > 0")
        xyz, nrm, x12 = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n)
        rc = _lib.lib().osc_surface_rectangle(plane.encode(), nx1, nx2, w1, w2, dptr(r), dptr(t), int(normal),
                                              dptr(xyz), dptr(nrm), dptr(x12))
        if rc != 0:
            raise ValueError(_lib.lib().osc_last_error(None).decode())
        return xyz, nrm, x12

    @staticmethod
    def _write_points(ofile, bofile, pos, out, dim):
        """ofile / bofile of the flux and power-density calls (T3DScalarContainer formats)."""
        if ofile:
            fileio.write_points_text(ofile, pos, out, dim)
        if bofile:
            fileio.write_points_binary(bofile, pos, out, dim)

    def _surface_points(self, points, rotations, translation, invert_normals):
        """Points with normals of the point-list calls (src/OSCARSSR_Python.cc:7728-7755, 6223-6255)."""
        r = np.array(_vec3(rotations, "rotations") if rotations else [0.0, 0.0, 0.0])
        t = np.array(_vec3(translation, "translation") if translation else [0.0, 0.0, 0.0])
        pts, nrm = [], []
        for item in points:
            if len(item) != 2:
                raise ValueError("Incorrect format in 'points'")
            if len(item[0]) != 3 or len(item[1]) != 3:
                raise ValueError("Incorrect format in 'points': Point or Normal does not have 3 elements")
            pts.append([float(v) for v in item[0]])
            nrm.append([float(v) for v in item[1]])
        n = len(pts)
        P = np.ascontiguousarray(np.array(pts, dtype=np.float64).reshape(-1))
        N = np.ascontiguousarray(np.array(nrm, dtype=np.float64).reshape(-1))
        xyz, nout = np.zeros(3 * n), np.zeros(3 * n)
        if n:
            rc = _lib.lib().osc_surface_points(n, dptr(P), dptr(N), dptr(r), dptr(t), int(bool(invert_normals)),
                                               dptr(xyz), dptr(nout))
            if rc != 0:
                raise ValueError(_lib.lib().osc_last_error(None).decode())
        return xyz, nout

    def calculate_flux(self, energy_eV=0.0, points=[], normal=0, rotations=None, translation=None, nparticles=0,
                       nthreads=0, gpu=-1, ngpu=None, precision=0.01, max_level=-2, max_level_extended=0, ofile="",
                       bofile="", quantity="flux", *, compute="fp64", return_numpy=False, shard=None):
        """Flux at arbitrary points ([[x, y, z], [nx, ny, nz]] each, rotated then translated), total
        polarization; returns [[x, y, z], F] (src/OSCARSSR_Python.cc:7628).  The reference binding
        raises before computing ("not currently used", :7812); here the flux is computed."""
        if self._nbeams < 1:
            raise ValueError("No particle beam defined")
        xyz, _ = self._surface_points(points, rotations, translation, False)
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        self._check_gpu(gpu, nthreads)
        q = _quantity(quantity)
        o = self._opts("", _ANGLE_UNSET, None, None, precision, max_level, max_level_extended, nparticles, q, compute,
                       shard)
        n = xyz.size // 3
        out = np.zeros(n)
        lv = np.zeros(n, dtype=np.int32)
        nnc = ctypes.c_longlong()
        if n:
            self._ctx.call("osc_flux", dptr(xyz), n, float(energy_eV), ctypes.byref(o), dptr(out), i32ptr(lv),
                           ctypes.byref(nnc))
        self.last_levels = lv
        self._report(nnc)
        self._write_points(ofile, bofile, xyz, out, 3)
        return self._points_result(xyz, out, return_numpy)

    def calculate_power_density(self, points, normal=0, rotations=None, translation=None, nparticles=0, gpu=-1,
                                ngpu=None, nthreads=0, precision=0.01, max_level=-2, max_level_extended=0,
                                quantity="power density", ofile="", bofile="", *, compute="fp64", return_numpy=False,
                                shard=None):
        """Power density [W/mm^2] at arbitrary points with surface normals ([[x, y, z], [nx, ny, nz]]
        each, rotated then translated; normal = -1 reverses the normals, normal != 0 makes it
        directional), src/OSCARSSR_Python.cc:6105-6370; returns [[x, y, z], P]."""
        if self._nbeams < 1:
            raise ValueError("No particle beam defined")
        xyz, nrm = self._surface_points(points, rotations, translation, normal == -1)
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        self._check_gpu(gpu, nthreads)
        q = _quantity(quantity, pd=True)
        o = self._opts("", _ANGLE_UNSET, None, None, precision, max_level, max_level_extended, nparticles, q, compute,
                       shard)
        n = xyz.size // 3
        out = np.zeros(n)
        lv = np.zeros(n, dtype=np.int32)
        nnc = ctypes.c_longlong()
        if n:
            self._ctx.call("osc_power_density", dptr(xyz), dptr(nrm), n, int(normal != 0), ctypes.byref(o), dptr(out),
                           i32ptr(lv), ctypes.byref(nnc))
        self.last_levels = lv
        self._report(nnc)
        self._write_points(ofile, bofile, xyz, out, 3)
        return self._points_result(xyz, out, return_numpy)

    @staticmethod
    def _points_result(pos, out, return_numpy):
        pos = pos.reshape(-1, 3)
        if return_numpy:
            return pos, out
        return [[pos[i].tolist(), float(out[i])] for i in range(out.size)]

    def calculate_flux_rectangle(self, energy_eV, npoints=[51, 51], plane="XY", normal=0, dim=2, width=None,
                                 rotations=None, translation=None, x0x1x2=None, polarization="", angle=_ANGLE_UNSET,
                                 horizontal_direction=None, propogation_direction=None, nparticles=0, nthreads=0,
                                 gpu=-1, ngpu=None, precision=0.01, max_level=-2, max_level_extended=0,
                                 quantity="flux", ofile="", bofile="", *, compute="fp64", return_numpy=False,
                                 shard=None):
        if self._nbeams < 1:
            raise ValueError("No particle beam defined")
        if dim not in (2, 3):
            raise ValueError("'dim' must be 2 or 3")
        xyz, nrm, x12 = self._rectangle(npoints, plane, width, x0x1x2, rotations, translation, normal, False)
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        self._check_gpu(gpu, nthreads)
        q = _quantity(quantity)
        o = self._opts(polarization, angle, horizontal_direction, propogation_direction, precision, max_level,
                       max_level_extended, nparticles, q, compute, shard)
        n = xyz.size // 3
        out = np.zeros(n)
        lv = np.zeros(n, dtype=np.int32)
        nnc = ctypes.c_longlong()
        self._ctx.call("osc_flux", dptr(xyz), n, float(energy_eV), ctypes.byref(o), dptr(out), i32ptr(lv), ctypes.byref(nnc))
        self.last_levels = lv
        self._report(nnc)
        self._write_points(ofile, bofile, xyz if dim == 3 else x12, out, dim)
        return self._points_result(xyz if dim == 3 else x12, out, return_numpy)

    def calculate_power_density_rectangle(self, npoints=[51, 51], plane="XY", width=None, x0x1x2=None,
                                          rotations=None, translation=None, ofile="", bofile="", normal=0,
                                          nparticles=0, gpu=-1, ngpu=None, nthreads=0, precision=0.01, max_level=-2,
                                          max_level_extended=0, dim=2, quantity="power density", *, compute="fp64",
                                          return_numpy=False, shard=None):
        if self._nbeams < 1:
            raise ValueError("No particle beam defined")
        if dim not in (2, 3):
            raise ValueError("'dim' must be 2 or 3")
        xyz, nrm, x12 = self._rectangle(npoints, plane, width, x0x1x2, rotations, translation, normal, True)
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        self._check_gpu(gpu, nthreads)
        q = _quantity(quantity, pd=True)
        o = self._opts("", _ANGLE_UNSET, None, None, precision, max_level, max_level_extended, nparticles, q, compute,
                       shard)
        n = xyz.size // 3
        out = np.zeros(n)
        lv = np.zeros(n, dtype=np.int32)
        nnc = ctypes.c_longlong()
        self._ctx.call("osc_power_density", dptr(xyz), dptr(nrm), n, int(normal != 0), ctypes.byref(o), dptr(out),
                       i32ptr(lv), ctypes.byref(nnc))
        self.last_levels = lv
        self._report(nnc)
        self._write_points(ofile, bofile, xyz if dim == 3 else x12, out, dim)
        return self._points_result(xyz if dim == 3 else x12, out, return_numpy)

    # ---- STL surfaces (src/OSCARSSR_Python.cc:6852-7280, 9262-9276) ----------------------------------
    def add_stl(self, ifile, rotations=None, translation=None, scale=1, name=""):
        """Import a binary STL mesh: vertices times `scale`, then translated; `rotations` is accepted
        and, as in the reference, not applied."""
        if rotations is not None:
            _vec3(rotations, "rotations")
        t = _vec3(translation, "translation") if translation is not None else [0.0, 0.0, 0.0]
        self._stl.add(ifile, float(scale), t, name)

    def clear_stl(self):
        self._stl.clear()

    def remove_stl(self, name):
        self._stl.remove(name)

    def print_stl(self):
        sys.stdout.write(self._stl.describe())

    def calculate_power_density_stl(self, farfield_origin, ofile="", bofile="", stlofile="", nparticles=0, gpu=-1,
                                    ngpu=None, nthreads=0, precision=0.01, max_level=-2, max_level_extended=0,
                                    quantity="power density"):
        """Power density [W/mm^2] at the centre of every facet of the STL objects, each trajectory
        sample skipped when another facet lies between it and the centre (src/OSCARSSR.cc:3154-3521);
        returns [[[A], [B], [C]], P] per facet.  As in the reference binding, ofile and bofile write
        nothing for this call and stlofile re-exports the meshes (TSTLContainer::WriteSTLFile);
        farfield_origin is read and not used (the reference's shadowing mode that used it is off)."""
        if self._nbeams < 1:
            raise ValueError("No particle beam defined")
        _vec3(farfield_origin, "farfield_origin")
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        self._check_gpu(gpu, nthreads)
        q = _quantity(quantity, pd=True)
        o = self._opts("", _ANGLE_UNSET, None, None, precision, max_level, max_level_extended, nparticles, q, "fp64")
        facets, centers = self._stl.facets()
        n = facets.shape[0]
        out = np.zeros(n)
        lv = np.zeros(n, dtype=np.int32)
        nnc = ctypes.c_longlong()
        if n:
            self._ctx.call("osc_power_density_stl", dptr(facets), dptr(centers), n, ctypes.byref(o), dptr(out),
                           i32ptr(lv), ctypes.byref(nnc))
        self.last_levels = lv
        if stlofile:
            self._stl.write_stl(stlofile)
        return [[[facets[i, 0:3].tolist(), facets[i, 3:6].tolist(), facets[i, 6:9].tolist()], float(out[i])]
                for i in range(n)]

    def last_stats(self):
        """(samples integrated, kernel launches) of the last radiation call."""
        s, l = ctypes.c_longlong(), ctypes.c_longlong()
        self._ctx.call("osc_last_stats", ctypes.byref(s), ctypes.byref(l))
        return s.value, l.value
