"""Python face of the CPU oracle (TEST INFRASTRUCTURE ONLY).

``OracleSR`` exposes the subset of the reference ``oscars.sr`` API that the radiation hot path uses,
with the same keyword names, defaults, return shapes and error behaviour, on top of the C
restatement in ``oscars_oracle.c``.  Tests drive the reference build (``oracle/_ref``), this oracle
and the oscars_b200 product with the same calls and compare the results.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module; the
product never does.

Front-end logic restated here (reference file:line):
  * rectangle surfaces: TSurfacePoints_Rectangle::Init/GetXYZ/GetX1/GetX2
    (src/TSurfacePoints_Rectangle.cc:140-315)
  * RotateSelfXYZ (src/TVector3D.cc RotateSelfX/Y/Z)
  * spectrum energies: TSpectrumContainer::Init (src/TSpectrumContainer.cc:57-92)
  * polarization strings: src/OSCARSSR.cc:4129-4150 and the binding defaults
    (src/OSCARSSR_Python.cc:5889-5899)
"""
from __future__ import annotations

import ctypes
import math
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboscars_oracle.so")
_ANGLE_UNSET = 112188979912321.0
_PARTICLE_TYPES = {
    "electron": 0, "anti-positron": 0, "positron": 1, "anti-electron": 1, "muon": 2,
    "anti-muon": 3, "proton": 4, "anti-proton": 5, "pi+": 6, "pi-": 7, "custom": 8,
}

_lib = None


def load():
    """Load (building if needed) the oracle shared library."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        import subprocess
        subprocess.check_call(["make", "-s", "-C", _HERE, "oracle"])
    lib = ctypes.CDLL(_LIB_PATH)
    D = ctypes.c_double
    P = ctypes.POINTER
    dp = P(D)
    ip = P(ctypes.c_int)
    lib.orc_new.restype = ctypes.c_void_p
    lib.orc_free.argtypes = [ctypes.c_void_p]
    lib.orc_last_error.restype = ctypes.c_char_p
    lib.orc_last_error.argtypes = [ctypes.c_void_p]
    lib.orc_clear_fields.argtypes = [ctypes.c_void_p]
    lib.orc_add_undulator.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_int, dp, D, D, D, D, D]
    lib.orc_add_epu.argtypes = [ctypes.c_void_p, dp, dp, dp, ctypes.c_int, dp, D, D, D, D, D]
    lib.orc_get_bfield.argtypes = [ctypes.c_void_p, dp, D, dp]
    lib.orc_set_half_period_scale.argtypes = [ctypes.c_void_p, dp, ctypes.c_int]
    lib.orc_add_grid.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long), dp, dp, dp, dp, dp, dp, D, D, D]
    lib.orc_set_beam.argtypes = [ctypes.c_void_p, ctypes.c_int, D, D, D, dp, dp, D, D, dp, ctypes.c_int, D, dp,
                                 ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, dp,
                                 ctypes.c_int, dp, ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, D,
                                 ctypes.c_int]
    lib.orc_set_new_particle_of.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    lib.orc_set_ctstartstop.argtypes = [ctypes.c_void_p, D, D]
    lib.orc_set_npoints_trajectory.argtypes = [ctypes.c_void_p, ctypes.c_long]
    lib.orc_get_npoints_trajectory.argtypes = [ctypes.c_void_p]
    lib.orc_get_npoints_trajectory.restype = ctypes.c_long
    lib.orc_set_seed.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.orc_uniform.argtypes = [ctypes.c_void_p]
    lib.orc_uniform.restype = D
    lib.orc_normal.argtypes = [ctypes.c_void_p]
    lib.orc_normal.restype = D
    lib.orc_set_new_particle.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.orc_get_particle.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp, dp, dp]
    lib.orc_set_particle.argtypes = [ctypes.c_void_p, dp, dp, D]
    lib.orc_calculate_trajectory.argtypes = [ctypes.c_void_p]
    lib.orc_trajectory_npoints.argtypes = [ctypes.c_void_p]
    lib.orc_trajectory_npoints.restype = ctypes.c_long
    lib.orc_get_trajectory.argtypes = [ctypes.c_void_p, dp, ctypes.c_long]
    lib.orc_get_spline_ypp.argtypes = [ctypes.c_void_p, dp, ctypes.c_long]
    lib.orc_get_level.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, ctypes.c_long]
    lib.orc_flux.argtypes = [ctypes.c_void_p, dp, ctypes.c_long, D, ctypes.c_int, D, dp, dp, D,
                             ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, ip]
    lib.orc_spectrum.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_long, ctypes.c_int, D, dp, dp,
                                 D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, ip]
    lib.orc_power_density.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_long, ctypes.c_int, D,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, ip]
    lib.orc_set_trajectory_calculation.argtypes = [ctypes.c_void_p, ctypes.c_int, D]
    lib.orc_power_density_stl.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_long, D, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, dp, ip]
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _v3(x, name="vector"):
    if x is None:
        return None
    x = list(x)
    if len(x) != 3:
        raise ValueError("Incorrect format in '%s'" % name)
    return [float(v) for v in x]


# ---- vector helpers restating src/TVector3D.cc (pure Python floats are IEEE doubles) ----------
def rotate_xyz(v, r):
    """TVector3D::RotateSelfXYZ: about X, then Y, then Z."""
    x, y, z = v
    s, c = math.sin(r[0]), math.cos(r[0])
    yy = y
    y = c * yy - s * z
    z = s * yy + c * z
    s, c = math.sin(r[1]), math.cos(r[1])
    zz = z
    z = c * zz - s * x
    x = s * zz + c * x
    s, c = math.sin(r[2]), math.cos(r[2])
    xx = x
    x = c * xx - s * y
    y = s * xx + c * y
    return [x, y, z]


def _mag(v):
    return math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])


def rectangle(plane, nx1, nx2, w1, w2, rotations, translation, normal):
    """TSurfacePoints_Rectangle::Init(plane, ...) + GetXYZ/GetX1/GetX2.  Returns (xyz, normals,
    x1x2) arrays in point order i = ix1*NX2 + ix2."""
    P = plane.upper()
    s1 = w1 / (nx1 - 1) if nx1 > 1 else 0
    s2 = w2 / (nx2 - 1) if nx2 > 1 else 0

    def start(a, b, c):
        return [a, b, c]
    table = {
        "XY": ((-w1 / 2., -w2 / 2., 0), (0, 0, 0), (0., -w2 / 2., 0), (-w1 / 2., 0, 0), (s1, 0, 0), (0, s2, 0), (0, 0, 1)),
        "YX": ((-w2 / 2., -w1 / 2., 0), (0, 0, 0), (-w2 / 2., 0, 0), (0, -w1 / 2., 0), (0, s1, 0), (s2, 0, 0), (0, 0, -1)),
        "XZ": ((-w1 / 2., 0, -w2 / 2.), (0, 0, 0), (0, 0, -w2 / 2.), (-w1 / 2., 0, 0), (s1, 0, 0), (0, 0, s2), (0, -1, 0)),
        "ZX": ((-w2 / 2., 0, -w1 / 2.), (0, 0, 0), (-w2 / 2., 0, 0), (0., 0, -w1 / 2.), (0, 0, s1), (s2, 0, 0), (0, 1, 0)),
        "YZ": ((0, -w1 / 2., -w2 / 2.), (0, 0, 0), (0, 0, -w2 / 2.), (0, -w1 / 2., 0), (0, s1, 0), (0, 0, s2), (1, 0, 0)),
        "ZY": ((0, -w2 / 2., -w1 / 2.), (0, 0, 0), (0, -w2 / 2., 0), (0, 0, -w1 / 2.), (0, 0, s1), (0, s2, 0), (-1, 0, 0)),
    }
    if P not in table:
        raise ValueError("not a valid surface string: XY YX XZ ZX YZ ZY")
    both, none, only2, only1, v1, v2, nv = table[P]
    if nx1 > 1 and nx2 > 1:
        st = list(both)
    elif nx1 <= 1 and nx2 <= 1:
        st = list(none)
    elif nx1 <= 1:
        st = list(only2)
    else:
        st = list(only1)
    st = [float(a) for a in st]
    v1 = [float(a) for a in v1]
    v2 = [float(a) for a in v2]
    nv = [float(a) for a in nv]
    st = rotate_xyz(st, rotations)
    v1 = rotate_xyz(v1, rotations)
    v2 = rotate_xyz(v2, rotations)
    st = [st[0] + translation[0], st[1] + translation[1], st[2] + translation[2]]
    nv = rotate_xyz(nv, rotations)
    if normal == -1:
        nv = [nv[0] * -1, nv[1] * -1, nv[2] * -1]
    elif normal not in (0, 1):
        raise ValueError("normal must be -1, 0, or 1")
    n = nx1 * nx2
    xyz = np.empty((n, 3))
    x1x2 = np.zeros((n, 3))
    m1, m2 = _mag(v1), _mag(v2)
    for i in range(n):
        ix1 = i // nx2
        ix2 = i % nx2
        a = [st[k] + ix1 * v1[k] for k in range(3)]
        xyz[i] = [a[k] + ix2 * v2[k] for k in range(3)]
        x1x2[i, 0] = s1 * ix1 - m1 * (nx1 - 1) / 2.
        x1x2[i, 1] = s2 * ix2 - m2 * (nx2 - 1) / 2.
    normals = np.tile(np.array(nv), (n, 1))
    return xyz, normals, x1x2


# ---- grid field files (restating src/TField3D_Grid.cc:365-530 and :572-870) -------------------
def rectangle_x0x1x2(nx1, nx2, x0, x1, x2, rotations, translation, normal):
    """TSurfacePoints_Rectangle::Init(NX1, NX2, X0, X1, X2, Normal) + GetXYZ/GetX1/GetX2
    (src/TSurfacePoints_Rectangle.cc:76-127, 280-317), after the binding rotates and translates the
    three points (src/OSCARSSR_Python.cc:6652-6658).  Returns (xyz, normals, x1x2)."""
    if nx1 < 2 or nx2 < 2:
        raise ValueError("'npoints' must be >= 2 in each direction with 'x0x1x2'")
    P = []
    for v in (x0, x1, x2):
        w = rotate_xyz([float(a) for a in v], rotations)
        P.append([w[k] + translation[k] for k in range(3)])
    X0, X1, X2 = P
    d1 = [X1[k] - X0[k] for k in range(3)]
    d2 = [X2[k] - X0[k] for k in range(3)]
    s1 = _mag(d1) / (nx1 - 1)
    s2 = _mag(d2) / (nx2 - 1)
    v1 = [d1[k] / (nx1 - 1) for k in range(3)]
    v2 = [d2[k] / (nx2 - 1) for k in range(3)]
    c = [v1[1] * v2[2] - v2[1] * v1[2], v1[2] * v2[0] - v2[2] * v1[0], v1[0] * v2[1] - v2[0] * v1[1]]
    m = _mag(c)
    nv = [c[0] / m, c[1] / m, c[2] / m]
    if normal == -1:
        nv = [nv[0] * -1, nv[1] * -1, nv[2] * -1]
    elif normal not in (0, 1):
        raise ValueError("fNormal is of the incorrect form.  Must be -1, 0, 1")
    n = nx1 * nx2
    xyz = np.empty((n, 3))
    x1x2 = np.zeros((n, 3))
    m1, m2 = _mag(v1), _mag(v2)
    for i in range(n):
        ix1, ix2 = i // nx2, i % nx2
        a = [X0[k] + v1[k] * ix1 for k in range(3)]
        xyz[i] = [a[k] + v2[k] * ix2 for k in range(3)]
        x1x2[i, 0] = s1 * ix1 - m1 * (nx1 - 1) / 2.
        x1x2[i, 1] = s2 * ix2 - m2 * (nx2 - 1) / 2.
    return xyz, np.tile(np.array(nv), (n, 1)), x1x2


def surface_points(points, rotations, translation, invert_normals):
    """Points with normals as the point-list bindings take them (src/OSCARSSR_Python.cc:7728-7755,
    6223-6255): point and normal rotated, the normal reversed on request, the point translated."""
    xyz, nrm = [], []
    for item in points:
        if len(item) != 2:
            raise ValueError("Incorrect format in 'points'")
        X = rotate_xyz([float(v) for v in item[0]], rotations)
        N = rotate_xyz([float(v) for v in item[1]], rotations)
        if invert_normals:
            N = [N[0] * -1, N[1] * -1, N[2] * -1]
        xyz.append([X[k] + translation[k] for k in range(3)])
        nrm.append(N)
    return np.array(xyz, dtype=np.float64).reshape(-1, 3), np.array(nrm, dtype=np.float64).reshape(-1, 3)


def _first_number(line):
    """TField3D_Grid::GetHeaderValue: the first number on the line (0 when there is none)."""
    tok = line.split()
    try:
        return float(tok[0]) if tok else 0.0
    except ValueError:
        return 0.0


def read_oscars_grid(path, rotations, scaling):
    """'OSCARS' format: comment line, 9 header lines (start, step, n for x, y, z), then
    nx*ny*nz lines 'Fx Fy Fz' with x slowest.  Returns (n, start, step, stop, values)."""
    with open(path) as fi:
        lines = fi.read().split("\n")
    hv = [_first_number(lines[1 + i]) if 1 + i < len(lines) else 0.0 for i in range(9)]
    xs, xst, nx, ys, yst, ny, zs, zst, nz = hv
    NX, NY, NZ = int(nx), int(ny), int(nz)
    sc = list(scaling)
    XStep = xst * sc[0] if len(sc) > 0 else xst
    YStep = yst * sc[1] if len(sc) > 1 else yst
    ZStep = zst * sc[2] if len(sc) > 2 else zst
    fsx = sc[3] if len(sc) > 3 else 1
    fsy = sc[4] if len(sc) > 4 else 1
    fsz = sc[5] if len(sc) > 5 else 1
    XStart = (xs + xst * (NX - 1) / 2.) - XStep * (NX - 1) / 2.
    YStart = (ys + yst * (NY - 1) / 2.) - YStep * (NY - 1) / 2.
    ZStart = (zs + zst * (NZ - 1) / 2.) - ZStep * (NZ - 1) / 2.
    if NX < 1 or NY < 1 or NZ < 1:
        raise ValueError("invalid number of points in at least one dimension")
    n = [NX, NY, NZ]
    start = [XStart, YStart, ZStart]
    step = [XStep, YStep, ZStep]
    stop = [start[a] + (n[a] - 1) * step[a] for a in range(3)]
    vals = np.empty((NX * NY * NZ, 3))
    k = 0
    for i in range(NX * NY * NZ):
        li = 10 + i
        if li >= len(lines) - 1:  # getline reached the end of the file (the reference checks eof())
            raise ValueError("error reading file.  Check format")
        tok = lines[li].split()
        try:
            fx, fy, fz = float(tok[0]), float(tok[1]), float(tok[2])
        except (IndexError, ValueError):
            raise ValueError("error reading file.  Check format")
        if fsx != 1:
            fx *= fsx
        if fsy != 1:
            fy *= fsy
        if fsz != 1:
            fz *= fsz
        vals[k] = rotate_xyz([fx, fy, fz], rotations)
        k += 1
    return n, start, step, stop, vals


def read_oscars1d_grid(path, fmt, rotations, scaling, comment="#"):
    """'OSCARS1D <columns>': irregular samples along one axis, sorted, resampled at 10000 points
    per metre by linear interpolation.  Returns (n, start, step, stop, values)."""
    order = [-1, -1, -1, -1]
    has = [False] * 4
    axis = ""
    index = xdim = fdim = 0
    for c in fmt[8:].split():
        if index > 3:
            raise ValueError("spatial or B-field dimensions are too large(index>3)")
        if c in ("X", "Y", "Z"):
            axis = c
            xdim += 1
            order[index] = 0
        elif c in ("Bx", "Ex", "Fx"):
            has[1] = True
            fdim += 1
            order[index] = 1
        elif c in ("By", "Ey", "Fy"):
            has[2] = True
            fdim += 1
            order[index] = 2
        elif c in ("Bz", "Ez", "Fz"):
            has[3] = True
            fdim += 1
            order[index] = 3
        else:
            raise ValueError("only excepts X Y Z Bx By Bz")
        index += 1
    count = xdim + fdim
    if xdim != 1:
        raise ValueError("spatial or B-field dimensions are too large")
    with open(path) as fi:
        lines = fi.read().split("\n")
    if lines and lines[-1] == "":
        lines = lines[:-1]
    data = []
    for L in lines[1:]:
        stripped = L.lstrip(" \t")
        if stripped == "" or stripped[0] == comment:
            continue
        tok = L.replace(",", " ").split()
        val = [0.0, 0.0, 0.0, 0.0]
        for i in range(count):
            try:
                val[order[i]] = float(tok[i])
            except (IndexError, ValueError):
                raise ValueError("something is incorrect with data format or iformat string")
        for i in range(min(len(scaling), 4)):
            if order[i] < 0:
                continue
            val[order[i]] *= scaling[i]
        data.append(val)
    data.sort(key=lambda a: a[0])
    if len(data) < 2:
        raise ValueError("not enough data points")
    first, last = data[0][0], data[-1][0]
    npts = int((last - first) * 10000)
    step = (last - first) / float(npts - 1)
    ax = {"X": 0, "Y": 1, "Z": 2}[axis]
    n, start, stp, stop = [1, 1, 1], [0.0] * 3, [0.0] * 3, [0.0] * 3
    n[ax], start[ax], stp[ax], stop[ax] = npts, first, step, last
    vals = np.empty((npts, 3))
    min_bin = after = before = 0
    for i in range(npts):
        z = i * step + first
        for j in range(min_bin + 1, len(data)):
            if data[j][0] > z:
                after, before, min_bin = j, j - 1, j - 1
                break
        nb = [0.0, 0.0, 0.0]
        for k in range(3):
            if has[k + 1]:
                slope = (data[after][k + 1] - data[before][k + 1]) / (data[after][0] - data[before][0])
                nb[k] = data[before][k + 1] + (z - data[before][0]) * slope
        vals[i] = rotate_xyz(nb, rotations)
    return n, start, stp, stop, vals


def polarization_code(polarization, angle):
    """Binding default (src/OSCARSSR_Python.cc:5889-5899) + string match (src/OSCARSSR.cc:4129-4150)."""
    if polarization == "all" and angle != _ANGLE_UNSET:
        raise ValueError("cannot specify 'all' and 'angle'.  This is to save you")
    pol = "all"
    if len(polarization) != 0:
        pol = polarization
    elif angle != _ANGLE_UNSET:
        pol = "linear"
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


def spectrum_energies(npoints, energy_range_eV, energy_points_eV):
    if energy_points_eV is not None:
        if len(energy_points_eV) == 0:
            raise ValueError("Number of points to calculate is zero.  Check input.")
        return np.array([float(e) for e in energy_points_eV])
    e0, e1 = 0.0, 0.0
    if energy_range_eV is not None:
        if len(energy_range_eV) != 2:
            raise ValueError("'energy_range_eV' must be a list of length 2")
        e0, e1 = float(energy_range_eV[0]), float(energy_range_eV[1])
    if npoints < 1:
        npoints = abs(int(e1 - e0) + 1) if abs(e1 - e0) + 1 > 100 else 100
    if npoints == 1:
        return np.array([e0])
    return np.array([e0 + (e1 - e0) / (npoints - 1) * float(i) for i in range(npoints)])


def _quantity(q, pd=False):
    Q = q.upper()
    if pd and Q in ("POWER DENSITY", "POWERDENSITY"):
        return 0
    if not pd and Q == "FLUX":
        return 0
    if Q == "PRECISION":
        return 1
    if Q == "LEVEL":
        return 2
    raise ValueError("'quantity' must be: 'flux', 'precision', 'level', or blank")


def read_stl(path, scale=1.0, translation=(0.0, 0.0, 0.0)):
    """TTriangle3DContainer::ReadSTLFile (src/TTriangle3DContainer.cc:109-214): binary STL, vertices
    float x scale, normals as stored, centre (A + B + C) / 3 before the translation, then vertices and
    centre translated; the rotations argument is reset before it is applied (identity).  Returns
    (n x 12 array of A, B, C, N; n x 3 centres)."""
    import struct
    with open(path, "rb") as f:
        data = f.read()
    n = struct.unpack_from("<I", data, 80)[0]
    tri = np.zeros((n, 12))
    cen = np.zeros((n, 3))
    T = [float(v) for v in translation]
    for i in range(n):
        vals = struct.unpack_from("<12f", data, 84 + 50 * i)
        N, A, B, C = vals[0:3], vals[3:6], vals[6:9], vals[9:12]
        A = [a * scale for a in A]
        B = [b * scale for b in B]
        C = [c * scale for c in C]
        ce = [((A[k] + B[k]) + C[k]) / 3. for k in range(3)]
        tri[i, 0:3] = [A[k] + T[k] for k in range(3)]
        tri[i, 3:6] = [B[k] + T[k] for k in range(3)]
        tri[i, 6:9] = [C[k] + T[k] for k in range(3)]
        tri[i, 9:12] = N
        cen[i] = [ce[k] + T[k] for k in range(3)]
    return tri, cen


class OracleSR:
    """CPU oracle with the ``oscars.sr.sr`` method names used on the radiation hot path."""

    def __init__(self, nthreads=0, gpu=0):
        self._lib = load()
        self._h = ctypes.c_void_p(self._lib.orc_new())
        self.last_levels = None

    def __del__(self):
        try:
            self._lib.orc_free(self._h)
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise ValueError(self._lib.orc_last_error(self._h).decode())

    # ---- setup ------------------------------------------------------------------------------
    def set_seed(self, seed):
        self._lib.orc_set_seed(self._h, int(float(seed)))

    def clear_bfields(self):
        self._lib.orc_clear_fields(self._h)

    def add_bfield_undulator(self, bfield, period, nperiods, phase=0, rotations=[], translation=[],
                             taper=0, frequency=0, frequency_phase=0, time_offset=0, name="",
                             half_period_scale=None):
        f = _v3(bfield, "bfield")
        p = _v3(period, "period")
        r = _v3(rotations, "rotations") if len(rotations) else [0.0, 0.0, 0.0]
        t = _v3(translation, "translation") if len(translation) else [0.0, 0.0, 0.0]
        f = rotate_xyz(f, r)
        p = rotate_xyz(p, r)
        a = lambda v: np.array(v, dtype=np.float64)
        F, Pp, T = a(f), a(p), a(t)
        self._check(self._lib.orc_add_undulator(self._h, _dp(F), _dp(Pp), int(nperiods), _dp(T),
                                                float(phase), float(taper), float(frequency),
                                                float(frequency_phase), float(time_offset)))
        if half_period_scale is not None:
            hs = np.ascontiguousarray(np.asarray(half_period_scale, dtype=np.float64))
            self._check(self._lib.orc_set_half_period_scale(self._h, _dp(hs), int(hs.size)))

    def _add_grid(self, n, start, step, stop, vals, rotations, translation, frequency, frequency_phase,
                  time_offset):
        N = (ctypes.c_long * 3)(*n)
        a = lambda v: np.ascontiguousarray(np.array(v, dtype=np.float64))
        S, St, Sp, V, R, T = a(start), a(step), a(stop), a(vals), a(rotations), a(translation)
        self._check(self._lib.orc_add_grid(self._h, N, _dp(S), _dp(St), _dp(Sp), _dp(V), _dp(R), _dp(T),
                                           float(frequency), float(frequency_phase), float(time_offset)))

    def add_bfield_file(self, ifile="", iformat="", rotations=[], translation=[], scale=[], frequency=0,
                        frequency_phase=0, time_offset=0, name=""):
        r = _v3(rotations, "rotations") if len(rotations) else [0.0, 0.0, 0.0]
        t = _v3(translation, "translation") if len(translation) else [0.0, 0.0, 0.0]
        F = iformat.upper()
        if F == "OSCARS":
            n, start, step, stop, vals = read_oscars_grid(ifile, r, list(scale))
        elif len(F) > 8 and F[:8] == "OSCARS1D":
            n, start, step, stop, vals = read_oscars1d_grid(ifile, iformat, r, list(scale))
        else:
            raise ValueError("format not restated by the oracle: %s" % iformat)
        self._add_grid(n, start, step, stop, vals, r, t, frequency, frequency_phase, time_offset)

    def add_bfield_grid(self, values, npoints, start, step, rotations=[], translation=[], frequency=0,
                        frequency_phase=0, time_offset=0, name=""):
        r = _v3(rotations, "rotations") if len(rotations) else [0.0, 0.0, 0.0]
        t = _v3(translation, "translation") if len(translation) else [0.0, 0.0, 0.0]
        n = [int(v) for v in npoints]
        st = [float(v) for v in step]
        st = [st[a] if n[a] > 1 else 0.0 for a in range(3)]
        start = [float(v) for v in start]
        stop = [start[a] + (n[a] - 1) * st[a] for a in range(3)]
        v = np.asarray(values, dtype=np.float64).reshape(-1, 3)
        vals = np.array([rotate_xyz(list(x), r) for x in v])
        self._add_grid(n, start, st, stop, vals, r, t, frequency, frequency_phase, time_offset)

    def add_bfield_epu(self, period, nperiods, bfieldA=[], bfieldB=[], phase=0, rotations=[],
                       translation=[], taper=0, frequency=0, frequency_phase=0, time_offset=0, name=""):
        if len(bfieldA) == 0 and len(bfieldB) == 0:
            raise ValueError("Must define at least one of 'bfieldA', 'bfieldB'")
        r = _v3(rotations, "rotations") if len(rotations) else [0.0, 0.0, 0.0]
        t = _v3(translation, "translation") if len(translation) else [0.0, 0.0, 0.0]
        fa = rotate_xyz(_v3(bfieldA, "bfieldA") if len(bfieldA) else [0.0, 0.0, 0.0], r)
        fb = rotate_xyz(_v3(bfieldB, "bfieldB") if len(bfieldB) else [0.0, 0.0, 0.0], r)
        p = rotate_xyz(_v3(period, "period"), r)
        a = lambda v: np.array(v, dtype=np.float64)
        A, B, Pp, T = a(fa), a(fb), a(p), a(t)
        self._check(self._lib.orc_add_epu(self._h, _dp(A), _dp(B), _dp(Pp), int(nperiods), _dp(T),
                                          float(phase), float(taper), float(frequency),
                                          float(frequency_phase), float(time_offset)))

    def set_particle(self, x0, beta0, t0=0.0):
        """Use a particle of the beam's species with these initial conditions."""
        a = lambda v: np.ascontiguousarray(np.array(v, dtype=np.float64))
        self._check(self._lib.orc_set_particle(self._h, _dp(a(x0)), _dp(a(beta0)), float(t0)))

    def get_bfield(self, x, t=0):
        X = np.array(_v3(x), dtype=np.float64)
        out = np.zeros(3)
        self._lib.orc_get_bfield(self._h, _dp(X), float(t), _dp(out))
        return list(out)

    def clear_particle_beams(self):
        self._beam_names = []

    def set_particle_beam(self, **kw):
        self._beam_names = []
        self.add_particle_beam(_append=0, **kw)

    def add_particle_beam(self, type="electron", name="", energy_GeV=-1, d0=None, x0=None, beam="",
                          sigma_energy_GeV=0, t0=0, current=0, weight=1, rotations=None,
                          translation=None, horizontal_direction=None, beta=None, alpha=None,
                          gamma=None, emittance=None, eta=None, lattice_reference=None, mass=0,
                          charge=0, ctstartstop=None, distribution="", _append=1):
        """OSCARSSR_AddParticleBeam (src/OSCARSSR_Python.cc:3699-4100)."""
        names = getattr(self, "_beam_names", [])
        if not _append:
            names = []
        predefined = 0
        if beam:
            predefined = {"NSLSII": 1, "NSLS2": 1, "NSLS-II": 1, "NSLSII-LONGSTRAIGHT": 2, "NSLS2-LONGSTRAIGHT": 2,
                          "NSLS-II-LONGSTRAIGHT": 2, "NSLSII-SHORTSTRAIGHT": 3, "NSLS2-SHORTSTRAIGHT": 3,
                          "NSLS-II-SHORTSTRAIGHT": 3}.get(beam.upper(), 0)
            if not predefined:
                raise ValueError("Error in predefined beam name / definition")
        elif type not in _PARTICLE_TYPES:
            raise ValueError("invalid argument in adding particle beam.  possibly 'name' already exists")
        my_name = name if name else "_beam%d" % len(names)
        if my_name in names:
            raise ValueError("invalid argument in adding particle beam.  possibly 'name' already exists")
        d = _v3(d0, "d0") if d0 is not None else [0.0, 0.0, 1.0]
        x = _v3(x0, "x0") if x0 is not None else [0.0, 0.0, 0.0]
        r = _v3(rotations, "rotations") if rotations is not None else [0.0, 0.0, 0.0]
        tr = _v3(translation, "translation") if translation is not None else [0.0, 0.0, 0.0]
        if horizontal_direction is not None:
            hd = _v3(horizontal_direction, "horizontal_direction")
        else:  # -Direction.Orthogonal() of the un-rotated direction (Python.cc:3912-3915)
            ax, ay, az = [abs(v) if v < 0 else v for v in d]
            if ax < ay:
                o = [0.0, d[2], -d[1]] if ax < az else [d[1], -d[0], 0.0]
            else:
                o = [-d[2], 0.0, d[0]] if ay < az else [d[1], -d[0], 0.0]
            hd = [-o[0], -o[1], -o[2]]
        x = rotate_xyz(x, r)
        d = rotate_xyz(d, r)
        x = [x[0] + tr[0], x[1] + tr[1], x[2] + tr[2]]
        a = lambda v: np.array(v, dtype=np.float64)
        X, Dd, H = a(x), a(d), a(hd)
        em = a(emittance if emittance is not None else [0, 0])
        bt = a(beta if beta is not None else [0, 0])
        al = a(alpha if alpha is not None else [0, 0])
        gm = a(gamma if gamma is not None else [0, 0])
        et = a(eta if eta is not None else [0, 0])
        lr = a(lattice_reference if lattice_reference is not None else [0, 0, 0])
        cs = a(ctstartstop if ctstartstop is not None else [0, 0])
        dist = {"": -1, "filament": 1, "gaussian": 2, "kv": 3}[distribution.lower()]
        self._check(self._lib.orc_set_beam(
            self._h, _PARTICLE_TYPES.get(type, 0), float(charge), float(mass), float(energy_GeV), _dp(X),
            _dp(Dd), float(t0), float(current), _dp(H), 1, float(sigma_energy_GeV), _dp(em),
            int(emittance is not None), _dp(bt), _dp(al), int(beta is not None),
            int(alpha is not None), _dp(et), dist, _dp(cs), int(ctstartstop is not None), _dp(gm),
            int(gamma is not None), _dp(lr), int(lattice_reference is not None), predefined, int(d0 is not None),
            float(weight), int(_append)))
        self._beam_names = names + [my_name]

    def set_ctstartstop(self, start, stop):
        self._lib.orc_set_ctstartstop(self._h, float(start), float(stop))

    def set_npoints_trajectory(self, n):
        self._lib.orc_set_npoints_trajectory(self._h, int(n))

    def get_npoints_trajectory(self):
        return self._lib.orc_get_npoints_trajectory(self._h)

    def set_new_particle(self, beam="", particle=""):
        names = getattr(self, "_beam_names", [])
        if beam and beam not in names:
            raise ValueError("beam name not in map")
        self._check(self._lib.orc_set_new_particle_of(self._h, names.index(beam) if beam else -1,
                                                      int(particle.lower() == "ideal")))

    def get_particle(self):
        vals = [np.zeros(3), np.zeros(3)] + [np.zeros(1) for _ in range(5)]
        self._lib.orc_get_particle(self._h, *[_dp(v) for v in vals])
        return vals

    def uniform(self):
        return self._lib.orc_uniform(self._h)

    def normal(self):
        return self._lib.orc_normal(self._h)

    # ---- trajectory -------------------------------------------------------------------------
    def calculate_trajectory(self, ofile="", bofile="", oformat=""):
        self._check(self._lib.orc_calculate_trajectory(self._h))
        return self.get_trajectory()

    def trajectory_array(self):
        """(10, n) SoA: t, x, y, z, bx, by, bz, ax, ay, az."""
        n = self._lib.orc_trajectory_npoints(self._h)
        out = np.zeros(10 * n)
        self._lib.orc_get_trajectory(self._h, _dp(out), out.size)
        return out.reshape(10, n)

    def spline_ypp(self):
        n = self._lib.orc_trajectory_npoints(self._h)
        out = np.zeros(9 * n)
        self._lib.orc_get_spline_ypp(self._h, _dp(out), out.size)
        return out.reshape(9, n)

    def level_samples(self, level):
        out = np.zeros(10 * (1 << level))
        self._check(self._lib.orc_get_level(self._h, int(level), _dp(out), out.size))
        return out.reshape(10, 1 << level)

    def get_trajectory(self):
        a = self.trajectory_array()
        return [[a[0, i], list(a[1:4, i]), list(a[4:7, i]), list(a[7:10, i])] for i in range(a.shape[1])]

    # ---- radiation --------------------------------------------------------------------------
    def _pol_args(self, polarization, angle, horizontal_direction, propogation_direction):
        code = polarization_code(polarization, angle)
        h = np.array(_v3(horizontal_direction) if horizontal_direction else [1.0, 0.0, 0.0])
        p = np.array(_v3(propogation_direction) if propogation_direction else [0.0, 0.0, 1.0])
        return code, float(angle), h, p

    def calculate_spectrum(self, obs, npoints=0, energy_range_eV=None, energy_points_eV=None,
                           points_eV=None, polarization="", angle=_ANGLE_UNSET,
                           horizontal_direction=None, propogation_direction=None, precision=0.01,
                           max_level=-2, max_level_extended=0, nparticles=0, nthreads=0, gpu=-1,
                           ngpu=None, quantity="flux", ofile="", bofile=""):
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        if points_eV is not None:
            energy_points_eV = points_eV
        E = spectrum_energies(npoints, energy_range_eV, energy_points_eV)
        O = np.array(_v3(obs, "obs"))
        q = _quantity(quantity)
        code, ang, h, p = self._pol_args(polarization, angle, horizontal_direction, propogation_direction)
        out = np.zeros(E.size)
        lv = np.zeros(E.size, dtype=np.int32)
        self._check(self._lib.orc_spectrum(self._h, _dp(O), _dp(E), E.size, code, ang, _dp(h), _dp(p),
                                           float(precision), int(max_level), int(max_level_extended),
                                           int(nparticles), q, _dp(out),
                                           lv.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self.last_levels = lv
        return [[float(E[i]), float(out[i])] for i in range(E.size)]

    def _surface(self, npoints, plane, width, x0x1x2, rotations, translation, normal, pd):
        if len(npoints) != 2:
            raise ValueError("'npoints' must be [int, int]")
        nx1, nx2 = int(npoints[0]), int(npoints[1])
        if nx1 <= 0 or nx2 <= 0:
            raise ValueError("an entry in 'npoints' is <= 0")
        r = _v3(rotations) if rotations else [0.0, 0.0, 0.0]
        t = _v3(translation) if translation else [0.0, 0.0, 0.0]
        w1, w2 = (0.010, 0.010) if pd else (0.0, 0.0)
        if width is not None and len(width) == 2:
            w1, w2 = float(width[0]), float(width[1])
        if abs(normal) > 1:
            raise ValueError("'normal' must be -1, 0, or 1")
        if x0x1x2 is not None:
            if len(x0x1x2) != 3:
                raise ValueError("'x0x1x2' must have 3 XYZ points defined correctly")
            return rectangle_x0x1x2(nx1, nx2, x0x1x2[0], x0x1x2[1], x0x1x2[2], r, t, normal)
        if pd and (w1 <= 0 or w2 <= 0):
            raise ValueError("'width' must be > 0")
        return rectangle(plane, nx1, nx2, w1, w2, r, t, normal)

    def calculate_flux_rectangle(self, energy_eV, npoints=[51, 51], plane="XY", normal=0, dim=2,
                                 width=None, rotations=None, translation=None, x0x1x2=None,
                                 polarization="", angle=_ANGLE_UNSET, horizontal_direction=None,
                                 propogation_direction=None, nparticles=0, nthreads=0, gpu=-1,
                                 ngpu=None, precision=0.01, max_level=-2, max_level_extended=0,
                                 quantity="flux", ofile="", bofile=""):
        if dim not in (2, 3):
            raise ValueError("'dim' must be 2 or 3")
        xyz, normals, x1x2 = self._surface(npoints, plane, width, x0x1x2, rotations, translation, normal, False)
        q = _quantity(quantity)
        code, ang, h, p = self._pol_args(polarization, angle, horizontal_direction, propogation_direction)
        n = xyz.shape[0]
        out = np.zeros(n)
        lv = np.zeros(n, dtype=np.int32)
        X = np.ascontiguousarray(xyz)
        self._check(self._lib.orc_flux(self._h, _dp(X), n, float(energy_eV), code, ang, _dp(h), _dp(p),
                                       float(precision), int(max_level), int(max_level_extended),
                                       int(nparticles), q, _dp(out),
                                       lv.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self.last_levels = lv
        pos = xyz if dim == 3 else x1x2
        return [[list(pos[i]), float(out[i])] for i in range(n)]

    def calculate_power_density_rectangle(self, npoints=[51, 51], plane="XY", width=None,
                                          x0x1x2=None, rotations=None, translation=None, ofile="",
                                          bofile="", normal=0, nparticles=0, gpu=-1, ngpu=None,
                                          nthreads=0, precision=0.01, max_level=-2,
                                          max_level_extended=0, dim=2, quantity="power density"):
        if dim not in (2, 3):
            raise ValueError("'dim' must be 2 or 3")
        xyz, normals, x1x2 = self._surface(npoints, plane, width, x0x1x2, rotations, translation, normal, True)
        q = _quantity(quantity, pd=True)
        n = xyz.shape[0]
        out = np.zeros(n)
        lv = np.zeros(n, dtype=np.int32)
        X = np.ascontiguousarray(xyz)
        Nn = np.ascontiguousarray(normals)
        self._check(self._lib.orc_power_density(self._h, _dp(X), _dp(Nn), n, int(normal != 0),
                                                float(precision), int(max_level),
                                                int(max_level_extended), int(nparticles), q,
                                                _dp(out), lv.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self.last_levels = lv
        pos = xyz if dim == 3 else x1x2
        return [[list(pos[i]), float(out[i])] for i in range(n)]


    def set_trajectory_calculation(self, method, precision=-1):
        """OSCARSSR::SetTrajectoryCalculation (src/OSCARSSR.cc:784-820)."""
        m = method.upper()
        msg = "RK4 Trajectory does not use the precision parameter and you are attempting to set it"
        if m == "RK4":
            if precision != -1:
                raise ValueError(msg)
            code = 0
        elif m == "RKAS":
            if precision != -1 and precision <= 0:
                raise ValueError("Trajectory precision cannot be >= 0")
            code = 1
        else:
            raise ValueError("Method requested is invalid.  Try again")
        self._check(self._lib.orc_set_trajectory_calculation(self._h, code, float(precision)))

    # ---- STL surfaces (src/OSCARSSR_Python.cc:6852-7212, src/TSTLContainer.cc) ---------------------
    def add_stl(self, ifile, rotations=None, translation=None, scale=1, name=""):
        if not hasattr(self, "_stl"):
            self._stl = []
        t = _v3(translation, "translation") if translation is not None else [0.0, 0.0, 0.0]
        tri, cen = read_stl(ifile, float(scale), t)
        self._stl.append((name or "_stl%d" % len(self._stl), tri, cen))

    def calculate_power_density_stl(self, farfield_origin, ofile="", bofile="", stlofile="", nparticles=0, gpu=-1,
                                    ngpu=None, nthreads=0, precision=0.01, max_level=-2, max_level_extended=0,
                                    quantity="power density"):
        stl = getattr(self, "_stl", [])
        tri = np.ascontiguousarray(np.vstack([t for _, t, _ in stl]) if stl else np.zeros((0, 12)))
        cen = np.ascontiguousarray(np.vstack([c for _, _, c in stl]) if stl else np.zeros((0, 3)))
        q = _quantity(quantity, pd=True)
        n = tri.shape[0]
        out = np.zeros(n)
        lv = np.zeros(n, dtype=np.int32)
        self._check(self._lib.orc_power_density_stl(self._h, _dp(tri), _dp(cen), n, float(precision), int(max_level),
                                                    int(max_level_extended), int(nparticles), q, _dp(out),
                                                    lv.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self.last_levels = lv
        return [[[list(tri[i, 0:3]), list(tri[i, 3:6]), list(tri[i, 6:9])], float(out[i])] for i in range(n)]

    def _points_call(self, points, rotations, translation, invert):
        r = _v3(rotations) if rotations else [0.0, 0.0, 0.0]
        t = _v3(translation) if translation else [0.0, 0.0, 0.0]
        return surface_points(points, r, t, invert)

    def calculate_flux(self, energy_eV=0.0, points=[], normal=0, rotations=None, translation=None, nparticles=0,
                       nthreads=0, gpu=-1, ngpu=None, precision=0.01, max_level=-2, max_level_extended=0, ofile="",
                       bofile="", quantity="flux"):
        """Flux at arbitrary points, polarization 'all' (the reference binding of calculate_flux raises
        before computing; this is the flux its CalculateFlux would give)."""
        xyz, _ = self._points_call(points, rotations, translation, False)
        q = _quantity(quantity)
        n = xyz.shape[0]
        out = np.zeros(n)
        lv = np.zeros(n, dtype=np.int32)
        h, p = np.array([1.0, 0.0, 0.0]), np.array([0.0, 0.0, 1.0])
        self._check(self._lib.orc_flux(self._h, _dp(np.ascontiguousarray(xyz)), n, float(energy_eV), 0, 0.0, _dp(h), _dp(p),
                                       float(precision), int(max_level), int(max_level_extended), int(nparticles), q,
                                       _dp(out), lv.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self.last_levels = lv
        return [[list(xyz[i]), float(out[i])] for i in range(n)]

    def calculate_power_density(self, points, normal=0, rotations=None, translation=None, nparticles=0, gpu=-1,
                                ngpu=None, nthreads=0, precision=0.01, max_level=-2, max_level_extended=0,
                                quantity="power density", ofile="", bofile=""):
        """Power density at arbitrary points with normals (src/OSCARSSR_Python.cc:6105-6370)."""
        xyz, nrm = self._points_call(points, rotations, translation, normal == -1)
        q = _quantity(quantity, pd=True)
        n = xyz.shape[0]
        out = np.zeros(n)
        lv = np.zeros(n, dtype=np.int32)
        self._check(self._lib.orc_power_density(self._h, _dp(np.ascontiguousarray(xyz)), _dp(np.ascontiguousarray(nrm)), n,
                                                int(normal != 0), float(precision), int(max_level),
                                                int(max_level_extended), int(nparticles), q, _dp(out),
                                                lv.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self.last_levels = lv
        return [[list(xyz[i]), float(out[i])] for i in range(n)]


def reference_module():
    """Import the reference's own CPU build from oracle/_ref when it exists (None otherwise)."""
    ref = os.path.join(_HERE, "_ref")
    if not os.path.isdir(os.path.join(ref, "oscars")):
        return None
    if ref not in sys.path:
        sys.path.insert(0, ref)
    import importlib
    return importlib.import_module("oscars.sr")
