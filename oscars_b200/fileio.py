"""Output files in the reference's formats (byte for byte).

* Points with a value (flux, power density: T3DScalarContainer::WriteToFileText / WriteToFileBinary,
  src/T3DScalarContainer.cc:396-470): text lines ``x1 x2 v`` (dim 2) or ``x y z v`` (dim 3) in
  ``std::scientific`` with its default precision (``%e``); binary float32 records of the same
  columns.
* Spectra (TSpectrumContainer::WriteToFileText / WriteToFileBinary, src/TSpectrumContainer.cc:282-353):
  text lines ``energy flux`` (``%e``); binary float32 pairs.
* Trajectories (TParticleTrajectoryPoints::WriteToFile / WriteToFileBinary,
  src/TParticleTrajectoryPoints.cc:259-470): text with a ``# <format>`` header and columns in
  ``%.35e``; binary with an int32 length and the upper-case format string, then float64 columns.  The
  default format is ``T X Y Z BX BY BZ BPX BPY BPZ`` (BP = a/c); a format names any of those columns.
"""
from __future__ import annotations

import struct

import numpy as np

TRAJECTORY_FORMAT = "T X Y Z BX BY BZ BPX BPY BPZ"
_COLUMNS = {"T": 0, "X": 1, "Y": 2, "Z": 3, "BX": 4, "BY": 5, "BZ": 6, "BPX": 7, "BPY": 8, "BPZ": 9}


def _open(path, mode):
    try:
        return open(path, mode)
    except OSError:
        raise ValueError("cannot open output file")


def write_points_text(path, pos, val, dim):
    """pos: (n, 3) positions as the call returns them (x1, x2, 0 for dim 2), val: (n,) values."""
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    val = np.asarray(val, dtype=np.float64).ravel()
    if dim not in (2, 3):
        raise ValueError("incorrect dimensions")
    with _open(path, "w") as f:
        if dim == 2:
            f.writelines("%e %e %e\n" % (p[0], p[1], v) for p, v in zip(pos.tolist(), val.tolist()))
        else:
            f.writelines("%e %e %e %e\n" % (p[0], p[1], p[2], v) for p, v in zip(pos.tolist(), val.tolist()))


def write_points_binary(path, pos, val, dim):
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    val = np.asarray(val, dtype=np.float64).ravel()
    if dim not in (2, 3):
        raise ValueError("incorrect dimensions")
    cols = [pos[:, 0], pos[:, 1]] + ([pos[:, 2]] if dim == 3 else []) + [val]
    with _open(path, "wb") as f:
        f.write(np.column_stack(cols).astype("<f4").tobytes())


def write_spectrum_text(path, energies, flux):
    with _open(path, "w") as f:
        f.writelines("%e %e\n" % (e, v) for e, v in zip(np.asarray(energies, dtype=np.float64).tolist(),
                                                          np.asarray(flux, dtype=np.float64).tolist()))


def write_spectrum_binary(path, energies, flux):
    with _open(path, "wb") as f:
        f.write(np.column_stack([np.asarray(energies, dtype=np.float64),
                                 np.asarray(flux, dtype=np.float64)]).astype("<f4").tobytes())


def _trajectory_columns(fmt):
    words = fmt.upper().split()
    if not words:
        raise ValueError("Format must contain at least one element")
    for w in words:
        if w not in _COLUMNS:
            raise ValueError("format specifier not recognized")
    return [_COLUMNS[w] for w in words]


def write_trajectory_text(path, traj, fmt=""):
    """traj: (10, n) -- t, x, y, z, beta_x, beta_y, beta_z, a_x/c, a_y/c, a_z/c."""
    traj = np.asarray(traj, dtype=np.float64)
    header = fmt if fmt else TRAJECTORY_FORMAT
    cols = _trajectory_columns(fmt if fmt else TRAJECTORY_FORMAT)
    rows = traj[cols].T.tolist()
    with _open(path, "w") as f:
        f.write("# %s\n" % header)
        f.writelines(" ".join("%.35e" % v for v in r) + "\n" for r in rows)


def write_trajectory_binary(path, traj, fmt=""):
    traj = np.asarray(traj, dtype=np.float64)
    form = fmt.upper() if fmt else TRAJECTORY_FORMAT
    cols = _trajectory_columns(form)
    with _open(path, "wb") as f:
        f.write(struct.pack("<i", len(form)) + form.encode())
        f.write(np.ascontiguousarray(traj[cols].T).astype("<f8").tobytes())
