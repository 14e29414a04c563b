"""Batches of independent radiation jobs (``osc_batch_flux``).

A job is one undulator / EPU set-up -- its own fields, an ideal particle, a trajectory range and
point count, observers and photon energies.  The reference computes such a set one
``calculate_flux`` / ``calculate_spectrum`` call at a time; here ``compute='mixed'`` integrates all
jobs in shared launches (trajectories, splines and level samples on the device, persistent wave
kernels over every job's entries, the launches up to level 13 replayed from a CUDA graph once a
shape has been seen), while ``compute='fp64'`` runs them one after another through the FP64 path
of ``oscars_b200.sr`` (the reference's arithmetic).

    from oscars_b200.batch import Job, undulator, BatchRunner
    jobs = [Job(fields=[undulator(bfield=[0, 0.5, 0], period=[0, 0, 0.05], nperiods=41)],
                energy_GeV=3, ctstartstop=(-1.5, 1.5), npoints=20001,
                obs=[[0, 0, 30]], energies_eV=[458.9]), ...]
    runner = BatchRunner(gpu=0)
    results = runner.flux(jobs, compute='mixed')      # list of (n_obs, n_energies) arrays
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from . import _lib
from .sr import _PARTICLES, _ANGLE_UNSET, _compute_mode, _polarization

__all__ = ["Job", "undulator", "epu", "grid", "BatchRunner", "flux_batch"]


def undulator(bfield, period, nperiods, translation=(0, 0, 0), phase=0.0, taper=0.0, frequency=0.0,
              frequency_phase=0.0, time_offset=0.0, half_period_scale=None):
    """An ideal planar undulator, with the arguments of sr.add_bfield_undulator (optionally with
    2 * nperiods half-period amplitude factors)."""
    return dict(kind=0, bfield=list(bfield), bfield_b=[0, 0, 0], period=list(period), nperiods=int(nperiods),
                center=list(translation), phase=phase, taper=taper, frequency=frequency,
                frequency_phase=frequency_phase, time_offset=time_offset, half_period_scale=half_period_scale)


def grid(values, npoints, start, step, rotations=(0, 0, 0), translation=(0, 0, 0), frequency=0.0,
         frequency_phase=0.0, time_offset=0.0):
    """A regular-grid field, as sr.add_bfield_grid."""
    return dict(kind=2, values=np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(-1, 3)),
                npoints=[int(v) for v in npoints], start=list(start), step=list(step), rotations=list(rotations),
                center=list(translation), frequency=frequency, frequency_phase=frequency_phase,
                time_offset=time_offset)


def epu(bfield, bfield_b, period, nperiods, translation=(0, 0, 0), phase=0.0, taper=0.0):
    """An ideal elliptically polarizing undulator (fields A and B), as sr.add_bfield_epu."""
    return dict(kind=1, bfield=list(bfield), bfield_b=list(bfield_b), period=list(period), nperiods=int(nperiods),
                center=list(translation), phase=phase, taper=taper, frequency=0.0, frequency_phase=0.0,
                time_offset=0.0)


@dataclass
class Job:
    fields: list
    energy_GeV: float
    ctstartstop: Sequence[float]
    npoints: int
    obs: np.ndarray                     # (n_obs, 3) [m]
    energies_eV: np.ndarray             # (n_energies,)
    particle: str = "electron"
    x0: Sequence[float] = (0.0, 0.0, 0.0)
    d0: Sequence[float] = (0.0, 0.0, 1.0)
    ct0: float = 0.0
    current: float = 0.5
    spectrum: bool = False              # normalise like calculate_spectrum (|current|)
    charge: float = 0.0                 # custom particle only
    mass: float = 0.0


class BatchRunner:
    """Owns a context on one GPU; repeated calls with the same shape replay the captured graph."""

    def __init__(self, gpu: int = 0):
        self.ctx = _lib.Context(gpu)
        self.last_levels = None
        self.last_not_converged = 0

    @staticmethod
    def _descriptors(jobs, average=False):
        """Field and job descriptors of a batch, the concatenated observers and energies, and the
        arrays the descriptors point into (to keep alive until the call returns)."""
        fdescs, jdescs, obs_all, e_all = [], [], [], []
        keep = []  # arrays the descriptors point into, alive until the call returns
        n_obs = n_e = 0
        for jb in jobs:
            fb = len(fdescs)
            for f in jb.fields:
                d = _lib.FieldDesc()
                d.kind = f["kind"]
                d.center[:] = f["center"]
                d.frequency, d.frequency_phase, d.time_offset = f["frequency"], f["frequency_phase"], f["time_offset"]
                if f["kind"] == 2:
                    keep.append(f["values"])
                    d.grid_n[:] = f["npoints"]
                    d.grid_start[:] = f["start"]
                    d.grid_step[:] = f["step"]
                    d.grid_values = _lib.dptr(f["values"])
                    d.rotations[:] = f["rotations"]
                else:
                    d.bfield[:] = f["bfield"]
                    d.bfield_b[:] = f["bfield_b"]
                    d.period[:] = f["period"]
                    d.nperiods = f["nperiods"]
                    d.phase, d.taper = f["phase"], f["taper"]
                    if f.get("half_period_scale") is not None:
                        hs = np.ascontiguousarray(np.asarray(f["half_period_scale"], dtype=np.float64).ravel())
                        keep.append(hs)
                        d.half_period_scale = _lib.dptr(hs)
                        d.n_half_periods = int(hs.size)
                fdescs.append(d)
            o = np.ascontiguousarray(np.asarray(jb.obs, dtype=np.float64).reshape(-1, 3))
            e = np.ascontiguousarray(np.asarray(jb.energies_eV, dtype=np.float64).reshape(-1))
            jd = _lib.JobDesc()
            jd.field_begin, jd.field_count = fb, len(jb.fields)
            if jb.particle.lower() not in _PARTICLES:
                raise ValueError("unknown particle type %r" % jb.particle)
            jd.particle = _PARTICLES[jb.particle.lower()]
            jd.charge, jd.mass = jb.charge, jb.mass
            jd.energy_GeV = jb.energy_GeV
            jd.x0[:] = list(jb.x0)
            jd.d0[:] = list(jb.d0)
            jd.t0 = jb.ct0
            jd.current = jb.current
            jd.ctstart, jd.ctstop = jb.ctstartstop
            jd.npoints = int(jb.npoints)
            if average and obs_all:
                jd.obs_begin, jd.n_obs = 0, o.shape[0]
                jd.energy_begin, jd.n_energies = 0, e.shape[0]
            else:
                jd.obs_begin, jd.n_obs = n_obs, o.shape[0]
                jd.energy_begin, jd.n_energies = n_e, e.shape[0]
                obs_all.append(o)
                e_all.append(e)
                n_obs += o.shape[0]
                n_e += e.shape[0]
            jd.spectrum = 1 if jb.spectrum else 0
            jdescs.append(jd)
        obs = np.ascontiguousarray(np.concatenate(obs_all))
        en = np.ascontiguousarray(np.concatenate(e_all))
        return fdescs, jdescs, obs, en, keep

    def flux(self, jobs: List[Job], compute: str = "mixed", polarization: str = "all", angle=_ANGLE_UNSET,
             horizontal_direction=None, propogation_direction=None, precision: float = 0.01, max_level: int = -2,
             max_level_extended: int = 0, quantity: str = "flux", average: bool = False):
        """Flux (or spectrum) of every job; a list of (n_obs, n_energies) arrays, or one array with
        average=True (jobs sharing observers and energies, mean with weight 1/N)."""
        if not jobs:
            return []
        fdescs, jdescs, obs, en, keep = self._descriptors(jobs, average)
        opts = self._opts(polarization, angle, horizontal_direction, propogation_direction, precision, max_level,
                          max_level_extended, quantity, compute)
        sizes = [jd.n_obs * jd.n_energies for jd in jdescs]
        total = sizes[0] if average else int(sum(sizes))
        out = np.zeros(total)
        lvl = np.zeros(total, dtype=np.int32)
        nnc = _lib.LL(0)
        F = (_lib.FieldDesc * max(1, len(fdescs)))(*fdescs)
        J = (_lib.JobDesc * len(jdescs))(*jdescs)
        self.ctx.call("osc_batch_flux", F, len(fdescs), J, len(jdescs), _lib.dptr(obs), obs.shape[0], _lib.dptr(en),
                      en.shape[0], ctypes.byref(opts), 1 if average else 0, _lib.dptr(out), _lib.i32ptr(lvl),
                      ctypes.byref(nnc))
        self.last_not_converged = nnc.value
        if average:
            self.last_levels = lvl.reshape(jdescs[0].n_obs, jdescs[0].n_energies)
            return out.reshape(jdescs[0].n_obs, jdescs[0].n_energies)
        res, levels, k = [], [], 0
        for jd, m in zip(jdescs, sizes):
            res.append(out[k:k + m].reshape(jd.n_obs, jd.n_energies))
            levels.append(lvl[k:k + m].reshape(jd.n_obs, jd.n_energies))
            k += m
        self.last_levels = levels
        return res

    def trajectories(self, jobs: List[Job]):
        """The jobs' trajectories as the batched mixed path integrates them on the device (RK4 and
        spline kernels): per job a (19, n) array -- t [s]; x, y, z [m]; beta_x, beta_y, beta_z;
        a_x/c, a_y/c, a_z/c [1/s]; and the 9 spline second derivatives of those components."""
        if not jobs:
            return []
        fdescs, jdescs, _, _, keep = self._descriptors(jobs)
        cap = 0
        for jd in jdescs:  # upper bound of the point count: npoints + 2
            cap += 19 * (int(jd.npoints) + 2)
        out = np.zeros(cap)
        npts = np.zeros(len(jdescs), dtype=np.int64)
        F = (_lib.FieldDesc * max(1, len(fdescs)))(*fdescs)
        J = (_lib.JobDesc * len(jdescs))(*jdescs)
        self.ctx.call("osc_batch_trajectories", F, len(fdescs), J, len(jdescs), _lib.dptr(out), cap,
                      npts.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
        res, k = [], 0
        for n in npts:
            res.append(out[k:k + 19 * n].reshape(19, n).copy())
            k += 19 * n
        return res

    def stats(self):
        """(samples integrated, kernel launches) of the last call."""
        s, l = _lib.LL(0), _lib.LL(0)
        self.ctx.call("osc_last_stats", ctypes.byref(s), ctypes.byref(l))
        return s.value, l.value

    def set_variant(self, variant: int):
        """Force a compiled variant of the batched wave kernel (-1: autotune per shape)."""
        self.ctx.call("osc_set_variant", 3, int(variant))

    def variant(self):
        v, n = ctypes.c_int(0), ctypes.c_int(0)
        self.ctx.call("osc_get_variant", 3, ctypes.byref(v), ctypes.byref(n))
        return v.value, n.value

    @staticmethod
    def _opts(polarization, angle, horizontal_direction, propogation_direction, precision, max_level,
              max_level_extended, quantity, compute):
        o = _lib.RadOpts()
        o.polarization = _polarization(polarization, angle)
        o.angle = float(angle)
        o.horizontal[:] = list(horizontal_direction) if horizontal_direction is not None else [1, 0, 0]
        o.propagation[:] = list(propogation_direction) if propogation_direction is not None else [0, 0, 1]
        o.precision = precision
        o.max_level = max_level
        o.max_level_extended = max_level_extended
        o.nparticles = 0
        q = {"flux": 0, "precision": 1, "level": 2}
        if quantity not in q:
            raise ValueError("'quantity' must be: 'flux', 'precision', 'level', or blank")
        o.quantity = q[quantity]
        o.precision_mode = _compute_mode(compute)
        return o


def flux_batch(jobs: List[Job], compute: str = "mixed", gpu: int = 0, **kw):
    """One-shot helper: BatchRunner(gpu).flux(jobs, compute, **kw)."""
    return BatchRunner(gpu).flux(jobs, compute=compute, **kw)
