"""Differentiable undulator tuning: flux as a function of per-half-period amplitude factors.

The field is an ideal planar undulator whose full-strength region (the 2 * nperiods half-periods
between the end poles) has one amplitude factor s_k per half-period (``add_bfield_undulator(...,
half_period_scale=s)``).  ``UndulatorFlux.apply(s, problem)`` returns the fixed-level flux of every
(observer, energy) entry as a torch tensor; its backward pass is the hand-written adjoint
(``osc_flux_vjp``: reverse mode through the radiation sum, the trajectory spline and the RK4 steps).
``compute='mixed'`` runs the radiation part in mixed precision (the mixed path's sums, an FP32
reverse sweep with the FP64 phase of each pair of samples), ``'fp64'`` in FP64; the RK4 part is FP64,
recomputes the trajectory from checkpoints every 256 steps and runs parallel in time over 64-step
segments joined by a sweep of their 6 x 6 Jacobians.  The forward pass keeps the entry sums, which
the backward pass on the same factors reuses.  PyTorch only carries the tensors.

    problem = TuningProblem(bfield=[0, 0.5, 0], period=[0, 0, 0.05], nperiods=41,
                            obs=obs_xyz, energies_eV=E, level=12, compute='mixed')
    s = torch.ones(82, dtype=torch.float64, requires_grad=True)
    F = UndulatorFlux.apply(s, problem)          # (n_obs, n_energies)
    loss = ((F - F_ideal) ** 2).sum(); loss.backward()   # s.grad
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from .sr import sr

__all__ = ["TuningProblem", "UndulatorFlux"]


class TuningProblem:
    """One undulator (with half-period factors), a 3 GeV-style beam and a fixed observation set."""

    def __init__(self, bfield, period, nperiods, obs, energies_eV, level=12, phase=-math.pi / 2,
                 beam=None, ctstartstop=(-1.5, 1.5), npoints=20001, spectrum=False, gpu=0, compute="fp64"):
        if compute not in ("fp64", "mixed"):
            raise ValueError("compute must be 'fp64' or 'mixed'")
        self.nperiods = int(nperiods)
        self.n_half = 2 * self.nperiods
        self.obs = np.ascontiguousarray(np.asarray(obs, dtype=np.float64).reshape(-1, 3))
        self.energies = np.ascontiguousarray(np.asarray(energies_eV, dtype=np.float64).reshape(-1))
        self.level = int(level)
        self.spectrum = bool(spectrum)
        self.sr = sr(gpu=1, device=gpu)
        self.sr.add_bfield_undulator(bfield=bfield, period=period, nperiods=nperiods, phase=phase,
                                     half_period_scale=np.ones(self.n_half))
        self.sr.set_particle_beam(**(beam or dict(type="electron", energy_GeV=3, x0=[0, 0, 0], d0=[0, 0, 1],
                                                  current=0.5)))
        self.sr.set_ctstartstop(*ctstartstop)
        self.sr.set_npoints_trajectory(npoints)
        self.compute = compute
        self._opts = self.sr._opts("", _lib_angle_unset(), None, None, 0.0, self.level, 0, 0, 0, compute)

    @property
    def shape(self):
        return (self.obs.shape[0], self.energies.shape[0])

    def set_scale(self, s):
        s = np.ascontiguousarray(np.asarray(s, dtype=np.float64).reshape(-1))
        if s.size != self.n_half:
            raise ValueError("expected %d half-period factors" % self.n_half)
        self.sr._ctx.call("osc_set_half_period_scale", -1, _lib.dptr(s), s.size)

    def flux(self, s):
        """Fixed-level flux for factors s, shape (n_obs, n_energies) (the forward pass of osc_flux_vjp,
        whose entry sums a following vjp at the same factors reuses)."""
        self.set_scale(s)
        n_o, n_e = self.shape
        out = np.zeros(n_o * n_e)
        self.sr._ctx.call("osc_flux_vjp", _lib.dptr(self.obs), n_o, _lib.dptr(self.energies), n_e, self.level,
                          ctypes.byref(self._opts), 1 if self.spectrum else 0, None, _lib.dptr(out), None, self.n_half,
                          None)
        return out.reshape(n_o, n_e)

    def vjp(self, s, grad_flux, knots=False):
        """(flux, (dF/ds)^T grad_flux) at factors s; with knots=True also the gradient with respect to
        the trajectory knots (9 x n_points)."""
        self.set_scale(s)
        n_o, n_e = self.shape
        g = np.ascontiguousarray(np.asarray(grad_flux, dtype=np.float64).reshape(-1))
        if g.size != n_o * n_e:
            raise ValueError("grad_flux must have n_obs * n_energies entries")
        out = np.zeros(n_o * n_e)
        gs = np.zeros(self.n_half)
        gk = np.zeros((9, self.npoints())) if knots else None
        self.sr._ctx.call("osc_flux_vjp", _lib.dptr(self.obs), n_o, _lib.dptr(self.energies), n_e, self.level,
                          ctypes.byref(self._opts), 1 if self.spectrum else 0, _lib.dptr(g), _lib.dptr(out),
                          _lib.dptr(gs), self.n_half, _lib.dptr(gk) if knots else None)
        if knots:
            return out.reshape(n_o, n_e), gs, gk
        return out.reshape(n_o, n_e), gs

    def npoints(self):
        """Points of the current trajectory."""
        self.sr.calculate_trajectory()
        return self.sr.trajectory_array().shape[1]

    def trajectory_vjp(self, s, knot_grad):
        """Gradient of sum(knot_grad * knots) with respect to the factors (knots: 9 x n_points)."""
        self.set_scale(s)
        kg = np.ascontiguousarray(np.asarray(knot_grad, dtype=np.float64))
        gs = np.zeros(self.n_half)
        self.sr._ctx.call("osc_trajectory_vjp", _lib.dptr(kg), kg.shape[1], _lib.dptr(gs), self.n_half)
        return gs


def _lib_angle_unset():
    from .sr import _ANGLE_UNSET
    return _ANGLE_UNSET


def _autograd_function():
    import torch

    class UndulatorFlux(torch.autograd.Function):
        """Flux (n_obs, n_energies) of a TuningProblem as a function of its half-period factors."""

        @staticmethod
        def forward(ctx, s, problem):
            sv = s.detach().to("cpu", torch.float64).numpy()
            F = problem.flux(sv)
            ctx.problem = problem
            ctx.save_for_backward(s.detach().clone())
            return torch.as_tensor(F, dtype=torch.float64, device=s.device)

        @staticmethod
        def backward(ctx, grad_F):
            (s,) = ctx.saved_tensors
            _, gs = ctx.problem.vjp(s.to("cpu", torch.float64).numpy(),
                                    grad_F.detach().to("cpu", torch.float64).numpy())
            return torch.as_tensor(gs, dtype=s.dtype, device=s.device), None

    return UndulatorFlux


class _Lazy:
    """Defers importing torch until the function is used."""
    _cls = None

    def __getattr__(self, name):
        if _Lazy._cls is None:
            _Lazy._cls = _autograd_function()
        return getattr(_Lazy._cls, name)


UndulatorFlux = _Lazy()
