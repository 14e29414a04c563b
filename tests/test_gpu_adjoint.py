"""Gradients with respect to per-half-period undulator amplitudes (osc_flux_vjp, osc_trajectory_vjp).

Configuration (tests/golden/cases.py adjoint_config): 41-period undulator with the 82 factors of
tests/golden/fields/halfscale_41.txt, 5 x 5 observers over 1 mm at z = 30 m, 8 energies over E1 +- 5 %,
fixed level 10; loss = sum (F(s) - F(1))^2.  Tolerance 1e-3 relative to the largest component.

Finite-difference step: the retarded phase is ~7e10 rad here and FP64 rounds it to ~1e-5 rad (in the
reference exactly as here), which is the size of the phase change a step of 1e-6 in a factor causes;
central differences of the flux loss with h = 1e-6 are therefore rounding noise at the 20 % level
(measured: 0.22 at 1e-6, 3e-2 at 1e-5, 7e-4 at 3e-4, 4e-4 at 1e-3).  The flux-loss checks use the
Richardson extrapolation of steps 1e-3 and 3e-3; the trajectory part, which has no phase, is checked
with h = 1e-6 directly.  The mixed-precision adjoint (compute='mixed') is checked against the FP64
adjoint and against the reference's differences; its flux against FP64 at 1e-4 of the peak.
"""
import os

import numpy as np
import pytest

from cases import adjoint_config, halfscale_41, richardson

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-3


def _problem(compute="fp64"):
    from oscars_b200.tuning import TuningProblem
    obs, energies, level = adjoint_config()
    return TuningProblem(bfield=[0, 0.5, 0], period=[0, 0, 0.05], nperiods=41, obs=obs, energies_eV=energies,
                         level=level, compute=compute)


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(b)))


def _host_knots(s):
    from oscars_b200.sr import sr
    o = sr(device=-1)
    o.add_bfield_undulator(bfield=[0, 0.5, 0], period=[0, 0, 0.05], nperiods=41, phase=-np.pi / 2,
                           half_period_scale=s)
    o.set_particle_beam(type="electron", energy_GeV=3, x0=[0, 0, 0], d0=[0, 0, 1], current=0.5)
    o.set_ctstartstop(-1.5, 1.5)
    o.set_npoints_trajectory(20001)
    o.calculate_trajectory()
    return o.trajectory_array()[1:]


def test_forward_matches_reference():
    g = np.load(os.path.join(GOLDEN, "adjoint_fd.npz"))
    p = _problem()
    assert _rel(p.flux(np.ones(82)), g["F1"]) <= 1e-9
    assert _rel(p.flux(g["s"]), g["F"]) <= 1e-9


def test_trajectory_vjp_matches_central_differences():
    """h = 1e-6 on the trajectory knots themselves (host RK4, bit-exact with the reference)."""
    p = _problem()
    s0 = np.array(halfscale_41())
    n = p.npoints()
    rng = np.random.default_rng(3)
    kg = rng.standard_normal((9, n)) * np.array([1, 1, 1, 1e-3, 1e-3, 1e-3, 1e-6, 1e-6, 1e-6])[:, None]
    g = p.trajectory_vjp(s0, kg)
    fd = np.zeros(82)
    for k in range(82):
        e = np.zeros(82)
        e[k] = 1e-6
        fd[k] = (np.sum(kg * _host_knots(s0 + e)) - np.sum(kg * _host_knots(s0 - e))) / 2e-6
    err = _rel(g, fd)
    print("trajectory adjoint vs central differences (h=1e-6): %.3e" % err)
    assert err <= 1e-5


def test_adjoint_matches_reference_finite_differences():
    g = np.load(os.path.join(GOLDEN, "adjoint_fd.npz"))
    h = list(g["h"])
    ref = richardson(g["grad_h%d" % h.index(1e-3)], g["grad_h%d" % h.index(3e-3)], 3.0)
    p = _problem()
    F1 = p.flux(np.ones(82))
    F, grad = p.vjp(g["s"], 2 * (p.flux(g["s"]) - F1))
    assert _rel(F, g["F"]) <= 1e-9
    e = _rel(grad, ref)
    print("adjoint vs reference differences (Richardson 1e-3/3e-3): %.3e; raw h=1e-6: %.3e"
          % (e, _rel(grad, g["grad_h%d" % h.index(1e-6)])))
    assert e <= TOL


def test_adjoint_matches_own_finite_differences():
    p = _problem()
    s0 = np.array(halfscale_41())
    F1 = p.flux(np.ones(82))

    def loss(s):
        return float(np.sum((p.flux(s) - F1) ** 2))

    def central(h):
        fd = np.zeros(82)
        for k in range(82):
            e = np.zeros(82)
            e[k] = h
            fd[k] = (loss(s0 + e) - loss(s0 - e)) / (2 * h)
        return fd
    _, grad = p.vjp(s0, 2 * (p.flux(s0) - F1))
    err = _rel(grad, richardson(central(1e-3), central(3e-3), 3.0))
    print("adjoint vs own differences (Richardson 1e-3/3e-3): %.3e" % err)
    assert err <= TOL


def test_torch_autograd_and_a_descent_step():
    import torch
    from oscars_b200.tuning import UndulatorFlux
    p = _problem()
    F1 = torch.as_tensor(p.flux(np.ones(82)))
    s = torch.tensor(halfscale_41(), dtype=torch.float64, requires_grad=True)
    loss = ((UndulatorFlux.apply(s, p) - F1) ** 2).sum()
    loss.backward()
    _, direct = p.vjp(s.detach().numpy(), 2 * (p.flux(s.detach().numpy()) - F1.numpy()))
    assert np.allclose(s.grad.numpy(), direct, rtol=1e-12, atol=0)
    with torch.no_grad():
        step = 1e-3 / float(s.grad.abs().max())
        loss2 = ((UndulatorFlux.apply(s - step * s.grad, p) - F1) ** 2).sum()
    assert float(loss2) < float(loss.detach())


def test_mixed_adjoint_against_fp64_and_reference():
    g = np.load(os.path.join(GOLDEN, "adjoint_fd.npz"))
    h = list(g["h"])
    ref = richardson(g["grad_h%d" % h.index(1e-3)], g["grad_h%d" % h.index(3e-3)], 3.0)
    p64, pmx = _problem(), _problem("mixed")
    F1, F1m = p64.flux(np.ones(82)), pmx.flux(np.ones(82))
    assert _rel(F1m, F1) <= 1e-4
    F, grad = p64.vjp(g["s"], 2 * (p64.flux(g["s"]) - F1))
    Fm, gradm = pmx.vjp(g["s"], 2 * (pmx.flux(g["s"]) - F1m))
    assert _rel(Fm, F) <= 1e-4
    e64, eref = _rel(gradm, grad), _rel(gradm, ref)
    print("mixed adjoint vs FP64 adjoint: %.3e; vs reference differences (Richardson): %.3e" % (e64, eref))
    assert e64 <= TOL
    assert eref <= TOL


@pytest.mark.parametrize("compute", ["fp64", "mixed"])
def test_forward_sums_are_reused_only_for_the_same_inputs(compute):
    """flux(s) keeps the entry sums; vjp at the same s reuses them and must equal a vjp computed from
    scratch; after flux at other factors, vjp at s must recompute."""
    g = np.load(os.path.join(GOLDEN, "adjoint_fd.npz"))
    s0 = g["s"]
    rng = np.random.default_rng(5)
    gf = rng.standard_normal(_problem().shape)
    fresh = _problem(compute)
    F_a, grad_a = fresh.vjp(s0, gf)
    p = _problem(compute)
    F_b = p.flux(s0)
    F_c, grad_c = p.vjp(s0, gf)
    assert np.array_equal(F_b, F_a) and np.array_equal(F_c, F_a)
    assert _rel(grad_c, grad_a) <= 1e-10  # the per-sample sums are folded with atomics (order varies)
    p.flux(np.ones(82))
    F_d, grad_d = p.vjp(s0, gf)
    assert np.array_equal(F_d, F_a) and _rel(grad_d, grad_a) <= 1e-10
