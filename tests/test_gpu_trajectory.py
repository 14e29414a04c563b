"""Device trajectories of the batched path against the host's.

The batched mixed path integrates every job's RK4 trajectory (k_batch_rk4) and clamped spline
(k_batch_spline) on the GPU; everything downstream of it (level samples, pair records, the flux) is
tested only through the flux elsewhere.  Here the device knots are read back through
osc_batch_trajectories and compared with the host trajectory, which follows the reference
(src/OSCARSSR.cc:910-1009, include/TOMATH.h:141-203) bit for bit -- the CPU oracle, pinned to the
reference build, gives it.  The device uses CUDA's sin / cos in the field evaluation, so the two
agree to rounding, not bit for bit.

Bounds.  The knot times are equal.  Per component c of the 9 value rows (x, y, z, beta, a/c):
max_i |dev_ci - host_ci| / max_i |host_ci| <= 1e-11.  The spline second derivatives are the solution
of a diagonally dominant tridiagonal system (diagonal 2, off-diagonals <= 1/2, inverse norm <= 1)
whose right side is 6 x the second divided differences of the values, so a difference d_c in a
component's values moves its second derivatives by at most 24 d_c / h^2 (h the knot spacing); with
both builds' own rounding of that right side, each second-derivative row is bounded by
24 (d_c + 8 eps max|y_c|) / h^2.  (z'' in particular is ulp-level differences of a nearly linear z
divided by h^2 -- rounding noise in both builds.)  What the sample sums use is the spline's value
between knots: at every interval midpoint (where the finest level samples lie) all 9 interpolated
components agree to <= 1e-11 of their peak.
"""
import math

import numpy as np
import pytest

from cases import E1_EPU, field_file, halfscale_41

pytestmark = pytest.mark.gpu
TOL = 1e-11
ROWS = ["t", "x", "y", "z", "bx", "by", "bz", "ax", "ay", "az"] + ["d2_" + r for r in ("x", "y", "z", "bx", "by", "bz",
                                                                                     "ax", "ay", "az")]


def _oracle_knots(fields, energy, x0, d0, ct, npoints):
    from oracle.oracle import OracleSR
    o = OracleSR()
    for kind, kw in fields:
        getattr(o, kind)(**kw)
    o.set_particle_beam(type="electron", energy_GeV=energy, x0=list(x0), d0=list(d0), current=0.5)
    o.set_ctstartstop(*ct)
    o.set_npoints_trajectory(npoints)
    o.calculate_trajectory()
    return np.vstack([o.trajectory_array(), o.spline_ypp()])


def _grid1d():
    from oracle.oracle import read_oscars1d_grid
    return read_oscars1d_grid(field_file("und1d.txt"), "OSCARS1D Z By Bx", [0.0, 0.0, 0.0], [1, 1.02, 1])


def _grid3d():
    from oracle.oracle import read_oscars_grid
    return read_oscars_grid(field_file("grid3d.txt"), [0.0, 0.0, 0.0], [1, 1, 1, 1, 1.1, 1])


def _cases():
    """(name, batch fields, oracle field calls, energy, x0, d0, ctstartstop, npoints)."""
    from oscars_b200.batch import epu, grid, undulator
    pi2 = -math.pi / 2
    und = dict(bfield=[0, 0.5, 0], period=[0, 0, 0.05], nperiods=41, phase=pi2)
    ey = dict(bfield=[0, 0.6, 0], period=[0, 0, 0.057], nperiods=30, phase=pi2)
    ex = dict(bfield=[0.4, 0, 0], period=[0, 0, 0.057], nperiods=30, phase=0)
    n1, s1, st1, _, v1 = _grid1d()
    n3, s3, st3, _, v3 = _grid3d()
    hs = halfscale_41()
    short = dict(bfield=[0, 1.0, 0], period=[0, 0, 0.02], nperiods=30, phase=pi2)
    return [
        ("undulator", [undulator(**und)], [("add_bfield_undulator", und)], 3.0, (0, 0, 0), (0, 0, 1), (-1.5, 1.5), 20001),
        ("epu_two_undulators", [undulator(**ey), undulator(**ex)],
         [("add_bfield_undulator", ey), ("add_bfield_undulator", ex)], 3.0, (0, 0, 0), (0, 0, 1), (-1.0, 1.0), 16001),
        ("epu", [epu([0, 0.6, 0], [0.4, 0, 0], [0, 0, 0.057], 30, phase=0.3)],
         [("add_bfield_epu", dict(period=[0, 0, 0.057], nperiods=30, bfieldA=[0, 0.6, 0], bfieldB=[0.4, 0, 0],
                                  phase=0.3))], 3.0, (0, 0, 0), (0, 0, 1), (-1.0, 1.0), 16001),
        ("grid_oscars1d", [grid(v1, n1, s1, st1, translation=(0, 0, 0.01))],
         [("add_bfield_grid", dict(values=v1, npoints=n1, start=s1, step=st1, translation=[0, 0, 0.01]))],
         3.0, (0, 0, 0), (0, 0, 1), (-1.5, 1.5), 16001),
        ("grid_oscars_3d", [grid(v3, n3, s3, st3, rotations=(0, 0, 0.002), translation=(0.0001, 0, 0))],
         [("add_bfield_grid", dict(values=v3, npoints=n3, start=s3, step=st3, rotations=[0, 0, 0.002],
                                   translation=[0.0001, 0, 0]))], 3.0, (0, 0, 0), (0, 0, 1), (-1.2, 1.2), 12001),
        ("halfscale_undulator", [undulator(**dict(und, half_period_scale=hs))],
         [("add_bfield_undulator", dict(und, half_period_scale=hs))], 3.0, (0, 0, 0), (0, 0, 1), (-1.5, 1.5), 20001),
        ("tilted_beam_short_period", [undulator(**short)], [("add_bfield_undulator", short)], 2.0,
         (0.001, -0.0005, -0.5), (0.0003, 0.0001, 1), (-0.9, 0.9), 7001),
    ]


@pytest.mark.parametrize("spline", [1, 2])  # the serial and the block-parallel spline kernel
@pytest.mark.parametrize("case", [c[0] for c in _cases()])
def test_device_trajectory_matches_host(case, spline):
    from oscars_b200.batch import BatchRunner, Job
    name, bfields, ofields, energy, x0, d0, ct, npts = next(c for c in _cases() if c[0] == case)
    job = Job(fields=bfields, energy_GeV=energy, ctstartstop=ct, npoints=npts, obs=[[0, 0, 30]],
              energies_eV=[E1_EPU], x0=x0, d0=d0)
    runner = BatchRunner(0)
    runner.ctx.call("osc_set_batch_spline_kernel", spline)
    dev = runner.trajectories([job])[0]
    host = _oracle_knots(ofields, energy, x0, d0, ct, npts)
    assert dev.shape == host.shape, (dev.shape, host.shape)
    assert np.array_equal(dev[0], host[0]), "knot times differ"
    errs = {}
    for r in range(1, 10):
        scale = np.max(np.abs(host[r]))
        errs[ROWS[r]] = float(np.max(np.abs(dev[r] - host[r])) / scale) if scale > 0 else float(np.max(np.abs(dev[r])))
    worst = max(errs, key=errs.get)
    h = float(np.min(np.diff(host[0])))
    eps = np.finfo(float).eps
    d2 = {}  # second-derivative differences as a fraction of the bound propagated from the values
    for c in range(9):
        d_c = float(np.max(np.abs(dev[1 + c] - host[1 + c])))
        bound = 24 * (d_c + 8 * eps * float(np.max(np.abs(host[1 + c])))) / h ** 2
        diff = float(np.max(np.abs(dev[10 + c] - host[10 + c])))
        d2[ROWS[10 + c]] = diff / bound if bound > 0 else (0.0 if diff == 0 else float("inf"))  # a zero component
    worst_d2 = max(d2, key=d2.get)
    mid = {}
    for c in range(9):
        def at_mid(k):
            y, ypp = k[1 + c], k[10 + c]
            hh = np.diff(k[0])
            return 0.5 * (y[:-1] + y[1:]) - (ypp[:-1] + ypp[1:]) * hh * hh / 16
        a, b = at_mid(dev), at_mid(host)
        scale = np.max(np.abs(b))
        mid[ROWS[1 + c]] = float(np.max(np.abs(a - b)) / scale) if scale > 0 else float(np.max(np.abs(a)))
    worst_mid = max(mid, key=mid.get)
    print("%s: values worst %s %.3e (x %.2e bx %.2e ax %.2e); second derivatives worst %s at %.2e of their bound; "
          "midpoints worst %s %.3e" % (case, worst, errs[worst], errs["x"], errs["bx"], errs["ax"], worst_d2, d2[worst_d2],
                                       worst_mid, mid[worst_mid]))
    assert errs[worst] <= TOL, errs
    assert d2[worst_d2] <= 1.0, d2
    assert mid[worst_mid] <= TOL, mid


def test_several_jobs_in_one_call_keep_their_own_knots():
    """Jobs of different lengths in one call: each job's block equals the job computed alone."""
    from oscars_b200.batch import BatchRunner, Job
    cs = _cases()
    jobs = [Job(fields=c[1], energy_GeV=c[3], ctstartstop=c[6], npoints=c[7], obs=[[0, 0, 30]], energies_eV=[E1_EPU],
                x0=c[4], d0=c[5]) for c in (cs[0], cs[4], cs[6])]
    r = BatchRunner(0)
    together = r.trajectories(jobs)
    for jb, t in zip(jobs, together):
        alone = r.trajectories([jb])[0]
        assert np.array_equal(alone, t)
