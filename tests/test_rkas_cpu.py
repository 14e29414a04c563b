"""Adaptive Cash-Karp trajectories (RKAS) on the host.

The product's host integrator is compared bit for bit with the reference's RKAS trajectories in the
golden fixtures traj_rkas and traj_rkas_epu by test_capi_cpu.py's trajectory test (every
calculate_trajectory case); here: the method switch and its errors as the reference's
SetTrajectoryCalculation raises them (src/OSCARSSR.cc:784-820, including that an RKAS request with a
bad precision leaves RKAS selected), print_trajectory's text, and a third configuration (a tilted
particle through a grid field at precision 1e-9) against the oracle.
"""
import numpy as np
import pytest

from cases import BEAM, UND_SHORT, field_file, run_case, traj


def _host():
    from oscars_b200.sr import sr
    return sr(gpu=1, device=-1)


def _method(s):
    import ctypes
    m, p = ctypes.c_int(), ctypes.c_double()
    s._ctx.call("osc_get_trajectory_calculation", ctypes.byref(m), ctypes.byref(p))
    return m.value, p.value


def test_method_switch_and_errors(capsys):
    s = _host()
    assert _method(s) == (0, 1e-6)
    with pytest.raises(ValueError, match="RK4 Trajectory does not use the precision parameter"):
        s.set_trajectory_calculation("RK4", 1e-3)
    assert _method(s) == (0, 1e-6)
    with pytest.raises(ValueError, match="Method requested is invalid.  Try again"):
        s.set_trajectory_calculation("euler")
    s.set_trajectory_calculation("rkas", 1e-8)
    assert _method(s) == (1, 1e-8)
    s.set_trajectory_calculation("RK4")
    assert _method(s) == (0, 1e-8)
    with pytest.raises(ValueError, match="Trajectory precision cannot be >= 0"):
        s.set_trajectory_calculation("RKAS", -1e-3)
    assert _method(s) == (1, 1e-8)  # the reference sets the method before it checks the precision
    s.print_trajectory()
    assert capsys.readouterr().out == "*Trajectory Calculation Globals*\nMethod:    RKAS\nPrecision: 1e-08\n\n"


def test_rkas_grid_field_tilted_particle_matches_oracle():
    from oracle.oracle import OracleSR
    calls = [("add_bfield_file", dict(ifile="und1d.txt", iformat="OSCARS1D Z By Bx", scale=[1, 1.02, 1])),
             ("set_particle_beam", dict(type="electron", energy_GeV=2.5, x0=[0.0005, 0, -1.2],
                                        d0=[0.0003, -0.0001, 1], current=0.3))] + traj(9001, -1.3, 1.3) + \
            [("set_trajectory_calculation", dict(method="RKAS", precision=1e-9)), ("calculate_trajectory", {})]
    s, o = _host(), OracleSR()
    run_case(s, calls)
    run_case(o, calls)
    a, b = s.trajectory_array(), o.trajectory_array()
    assert a.shape == b.shape and np.array_equal(a, b)
    assert np.sum(np.diff(a[0]) == 0) == 1  # the start time appears twice, as in the reference
