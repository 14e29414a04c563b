"""CPU-side checks of the product library (no GPU needed).

* liboscars_b200.so loads and exports every entry point that include/oscars_b200.h declares;
* the host model behind the C ABI (RK4 trajectory, spline, beam sampling, rectangle surfaces)
  reproduces the reference bit for bit (golden fixtures / CPU oracle), through a host-only
  context (device -1);
* argument errors surface as ValueError with the reference's messages; a radiation call on a
  host-only context fails loudly instead of falling back to the CPU.
"""
import os
import re

import numpy as np
import pytest

from cases import CASES, run_case
from make_golden import exact_sums
from oracle.oracle import OracleSR, rectangle as oracle_rectangle

from oscars_b200 import _lib
from oscars_b200.sr import sr as SR

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def host_sr():
    return SR(device=-1)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    text = open(os.path.join(ROOT, "include", "oscars_b200.h")).read()
    declared = set(re.findall(r"OSC_API\s+[\w\s\*]+?\b(osc_\w+)\s*\(", text))
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    assert declared == set(_lib.SIGNATURES), declared ^ set(_lib.SIGNATURES)


@pytest.mark.parametrize("name", sorted(k for k, v in CASES.items() if v[-1][0] == "calculate_trajectory"))
def test_trajectory_bit_exact_with_reference(name):
    """Ideal undulator, grid fields from both text formats, and the half-period-scaled undulator
    (given to the reference as a Python field function)."""
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    s = host_sr()
    run_case(s, CASES[name])
    a = s.trajectory_array()
    assert a.shape[1] == int(g["n"])
    assert np.array_equal(a[:, g["idx"]], g["sub"])
    assert np.array_equal(exact_sums(a), g["sums"])
    assert np.array_equal(exact_sums(np.abs(a)), g["abssums"])


@pytest.mark.parametrize("name", ["spec_taper_time", "epu_field_spec", "flux_epu_21"])
def test_trajectory_bit_exact_with_oracle(name):
    setup = [c for c in CASES[name] if not c[0].startswith("calculate")]
    s, o = host_sr(), OracleSR()
    run_case(s, setup)
    run_case(o, setup)
    s.calculate_trajectory()
    o.calculate_trajectory()
    assert np.array_equal(s.trajectory_array(), o.trajectory_array())


def test_gaussian_beam_sampling_matches_oracle():
    setup = [c for c in CASES["flux_epu_multi"] if not c[0].startswith("calculate")]
    s, o = host_sr(), OracleSR()
    run_case(s, setup)
    run_case(o, setup)
    for _ in range(5):
        s.set_new_particle()
        o.set_new_particle()
        x0, b0, t0, g, *_ = o.get_particle()
        assert s.get_particle_x0() == list(x0)
        assert s.get_particle_beta0() == list(b0)


@pytest.mark.parametrize("plane", ["XY", "YX", "XZ", "ZX", "YZ", "ZY"])
@pytest.mark.parametrize("n", [(1, 1), (1, 5), (4, 1), (7, 3)])
def test_rectangle_matches_reference_layout(plane, n):
    rot, tr = [0.1, -0.2, 0.3], [0.01, 0.02, 30.0]
    s = host_sr()
    xyz, nrm, x12 = s._rectangle(list(n), plane, [0.01, 0.02], None, rot, tr, -1, False)
    oxyz, onrm, ox12 = oracle_rectangle(plane, n[0], n[1], 0.01, 0.02, rot, tr, -1)
    assert np.array_equal(xyz.reshape(-1, 3), oxyz)
    assert np.array_equal(nrm.reshape(-1, 3), onrm)
    assert np.array_equal(x12.reshape(-1, 3), ox12)


def test_golden_positions_reproduced():
    for name in ("flux_und_41", "flux_und_dim3_yz", "pd_und_41"):
        g = np.load(os.path.join(GOLDEN, name + ".npz"))
        last, kw = CASES[name][-1]
        s = host_sr()
        plane = kw.get("plane", "XY")
        xyz, nrm, x12 = s._rectangle(kw["npoints"], plane, kw.get("width"), None, kw.get("rotations"),
                                     kw.get("translation"), kw.get("normal", 0), last.startswith("calculate_power"))
        pos = (xyz if kw.get("dim", 2) == 3 else x12).reshape(-1, 3)
        assert np.array_equal(pos, g["pos"])


def test_spectrum_energy_grid_matches_golden():
    g = np.load(os.path.join(GOLDEN, "spec_und_2000.npz"))
    E = SR._energies(2000, [100, 3000], None)
    assert np.array_equal(E, g["pos"])


def test_grid_file_errors():
    s = host_sr()
    with pytest.raises(ValueError, match="cannot specify both 'ifile' and 'bifile'"):
        s.add_bfield_file(ifile="a", bifile="b")
    with pytest.raises(ValueError, match="'iformat' is blank"):
        s.add_bfield_file(ifile="a")
    with pytest.raises(ValueError, match="Could not import magnetic field"):
        s.add_bfield_file(ifile="/nonexistent/file.txt", iformat="OSCARS")
    with pytest.raises(ValueError, match="Could not import magnetic field"):
        s.add_bfield_file(ifile=os.path.join(GOLDEN, "fields", "und1d.txt"), iformat="OSCARS1D Z Q")
    with pytest.raises(ValueError, match="Could not import magnetic field"):
        s.add_bfield_file(ifile=os.path.join(GOLDEN, "fields", "und1d.txt"), iformat="TEXT")
    with pytest.raises(ValueError, match="2 \\* nperiods"):
        s.add_bfield_undulator(bfield=[0, 0.5, 0], period=[0, 0, 0.05], nperiods=41, half_period_scale=[1.0] * 80)


def test_grid_from_memory_matches_file_grid():
    """add_bfield_grid with the values of an 'OSCARS' file gives the file's field."""
    from oracle.oracle import read_oscars_grid
    path = os.path.join(GOLDEN, "fields", "grid3d.txt")
    n, start, step, stop, vals = read_oscars_grid(path, [0.0, 0.0, 0.0], [])
    a, b = host_sr(), host_sr()
    a.add_bfield_file(ifile=path, iformat="OSCARS", translation=[0.0001, 0, 0])
    b.add_bfield_grid(vals, n, start, step, translation=[0.0001, 0, 0])
    pts = [[-0.0015 + 1.5e-5 * i, 0.0012 - 1.2e-5 * i, -1.0 + 0.01 * i] for i in range(201)]
    fa = np.array([a.get_bfield(p) for p in pts])
    assert np.array_equal(fa, np.array([b.get_bfield(p) for p in pts])) and np.abs(fa).max() > 0.1


def test_errors_are_value_errors():
    s = host_sr()
    with pytest.raises(ValueError, match="No particle beam defined"):
        s.calculate_flux_rectangle(energy_eV=100, npoints=[3, 3], width=[0.01, 0.01], translation=[0, 0, 30])
    run_case(s, CASES["traj_und"][:-1])
    with pytest.raises(ValueError, match="Polarization requested not recognized"):
        s.calculate_spectrum(obs=[0, 0, 30], energy_range_eV=[100, 200], npoints=3, polarization="diagonal")
    with pytest.raises(ValueError, match="cannot specify 'all' and 'angle'"):
        s.calculate_spectrum(obs=[0, 0, 30], energy_range_eV=[100, 200], npoints=3, polarization="all", angle=0.1)
    with pytest.raises(ValueError, match="'quantity' must be"):
        s.calculate_spectrum(obs=[0, 0, 30], energy_range_eV=[100, 200], npoints=3, quantity="bogus")
    with pytest.raises(ValueError, match="an entry in 'npoints' is <= 0"):
        s.calculate_flux_rectangle(energy_eV=100, npoints=[0, 3], width=[0.01, 0.01])
    with pytest.raises(ValueError, match="'dim' must be 2 or 3"):
        s.calculate_flux_rectangle(energy_eV=100, npoints=[3, 3], width=[0.01, 0.01], dim=4)
    with pytest.raises(ValueError, match="gpu is 1 and nthreads > 0"):
        s.calculate_spectrum(obs=[0, 0, 30], energy_range_eV=[100, 200], npoints=3, gpu=1, nthreads=2)
    with pytest.raises(ValueError, match="start time is greater than stop time"):
        s.set_ctstartstop(0, 0)
        s.calculate_trajectory()


def test_radiation_without_gpu_fails_loudly():
    s = host_sr()
    run_case(s, CASES["traj_und"][:-1])
    with pytest.raises(RuntimeError, match="no usable GPU|without a GPU"):
        s.calculate_spectrum(obs=[0, 0, 30], energy_range_eV=[100, 200], npoints=3)


def test_variant_names():
    from oscars_b200 import _lib
    for kind, n in ((0, 4), (2, 4), (3, 4)):
        names = [_lib.variant_name(kind, v) for v in range(n)]
        assert all(names) and len(set(names)) == n
    assert _lib.variant_name(2, 0) == "k_fd_wave_mixed_pair<4,4,128,false>"
    assert _lib.variant_name(3, 3) == "k_batch_wave<1,4>"
    with pytest.raises(ValueError, match="out of range"):
        _lib.variant_name(2, 4)
    with pytest.raises(ValueError, match="kind"):
        _lib.variant_name(1, 0)


def test_tuning_setters_and_vjp_buffers_checked_on_the_host():
    """The beam routing threshold, the batch spline kernel choice and the adjoint's buffer rules are
    argument checks of the C ABI: they answer on a host-only context without launching anything."""
    import ctypes
    ctx = _lib.Context(-1)
    ctx.call("osc_set_beam_batch_threshold", 1)
    ctx.call("osc_set_beam_batch_threshold", 4096)
    with pytest.raises(ValueError, match="at least 1 particle"):
        ctx.call("osc_set_beam_batch_threshold", 0)
    for k in (0, 1, 2):
        ctx.call("osc_set_batch_spline_kernel", k)
    for k in (-1, 3):
        with pytest.raises(ValueError, match="kernel must be 0, 1 or 2"):
            ctx.call("osc_set_batch_spline_kernel", k)
    DP = ctypes.POINTER(ctypes.c_double)
    obs = (ctypes.c_double * 3)(0.0, 0.0, 30.0)
    en = (ctypes.c_double * 1)(100.0)
    opts = _lib.RadOpts(precision=0.01, max_level=10, max_level_extended=10, shard_count=1)
    none = ctypes.cast(None, DP)
    # forward only (no gradient) needs flux_out; with a gradient, grad_half_scale is required
    with pytest.raises(ValueError, match="bad buffers"):
        ctx.call("osc_flux_vjp", obs, 1, en, 1, 8, ctypes.byref(opts), 0, none, none, none, 0, none)
    g = (ctypes.c_double * 1)(1.0)
    with pytest.raises(ValueError, match="bad buffers"):
        ctx.call("osc_flux_vjp", obs, 1, en, 1, 8, ctypes.byref(opts), 0, g, none, none, 0, none)
    opts.nparticles = 2
    with pytest.raises(ValueError, match="one particle"):
        ctx.call("osc_flux_vjp", obs, 1, en, 1, 8, ctypes.byref(opts), 0, g, none, none, 0, none)
    ctx.close()
