"""GPU parity of the plain FP64 path against the reference.

Every golden case (values computed by the reference's own CPU build) is replayed through
``oscars_b200.sr`` on the GPU.  Tolerance for values: relative error <= 1e-9, measured against the
case's peak (max_i |F_i - F_ref_i| / max_i |F_ref_i|); stop levels must be identical.  At the full
201 x 201 flux / power-density grid the comparison is against the CPU oracle (itself pinned bit for
bit to the reference by test_oracle_pin.py).
"""
import os

import numpy as np
import pytest

from cases import CASES, E1_U, UND_SETUP, carried_levels, run_case
from oracle.oracle import OracleSR

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-9

pytestmark = pytest.mark.gpu


def _sr():
    from oscars_b200.sr import sr
    return sr(gpu=1)


def _flat(res):
    return (np.array([r[0] for r in res], dtype=np.float64), np.array([r[1] for r in res], dtype=np.float64))


def _peak_rel(a, b):
    """Peak-normalised difference; NaN entries (0 / 0 in the reference's precision of a fully shadowed
    STL facet) must sit at the same places."""
    nan = np.isnan(b)
    if not np.array_equal(np.isnan(a), nan):
        return float("inf")
    a, b = a[~nan], b[~nan]
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) if b.size else 0.0


RADIATION_CASES = sorted(k for k, v in CASES.items() if v[-1][0] != "calculate_trajectory")


@pytest.mark.parametrize("name", RADIATION_CASES)
def test_golden_case_on_gpu(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    s = _sr()
    calls = list(CASES[name])
    last, kw = calls[-1]
    pos, val = _flat(run_case(s, calls[:-1] + [(last, dict(kw, gpu=1))]))
    assert np.array_equal(pos, g["pos"])
    err = _peak_rel(val, g["val"])
    if kw.get("quantity") == "level":
        assert np.array_equal(carried_levels(val), g["val"])
    else:
        assert err <= TOL, "%s: peak-normalised error %.3e" % (name, err)
    if "level" in g.files:
        s2 = _sr()
        _, lev = _flat(run_case(s2, calls[:-1] + [(last, dict(kw, gpu=1, quantity="level"))]))
        lev = carried_levels(lev)
        assert np.array_equal(lev, g["level"]), "stop levels differ at %d entries" % int(np.sum(lev != g["level"]))


def _cfg1(obj, what):
    run_case(obj, UND_SETUP)
    if what == "flux":
        return obj.calculate_flux_rectangle(energy_eV=E1_U, npoints=[201, 201], width=[0.01, 0.01], translation=[0, 0, 30])
    return obj.calculate_power_density_rectangle(npoints=[201, 201], width=[0.01, 0.01], translation=[0, 0, 30])


@pytest.mark.parametrize("what", ["flux", "pd"])
def test_full_201x201_grid_against_oracle(what):
    _, ref = _flat(_cfg1(OracleSR(), what))
    s = _sr()
    _, val = _flat(_cfg1(s, what))
    err = _peak_rel(val, ref)
    assert err <= TOL, "peak-normalised error %.3e" % err
    # per-entry relative error where the value is not vanishingly small
    big = np.abs(ref) > 1e-6 * np.max(np.abs(ref))
    assert np.max(np.abs(val[big] - ref[big]) / np.abs(ref[big])) <= 1e-7


def test_device_entry_point_matches_host_entry_point():
    import ctypes
    import torch
    from oscars_b200._lib import RadOpts
    s = _sr()
    run_case(s, UND_SETUP)
    pos, host = _flat(s.calculate_flux_rectangle(energy_eV=E1_U, npoints=[31, 31], width=[0.01, 0.01],
                                                 translation=[0, 0, 30], dim=3))
    obs = torch.tensor(pos, dtype=torch.float64, device="cuda")
    out = torch.zeros(pos.shape[0], dtype=torch.float64, device="cuda")
    lvl = torch.zeros(pos.shape[0], dtype=torch.int32, device="cuda")
    o = RadOpts(precision=0.01, max_level=-2, max_level_extended=0, nparticles=0, quantity=0, precision_mode=0)
    o.horizontal[:] = [1, 0, 0]
    o.propagation[:] = [0, 0, 1]
    s._ctx.call("osc_flux_device", ctypes.c_void_p(obs.data_ptr()), pos.shape[0], E1_U, ctypes.byref(o),
                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(lvl.data_ptr()), None)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), host)


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("power_density", [False, True])
def test_pinned_host_outputs_match_pageable_outputs(mode, power_density):
    """Page-locked and pageable host buffers (observers, normals, outputs) give the same values and
    levels, and the same as device buffers; so do repeated calls of one request shape, whose later
    calls enqueue their waves and result downloads without a host round trip."""
    import ctypes
    import torch
    from oscars_b200 import _lib
    from oscars_b200._lib import RadOpts
    s = _sr()
    run_case(s, UND_SETUP)
    xyz, _, _ = s._rectangle([41, 37], "XY", [0.006, 0.006], None, None, [0, 0, 30], 0, False)
    xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
    n = xyz.shape[0]
    o = RadOpts(precision=0.01, max_level=-2, max_level_extended=0, nparticles=0, quantity=0, precision_mode=mode)
    o.horizontal[:] = [1, 0, 0]
    o.propagation[:] = [0, 0, 1]

    nrm = np.ascontiguousarray(np.tile([0.0, 0.0, 1.0], (n, 1)))
    pin_nrm_t = torch.from_numpy(nrm.copy()).pin_memory()

    def call(obs, out, lvl):
        if power_density:  # normals page-locked with page-locked observers
            nv = pin_nrm_t.numpy() if obs is not xyz else nrm
            s._ctx.call("osc_power_density", _lib.dptr(obs), _lib.dptr(nv), n, 0, ctypes.byref(o), _lib.dptr(out),
                        _lib.i32ptr(lvl), None)
        else:
            s._ctx.call("osc_flux", _lib.dptr(obs), n, E1_U, ctypes.byref(o), _lib.dptr(out), _lib.i32ptr(lvl), None)

    ref_out, ref_lvl = np.zeros(n), np.zeros(n, dtype=np.int32)
    call(xyz, ref_out, ref_lvl)
    assert np.all(ref_out != 0) and len(set(ref_lvl.tolist())) > 1
    pin_obs_t = torch.from_numpy(xyz.copy()).pin_memory()
    pin_obs = pin_obs_t.numpy()
    for k in range(3):
        for obs in (xyz, pin_obs):
            out_t = torch.full((n,), -1.0, dtype=torch.float64).pin_memory()
            lvl_t = torch.full((n,), -7, dtype=torch.int32).pin_memory()
            call(obs, out_t.numpy(), lvl_t.numpy())
            assert np.array_equal(out_t.numpy(), ref_out), k
            assert np.array_equal(lvl_t.numpy(), ref_lvl), k
            out_p, lvl_p = np.full(n, -1.0), np.full(n, -7, dtype=np.int32)
            call(obs, out_p, lvl_p)
            assert np.array_equal(out_p, ref_out) and np.array_equal(lvl_p, ref_lvl), k
    if not power_density:
        d_obs = torch.tensor(xyz, device="cuda")
        d_out = torch.zeros(n, dtype=torch.float64, device="cuda")
        d_lvl = torch.zeros(n, dtype=torch.int32, device="cuda")
        s._ctx.call("osc_flux_device", ctypes.c_void_p(d_obs.data_ptr()), n, E1_U, ctypes.byref(o),
                    ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_lvl.data_ptr()), None)
        torch.cuda.synchronize()
        assert np.array_equal(d_out.cpu().numpy(), ref_out) and np.array_equal(d_lvl.cpu().numpy(), ref_lvl)


def test_flux_multi_matches_single_energy_calls():
    """osc_flux_multi (all observers x energies in one request) against osc_flux per energy and
    osc_spectrum, FP64, fixed level."""
    import ctypes
    from oscars_b200 import _lib
    from oscars_b200._lib import RadOpts
    s = _sr()
    run_case(s, UND_SETUP)
    xyz, _, _ = s._rectangle([7, 5], "XY", [0.004, 0.004], None, None, [0, 0, 30], 0, False)
    xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
    E = np.array([440.0, 458.9458, 470.0])
    o = RadOpts(precision=0.0, max_level=11, max_level_extended=0, nparticles=0, quantity=0, precision_mode=0)
    o.horizontal[:] = [1, 0, 0]
    o.propagation[:] = [0, 0, 1]
    n = xyz.shape[0]
    multi = np.zeros(n * E.size)
    s._ctx.call("osc_flux_multi", _lib.dptr(xyz), n, _lib.dptr(E), E.size, ctypes.byref(o), 0, _lib.dptr(multi),
                None, None)
    for j, e in enumerate(E):
        one = np.zeros(n)
        s._ctx.call("osc_flux", _lib.dptr(xyz), n, float(e), ctypes.byref(o), _lib.dptr(one), None, None)
        assert _peak_rel(multi[j::E.size], one) <= 1e-12
    spec = np.zeros(E.size)
    s._ctx.call("osc_spectrum", _lib.dptr(xyz[3].copy()), _lib.dptr(E), E.size, ctypes.byref(o), _lib.dptr(spec),
                None, None)
    one_obs = np.zeros(E.size)
    s._ctx.call("osc_flux_multi", _lib.dptr(xyz[3].copy()), 1, _lib.dptr(E), E.size, ctypes.byref(o), 1,
                _lib.dptr(one_obs), None, None)
    assert _peak_rel(one_obs, spec) <= 1e-12
