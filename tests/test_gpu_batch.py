"""Batched mixed-precision path: osc_batch_flux (uneven jobs) and multi-particle compute='mixed'.

Tolerance as for the single-trajectory mixed path: peak-normalised relative error
max_i |F_i - F64_i| / max_i |F64_i| <= 1e-4 against the FP64 GPU path, at a fixed level
(precision=0, max_level=L) so that both integrate the same samples.  The FP64 path matches the
reference CPU path to <= 1e-9 (test_gpu_parity.py).  In the batch, trajectories, splines and level
samples are computed on the device, so these tests also cover those kernels.  Multi-particle mixed
requests run as a batch from a threshold of particles on (osc_set_beam_batch_threshold) and per
particle with host trajectories below it: the beam tests run both routes.
"""
import math

import numpy as np
import pytest

from cases import BEAM_GAUSS, E1_EPU, EPU_X, EPU_Y, UND_SETUP, run_case, traj

pytestmark = pytest.mark.gpu
TOL = 1e-4


ROUTES = {"batch": 1, "per_particle": 1 << 30}  # osc_set_beam_batch_threshold for each route


def _sr_route(route):
    from oscars_b200.sr import sr
    s = sr(gpu=1)
    s._ctx.call("osc_set_beam_batch_threshold", ROUTES[route])
    return s


def _err(a, ref):
    a, ref = np.asarray(a, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    return float(np.max(np.abs(a - ref)) / np.max(np.abs(ref)))


def _e1_eV(bfield, period, energy_GeV=3.0):
    lam_cm = period * 100
    K = 0.9337 * bfield * lam_cm
    return 1000 * 0.9496 * energy_GeV ** 2 / (lam_cm * (1 + K * K / 2))


def _grid(nx, ny, w, z):
    xs = np.linspace(-w / 2, w / 2, nx) if nx > 1 else np.zeros(1)
    ys = np.linspace(-w / 2, w / 2, ny) if ny > 1 else np.zeros(1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), np.full(X.size, z)], axis=1)


def uneven_jobs(seed=5, n=6):
    from oscars_b200.batch import Job, undulator
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n):
        lam = float(rng.uniform(0.02, 0.08))
        B = float(rng.uniform(0.3, 1.0))
        N = int(rng.integers(10, 40))
        half = lam * (N + 2) / 2 + 0.2
        npts = int(rng.integers(3000, 12000))
        nx, ny = int(rng.integers(1, 9)), int(rng.integers(1, 9))
        z = float(rng.uniform(20, 40))
        ne = int(rng.integers(1, 17))
        e1 = _e1_eV(B, lam)
        jobs.append(Job(fields=[undulator([0, B, 0], [0, 0, lam], N, phase=-math.pi / 2)], energy_GeV=3.0,
                        ctstartstop=(-half, half), npoints=npts, obs=_grid(nx, ny, 0.004, z),
                        energies_eV=np.linspace(0.95 * e1, 1.05 * e1, ne), current=0.5))
    return jobs


def test_uneven_batch_matches_fp64_fixed_level():
    from oscars_b200.batch import BatchRunner
    r = BatchRunner(0)
    jobs = uneven_jobs()
    mx = r.flux(jobs, compute="mixed", precision=0, max_level=11)
    f64 = r.flux(jobs, compute="fp64", precision=0, max_level=11)
    for k, (a, b) in enumerate(zip(mx, f64)):
        assert a.shape == b.shape == (jobs[k].obs.shape[0], len(jobs[k].energies_eV))
        e = _err(a, b)
        print("job %d %s: mixed vs fp64 %.3e" % (k, a.shape, e))
        assert e <= TOL, (k, e)


def test_batch_repeats_identically_through_the_graph():
    """The first call of a shape tunes and runs eagerly; later calls replay the captured graph."""
    from oscars_b200.batch import BatchRunner
    r = BatchRunner(0)
    jobs = uneven_jobs(seed=11, n=5)
    runs = [r.flux(jobs, compute="mixed") for _ in range(3)]
    levels = r.last_levels
    for k in range(len(jobs)):
        assert np.array_equal(runs[0][k], runs[1][k]) and np.array_equal(runs[1][k], runs[2][k])
        assert np.all((levels[k] >= 9) | (levels[k] == -1))
    s, launches = r.stats()
    assert s > 0 and launches > 0


def test_batch_levels_beyond_the_resident_ones():
    """Levels above 13 are filled one at a time for the jobs still active."""
    from oscars_b200.batch import BatchRunner
    r = BatchRunner(0)
    jobs = uneven_jobs(seed=3, n=3)
    mx = r.flux(jobs, compute="mixed", precision=0, max_level=15)
    f64 = r.flux(jobs, compute="fp64", precision=0, max_level=15)
    for a, b in zip(mx, f64):
        assert _err(a, b) <= TOL


def test_batch_adaptive_levels_agree_with_fp64():
    from oscars_b200.batch import BatchRunner
    r = BatchRunner(0)
    jobs = uneven_jobs(seed=7, n=4)
    mx = r.flux(jobs, compute="mixed")
    lm = [l.copy() for l in r.last_levels]
    f64 = r.flux(jobs, compute="fp64")
    lf = r.last_levels
    same = np.concatenate([(a == b).ravel() for a, b in zip(lm, lf)])
    print("fraction of entries stopping at another level: %.4f" % (1 - same.mean()))
    assert same.mean() >= 0.97
    for a, b, la, lb in zip(mx, f64, lm, lf):
        m = la == lb
        if m.any():
            assert float(np.max(np.abs(a[m] - b[m])) / np.max(np.abs(b))) <= TOL


def test_batch_spectrum_job_matches_sr_spectrum():
    from oscars_b200.batch import BatchRunner, Job, undulator
    from oscars_b200.sr import sr
    s = sr(gpu=1)
    run_case(s, UND_SETUP)
    E = np.linspace(100, 3000, 200)
    ref = np.array([v[1] for v in s.calculate_spectrum(obs=[0, 0, 30], energy_points_eV=list(E), precision=0,
                                                       max_level=12)])
    job = Job(fields=[undulator([0, 0.5, 0], [0, 0, 0.05], 41, phase=-math.pi / 2)], energy_GeV=3,
              ctstartstop=(-1.5, 1.5), npoints=20001, obs=[[0, 0, 30]], energies_eV=E, spectrum=True, current=0.5)
    out = BatchRunner(0).flux([job], compute="mixed", precision=0, max_level=12)[0].ravel()
    assert _err(out, ref) <= TOL


@pytest.mark.parametrize("route", sorted(ROUTES))
@pytest.mark.parametrize("nparticles", [1, 6])
def test_beam_mixed_matches_fp64_fixed_level(nparticles, route):
    setup = [EPU_Y, EPU_X, BEAM_GAUSS] + traj(16001) + [("set_seed", dict(seed=17))]
    kw = dict(energy_eV=E1_EPU, npoints=[21, 21], width=[0.008, 0.008], translation=[0, 0, 30],
              nparticles=nparticles, precision=0, max_level=11)
    out = {}
    for compute in ("fp64", "mixed"):
        s = _sr_route(route)
        run_case(s, setup)
        out[compute] = np.array([v[1] for v in s.calculate_flux_rectangle(**dict(kw, compute=compute))])
    e = _err(out["mixed"], out["fp64"])
    print("beam of %d, 21x21, L=11: mixed vs fp64 %.3e" % (nparticles, e))
    assert e <= TOL


@pytest.mark.parametrize("route", sorted(ROUTES))
def test_epu_beam_101x101_64_particles_fixed_level(route):
    """The multi-particle EPU configuration on its full 101 x 101 grid (8 mm at 30 m, E1) with a
    64-particle subset of the beam, mixed (device trajectories in the batch route, host ones per
    particle) against host RK4 (FP64)."""
    setup = [EPU_Y, EPU_X, BEAM_GAUSS] + traj(16001) + [("set_seed", dict(seed=42))]
    kw = dict(energy_eV=E1_EPU, npoints=[101, 101], width=[0.008, 0.008], translation=[0, 0, 30],
              nparticles=64, precision=0, max_level=12)
    out = {}
    for compute in ("fp64", "mixed"):
        s = _sr_route(route)
        run_case(s, setup)
        out[compute] = np.array([v[1] for v in s.calculate_flux_rectangle(**dict(kw, compute=compute))])
    e = _err(out["mixed"], out["fp64"])
    print("beam of 64, 101x101, L=12: mixed vs fp64 %.3e" % e)
    assert e <= TOL


@pytest.mark.parametrize("route", sorted(ROUTES))
def test_beam_mixed_polarized_and_spectrum(route):
    setup = [EPU_Y, EPU_X, BEAM_GAUSS] + traj(16001) + [("set_seed", dict(seed=2))]
    for call, kw in (("calculate_flux_rectangle", dict(energy_eV=E1_EPU, npoints=[11, 11], width=[0.006, 0.006],
                                                       translation=[0, 0, 30], polarization="cl")),
                     ("calculate_spectrum", dict(obs=[0.0005, 0, 30], energy_range_eV=[150, 220], npoints=24))):
        out = {}
        for compute in ("fp64", "mixed"):
            s = _sr_route(route)
            run_case(s, setup)
            out[compute] = np.array([v[1] for v in getattr(s, call)(**dict(kw, nparticles=3, precision=0,
                                                                             max_level=11, compute=compute))])
        assert _err(out["mixed"], out["fp64"]) <= TOL, call


def test_batch_rejects_far_off_axis_observers():
    from oscars_b200.batch import BatchRunner
    jobs = uneven_jobs(seed=1, n=2)
    jobs[1].obs = np.array([[2.0, 0.0, 30.0]])
    with pytest.raises(ValueError, match="compute='fp64'"):
        BatchRunner(0).flux(jobs, compute="mixed", precision=0, max_level=10)


def test_batch_grid_and_halfscale_fields_match_fp64():
    """Device RK4 through a grid field (both text formats) and a half-period-scaled undulator."""
    from oscars_b200.batch import BatchRunner, Job, grid, undulator
    from cases import field_file, halfscale_41
    from oracle.oracle import read_oscars1d_grid, read_oscars_grid
    n1, s1, st1, _, v1 = read_oscars1d_grid(field_file("und1d.txt"), "OSCARS1D Z By Bx", [0.0, 0.0, 0.0], [1, 1.02, 1])
    n3, s3, st3, _, v3 = read_oscars_grid(field_file("grid3d.txt"), [0.0, 0.0, 0.0], [1, 1, 1, 1, 1.1, 1])
    obs = _grid(5, 5, 0.004, 30.0)
    jobs = [Job(fields=[grid(v1, n1, s1, st1, translation=(0, 0, 0.01))], energy_GeV=3, ctstartstop=(-1.5, 1.5),
                npoints=16001, obs=obs, energies_eV=[440.0, 459.0]),
            Job(fields=[grid(v3, n3, s3, st3, rotations=(0, 0, 0.002), translation=(0.0001, 0, 0))], energy_GeV=3,
                ctstartstop=(-1.2, 1.2), npoints=12001, obs=obs, energies_eV=[516.0]),
            Job(fields=[undulator([0, 0.5, 0], [0, 0, 0.05], 41, phase=-math.pi / 2, half_period_scale=halfscale_41())],
                energy_GeV=3, ctstartstop=(-1.5, 1.5), npoints=20001, obs=obs, energies_eV=[458.9458])]
    r = BatchRunner(0)
    mx = r.flux(jobs, compute="mixed", precision=0, max_level=11)
    f64 = r.flux(jobs, compute="fp64", precision=0, max_level=11)
    for a, b in zip(mx, f64):
        e = _err(a, b)
        print("grid/halfscale job: mixed vs fp64 %.3e" % e)
        assert e <= TOL


@pytest.mark.parametrize("compute,tol,route", [("fp64", 1e-12, "per_particle"), ("mixed", 1e-6, "per_particle"),
                                               ("mixed", 1e-6, "batch")])
def test_particle_shards_add_up_to_the_whole_request(compute, tol, route):
    """shard=(rank, count): each share integrates particles rank, rank + count, ... with weight 1/N."""
    setup = [EPU_Y, EPU_X, BEAM_GAUSS] + traj(16001) + [("set_seed", dict(seed=5))]
    kw = dict(energy_eV=E1_EPU, npoints=[9, 9], width=[0.006, 0.006], translation=[0, 0, 30], nparticles=7,
              precision=0, max_level=10, compute=compute, return_numpy=True)
    s = _sr_route(route)
    run_case(s, setup)
    whole = s.calculate_flux_rectangle(**kw)[1]
    total = np.zeros_like(whole)
    for r in range(3):
        t = _sr_route(route)
        run_case(t, setup)
        total += t.calculate_flux_rectangle(shard=(r, 3), **kw)[1]
    assert _err(total, whole) <= tol
