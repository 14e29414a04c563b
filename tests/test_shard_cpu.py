"""Host side of the multi-particle split over processes (no GPU).

* The shards of ``beam_particles`` partition the particle sequence a multi-particle request draws,
  and that sequence is the reference's (pinned through the CPU oracle's sampler).
* Two gloo ranks each integrate their particles (round robin, weight 1/N) and one all_reduce gives
  the whole multi-particle flux: checked against the oracle's own N-particle request.  The
  per-particle integrals run on the CPU oracle here (no GPU); test_gpu_shard.py runs the same split
  with two processes computing with the product.
"""
import math
import os
import socket

import numpy as np
import pytest

from cases import BEAM_GAUSS, EPU_X, EPU_Y, run_case, traj

N_PART = 5
SETUP = [EPU_Y, EPU_X, BEAM_GAUSS] + traj(4001) + [("set_seed", dict(seed=11))]
FLUX = dict(energy_eV=179.2558, npoints=[3, 3], width=[0.004, 0.004], translation=[0, 0, 30], precision=0,
            max_level=8)


def _host_sr():
    from oscars_b200.sr import sr
    return sr(device=-1)


def test_shards_partition_the_particle_sequence():
    from oracle.oracle import OracleSR
    s = _host_sr()
    run_case(s, SETUP)
    whole = s.beam_particles(N_PART)
    o = OracleSR()
    run_case(o, SETUP)
    seq = []
    for _ in range(N_PART):
        o.set_new_particle()
        x0, b0 = o.get_particle()[:2]
        seq.append(list(x0) + list(b0))
    assert np.array_equal(whole, np.array(seq))
    parts = []
    for r in range(3):
        t = _host_sr()
        run_case(t, SETUP)
        parts.append(t.beam_particles(N_PART, shard=(r, 3)))
    merged = np.zeros_like(whole)
    for r in range(3):
        merged[r::3] = parts[r]
    assert np.array_equal(merged, whole) and sum(len(p) for p in parts) == N_PART


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from oracle.oracle import OracleSR
    from oscars_b200.shard import allreduce_sum
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        s = _host_sr()
        run_case(s, SETUP)
        mine = s.beam_particles(N_PART, shard=(rank, world))
        part = np.zeros(9)
        o = OracleSR()
        run_case(o, SETUP)
        for p in mine:
            o.set_particle(p[:3], p[3:])
            part += np.array([v[1] for v in o.calculate_flux_rectangle(**FLUX)]) / N_PART
        total = allreduce_sum(part)
        q.put((rank, total))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sum_to_the_whole_request():
    import torch.multiprocessing as mp
    from oracle.oracle import OracleSR
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    res = dict(q.get() for _ in range(2))
    o = OracleSR()
    run_case(o, SETUP)
    whole = np.array([v[1] for v in o.calculate_flux_rectangle(nparticles=N_PART, **FLUX)])
    for r in range(2):
        assert np.max(np.abs(res[r] - whole)) / np.max(np.abs(whole)) <= 1e-13
