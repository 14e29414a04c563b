"""A multi-particle request split over two processes that compute with the product.

Two spawned ranks (gloo for the exchange) each run ``oscars_b200.shard.sharded`` on the same GPU:
the rank's share of the seeded particle sequence through the product's own radiation call (FP64
single-trajectory path, and the mixed batched path) with weight 1/N, then one all_reduce(SUM).  Every
rank's sum must equal the whole request computed in one process (within 1e-12 of the peak: the
compensated per-process sums are added in another order).  The ranks' kernels never wait on one
another, so sharing one GPU is only a smaller machine, not a stand-in for peer exchange.
"""
import socket

import numpy as np
import pytest

from cases import BEAM_GAUSS, EPU_X, EPU_Y, run_case, traj

pytestmark = pytest.mark.gpu
N_PART = 6
SETUP = [EPU_Y, EPU_X, BEAM_GAUSS] + traj(16001) + [("set_seed", dict(seed=21))]
FLUX = dict(energy_eV=179.2558, npoints=[11, 11], width=[0.006, 0.006], translation=[0, 0, 30], precision=0,
            max_level=11, nparticles=N_PART)


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _worker(rank, world, port, compute, q):
    import torch.distributed as dist
    from oscars_b200.shard import sharded
    from oscars_b200.sr import sr
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        s = sr(gpu=1, device=0)
        run_case(s, SETUP)
        _, total = sharded(s.calculate_flux_rectangle, compute=compute, **FLUX)
        q.put((rank, total))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("compute", ["fp64", "mixed"])
def test_two_product_ranks_sum_to_the_whole_request(compute):
    import torch.multiprocessing as mp
    from oscars_b200.sr import sr
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, compute, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
        assert p.exitcode == 0
    res = dict(q.get() for _ in range(2))
    s = sr(gpu=1)
    run_case(s, SETUP)
    _, whole = s.calculate_flux_rectangle(compute=compute, return_numpy=True, **FLUX)
    for r in range(2):
        err = float(np.max(np.abs(res[r] - whole)) / np.max(np.abs(whole)))
        print("%s rank %d: %.3e" % (compute, r, err))
        assert err <= 1e-12
