"""Multi-particle requests split over processes (one process per GPU, torch.distributed).

Particles are independent; the only exchange is the sum over particles (src/OSCARSSR.cc:4026-4062
adds every particle's flux with weight 1/N).  Each rank draws the same seeded particle sequence,
integrates particles rank, rank + W, rank + 2W, ... with weight 1/N (``shard=(rank, W)`` of the
``oscars_b200.sr`` radiation calls), and one all_reduce(SUM) over the output gives the whole
request on every rank.  With the NCCL backend the partial sums are reduced on the GPU.
"""
from __future__ import annotations

import numpy as np

__all__ = ["allreduce_sum", "sharded"]


def allreduce_sum(values, group=None):
    """Sum a float64 array over the ranks of `group` (NCCL on the current CUDA device, or gloo on
    the CPU); every rank gets the sum."""
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.as_tensor(np.ascontiguousarray(values, dtype=np.float64), device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def sharded(call, *args, group=None, **kwargs):
    """Run an ``oscars_b200.sr`` radiation call with nparticles > 0 on this rank's share and sum the
    shares: ``sharded(s.calculate_flux_rectangle, energy_eV=..., nparticles=10000, compute='mixed')``
    returns (positions, values) on every rank."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    pos, val = call(*args, return_numpy=True, shard=(rank, world), **kwargs)
    return pos, allreduce_sum(val, group)
