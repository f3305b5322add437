"""Host logic of the particle decomposition over several GPUs (one process per GPU).

The reference decomposes by particles with a replicated grid (src/mpi_comm.cpp):
every rank pushes and deposits its own particles, the moments are summed over
the ranks (mpi_reduce_densities, called at src/sputniPIC_CPU.cpp:262-265), and the
fields are broadcast from the solver rank. Here every rank holds a full, independently
seeded workload (weak scaling). The one data-path collective is the moment sum. Timing is
the maximum over ranks.

Every function takes the torch.distributed module (or None for one process), so the
same code runs over NCCL on GPUs and over gloo on the CPU in the tests.
"""
from __future__ import annotations


def rank_workload(wl, rank: int):
    """The workload of one rank: the same configuration, seeded by the rank."""
    return wl.with_(seed=int(wl.seed) + rank)


def reduce_moments(mom, dist) -> None:
    """Sums a moment tensor over the ranks, in place (every rank gets the sum)."""
    if dist is not None:
        dist.all_reduce(mom, op=dist.ReduceOp.SUM)


def max_over_ranks(value: float, dist, device="cuda") -> float:
    """The largest value over the ranks (timings are reported as the slowest rank)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(particles_per_rank: int, world: int, steps: int, seconds: float) -> float:
    """Whole-job particles/s: every rank pushed its own particles `steps` times."""
    return particles_per_rank * world * steps / seconds
