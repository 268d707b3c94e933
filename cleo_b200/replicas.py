"""One independent domain per rank (weak scaling): the host logic of multi-GPU runs.

The reference decomposes one domain over MPI ranks and exchanges emigrating superdroplets after
every motion step (libs/cartesiandomain/movement/cartesian_transport_across_domain.hpp:66-239).
Here each rank (one process per GPU) steps its own domain, seeded by its rank, with no collective
on the data path; the process group only aligns the timed regions and combines the timings:
the job's time is the slowest rank's, the job's work is the sum over ranks.
"""
from __future__ import annotations


def domain_seed(base: int, rank: int) -> int:
    """Seed of the synthetic domain of one rank."""
    return int(base) + int(rank)


def combine(times_ms, counts, dist=None, device="cpu"):
    """Max over ranks of each time and sum over ranks of each count (all ranks call this with
    lists of the same lengths, in the same order)."""
    import torch
    t = torch.tensor([float(x) for x in times_ms], dtype=torch.float64, device=device)
    c = torch.tensor([float(x) for x in counts], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.cpu()], [float(x) for x in c.cpu()]
