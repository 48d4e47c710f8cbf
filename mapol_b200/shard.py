"""Multi-GPU plumbing: one process per GPU, cases sharded across ranks.

Contingency cases are independent, so the path shards with no collective on the
data path: rank r solves its own N-1 set of the same grid (outage seed + r, i.e.
weak scaling).  The only collective is the timing reduction (max over ranks).
"""
import os

from .grid import WORKLOADS, n1_cases, workload


def dist_env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def rank_cases(name, rank, outage_seed=7):
    """(buses, branches, cases) of workload `name` for `rank`."""
    buses, branches, _ = workload(name)
    w = WORKLOADS[name]
    cases = n1_cases(branches, w["n_bus"], w["n_out"], outage_seed + rank, w["with_base"]) if w["n_out"] else [[]]
    return buses, branches, cases


def max_over_ranks(x, world, device=None):
    """Max of a float over all ranks (all_reduce MAX); identity when world == 1."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
