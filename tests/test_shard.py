"""The multi-GPU host logic on CPU: two gloo ranks shard the N-1 cases of one grid
(distinct sets, no collective on the data path) and reduce the step time with MAX."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from mapol_b200.shard import dist_env, max_over_ranks, rank_cases

    r, w, lr = dist_env()
    buses, branches, cases = rank_cases("cfg1_300bus", r)
    t = max_over_ranks(1.0 + r, w)
    out[r] = (len(cases), sorted(c[0] for c in cases), t, buses.tobytes() == rank_cases("cfg1_300bus", 0)[0].tobytes())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_gloo(built):
    port = 29500 + (os.getpid() % 1000)
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    n0, c0, t0, same0 = out[0]
    n1, c1, t1, same1 = out[1]
    assert n0 == n1 == 200
    assert c0 != c1
    assert t0 == t1 == 2.0
    assert same0 and same1
