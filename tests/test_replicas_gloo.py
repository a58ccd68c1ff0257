"""Replica partitioning and the max-over-ranks timing reduction, as two gloo
ranks on CPU (the multi-GPU bench path without GPUs)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from openparem_b200.replicas import partition, max_over_ranks
    freqs = np.linspace(8e9, 12e9, 51)
    mine = partition(freqs, rank, world)
    t = max_over_ranks([float(len(mine)) + rank * 0.5, 1.0 + rank], dist)
    out[rank] = (list(mine), t)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_cover_the_sweep_and_reduce_max():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    allf = sorted(f for r in range(world) for f in res[r][0])
    assert np.allclose(allf, np.linspace(8e9, 12e9, 51))
    assert len(set(res[0][0]) & set(res[1][0])) == 0
    # rank 0 holds 26 points, rank 1 holds 25 (+0.5): the max is rank 0's 26 and rank 1's 2
    for r in range(world):
        assert res[r][1] == [26.0, 2.0]
