"""Replica parallelism for sweeps: every (frequency, driving set) solve is
independent, so N GPUs each take their own frequency points and no data-path
collective is needed (the reference distributes one mesh over MPI ranks
instead, OpenParEM3D.cpp:357; here one GPU holds a whole problem).  The only
collective is the timing reduction: the job's time is the slowest rank's."""


def partition(freqs, rank, world):
    """Frequency points of this rank (round robin, so ranks get similar bands)."""
    return freqs[rank::world]


def max_over_ranks(values, dist=None, device="cpu"):
    """Element-wise maximum of a list of floats over all ranks."""
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]
