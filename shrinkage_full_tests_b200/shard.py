"""Data-parallel sharding of the batched training forward.

The B images of srkTrainingForward are independent, so N GPUs split the batch
into contiguous shards and run with no data-path collective
(training/srk_training_forward.cuh:148-155 batches the same way on one GPU).
Timing across ranks is the max of the per-rank device times.
"""


def batch_shard(B, rank, world):
    """Contiguous shard [start, start+count) of a batch of B images for `rank`
    of `world`; the first B % world ranks take one extra image."""
    if world < 1 or not (0 <= rank < world) or B < 0:
        raise ValueError("bad shard request B=%d rank=%d world=%d" % (B, rank, world))
    base, extra = divmod(B, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def max_over_ranks(value, dist=None, device=None):
    """Max of a per-rank float over the process group (identity without one)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
