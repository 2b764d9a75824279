"""Replica bookkeeping for runs on several GPUs of one node.

The flow-solver pass does not shard (one GPU holds the whole mesh), so N > 1
means N independent replicas, one per rank, with no data-path collective.  The
whole-job rate is the passes all ranks completed divided by the slowest
rank's device time; this module holds that arithmetic and the one collective
it needs, so it can be exercised with the gloo backend on CPU.
"""


def max_over_ranks(value, dist=None, device="cpu"):
    """The largest `value` over the ranks of the default process group
    (the value itself without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(steps_per_rank, slowest_seconds, world):
    """Passes per second of the whole job: every rank ran `steps_per_rank`
    passes; the job took as long as its slowest rank."""
    if slowest_seconds <= 0:
        raise ValueError("elapsed time must be positive")
    return world * steps_per_rank / slowest_seconds
