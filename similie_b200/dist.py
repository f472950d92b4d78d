"""Multi-GPU plumbing for the batched workloads: one process per GPU, problems
sharded across ranks with no data-path collective (independent problems);
torch.distributed is used only to time the job as the maximum over ranks and
to gather per-problem diagnostics on rank 0."""
import os


def env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(items, rank, world):
    """Contiguous, balanced split of a list: rank r gets items[lo:hi]."""
    n = len(items)
    lo = n * rank // world
    hi = n * (rank + 1) // world
    return items[lo:hi]


def shard_by_work(costs, world):
    """Assign items to ranks greedily by cost (largest first) so the slowest
    rank, which sets the job time, carries as little as possible.  Returns
    one list of item indices per rank, each in ascending order."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(o) for o in out]


def max_over_ranks(value, device=None):
    """Maximum of a float over all ranks (the job's device time)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_rank0(obj):
    """List of every rank's object on rank 0 (None elsewhere)."""
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out


def merge_records(gathered, sum_keys, max_keys):
    """Per-kind records of every rank (rank 0's gather_to_rank0 result, a list
    of {kind: {key: value}}) merged into rank 0's: the keys of sum_keys added
    over ranks, those of max_keys maximised; other keys keep rank 0's value."""
    out = {kind: dict(rec) for kind, rec in gathered[0].items()}
    for kind, rec in out.items():
        for key in sum_keys:
            rec[key] = sum(g[kind][key] for g in gathered)
        for key in max_keys:
            rec[key] = max(g[kind][key] for g in gathered)
    return out
