"""Host-side multi-rank plumbing (one process per GPU, torch.distributed).

The explicit residual/update path needs no data exchange between ranks in the configurations this
library runs: a single mesh runs as independent replicas (one per GPU), and a batch of independent
solves is split across ranks by instance.  Timing follows the device-time, max-over-ranks rule.
"""


def shard_instances(cells, rank, world):
    """Contiguous split of instances (given their cell counts) into `world` groups of nearly equal
    total cell count; returns the instance indices of `rank`.  Deterministic, every instance in
    exactly one group."""
    n = len(cells)
    total = float(sum(cells))
    bounds = [0]
    acc = 0.0
    k = 1
    for i, c in enumerate(cells):
        acc += c
        while k < world and acc >= total * k / world and len(bounds) < world:
            bounds.append(i + 1)
            k += 1
    while len(bounds) < world:
        bounds.append(n)
    bounds.append(n)
    return list(range(bounds[rank], bounds[rank + 1]))


def max_over_ranks(value, dist=None, device=None):
    """Max of a float over all ranks (identity with one rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist=None, device=None):
    """Sum of a float over all ranks (identity with one rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
