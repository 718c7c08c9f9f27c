"""One process per GPU, no data-path collective.

The path has no exchange step: the reference distributes q points (and k
partitions) over MPI ranks and each rank's chi0 -> W -> Sigma_c runs alone
(main_hrcxq.f90:94-96).  Here every rank drives its own GPU; the only
collectives are for measurement (the maximum of the ranks' times) and a
barrier around timed regions.  Works with the nccl (GPU) and gloo (CPU)
process groups.
"""


def shard(n, rank, world):
    """Contiguous block of the n items (q points) that rank owns: range(lo, hi).
    Blocks differ in size by at most one and cover 0..n-1 exactly once."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return range(lo, lo + base + (1 if rank < extra else 0))


def max_over_ranks(value, dist=None, device="cpu"):
    """The maximum of a per-rank number over all ranks (value itself when not
    distributed).  device: where the process group's backend reduces
    ("cuda" for nccl, "cpu" for gloo)."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
