"""Multi-process plumbing for the weak-scaling evaluation: one process per GPU, every
rank evaluates its own independent suspension (no data-path collective); timing is the
maximum over ranks. Uses torch.distributed (NCCL on GPUs, gloo on CPU)."""
import os


def rank_seed(base_seed, rank):
    """Seed of the suspension owned by a rank (rank 0 keeps the configuration's seed)."""
    return int(base_seed) + 100 * int(rank)


def env_world():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def barrier(world):
    """Barrier over all ranks (no-op for one rank)."""
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, device=None):
    """Maximum of a float over all ranks (every rank gets it)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_throughput(units_per_rank, seconds_max, world):
    """Whole-job throughput: every rank processes units_per_rank in at most seconds_max."""
    return units_per_rank * world / seconds_max
