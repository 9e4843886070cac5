"""Row sharding across ranks (one process per GPU).

Vectors are independent, so a table splits into contiguous vector ranges per
rank; dimension tables and perfect-hash tables are replicated.  The only
exchange of a fused query is the sum of the ranks' partial int64 aggregates
(8 bytes for a filter-aggregate, 7000 x 8 bytes for the group-by), done with
one all-reduce."""
from __future__ import annotations


def vector_range(n_values: int, world: int, rank: int) -> tuple[int, int]:
    """[first, last) row range of `rank` when n_values rows are split into
    whole 1024-value vectors as evenly as possible (strong scaling)."""
    n_vec = (n_values + 1023) // 1024
    per, extra = divmod(n_vec, world)
    v0 = rank * per + min(rank, extra)
    v1 = v0 + per + (1 if rank < extra else 0)
    return min(v0 * 1024, n_values), min(v1 * 1024, n_values)


def shard_seed(base: int, rank: int) -> int:
    """Seed of a rank's own shard of synthetic rows (weak scaling)."""
    return base * (rank + 1)


def allreduce_sum(t, group=None):
    """Sum a partial-aggregate tensor over all ranks, in place."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t
