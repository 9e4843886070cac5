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


def combine_group_records(res, stride: int, sum_slot: int, sum_bits: int = 64, group=None):
    """Combine the ranks' group records in place: key words are equal on every
    rank that saw a group and 0 on the others (payloads are >= 0), so they
    combine by MAX; the sums add (an int64 at words sum_slot, sum_slot + 1, or
    a wrapping int32 at word sum_slot, added as int64 and wrapped back)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1):
        return res
    rec = res.view(-1, stride)
    sw = 1 if sum_bits == 32 else 2
    is_sum = torch.zeros(stride, dtype=torch.bool, device=res.device)
    is_sum[sum_slot:sum_slot + sw] = True
    if stride > sw:
        keys = rec[:, ~is_sum].contiguous()
        dist.all_reduce(keys, op=dist.ReduceOp.MAX, group=group)
        rec[:, ~is_sum] = keys
    if sw == 2:
        sums = rec[:, sum_slot:sum_slot + 2].contiguous().view(torch.int64)
    else:
        sums = rec[:, sum_slot].to(torch.int64)
    dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    if sw == 2:
        rec[:, sum_slot:sum_slot + 2] = sums.view(torch.int32)
    else:
        rec[:, sum_slot] = (((sums + (1 << 31)) % (1 << 32)) - (1 << 31)).to(torch.int32)
    return res
