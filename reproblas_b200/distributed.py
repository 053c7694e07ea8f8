"""Multi-GPU reproducible reductions: shard, reduce locally, exchange the binned states.

One process per GPU. Each rank reduces its contiguous shard of a vector into a fold-k
binned state (2k doubles, the reference layout) with the library's single-pass kernels;
the states are all-gathered (NCCL over NVLink on GPUs; any torch.distributed backend
works) and merged on every rank with the binned addition (binned_dbdbadd arithmetic,
rb_dbdbadd_states on the GPU). The binned state depends only on the multiset of
deposited values, so every rank obtains the bits a single GPU -- or the reference CPU
library -- computes for the whole vector, whatever the number of ranks or the merge
order. NCCL's built-in sum is not the binned addition and is never used on states.
"""
import torch
import torch.distributed as dist


def shard(n, rank, world):
    """Contiguous shard [start, start + length) of n elements for `rank` of `world`."""
    base, rem = divmod(n, world)
    start = rank * base + min(rank, rem)
    return start, base + (1 if rank < rem else 0)


def _gpu_merge(fold, count, gathered, out):
    import reproblas_b200 as rb
    rb.call("rb_dbdbadd_states", fold, count, gathered, out)


def allgather_merge(state, fold, group=None, merge=None):
    """All-gather the 2*fold-double binned `state` of every rank and return their binned
    sum (identical on every rank). `merge(fold, count, gathered, out)` adds `count`
    consecutive states of `gathered` into `out`; by default the GPU merge kernel."""
    world = dist.get_world_size(group)
    parts = [torch.empty_like(state) for _ in range(world)]
    dist.all_gather(parts, state.contiguous(), group=group)
    gathered = torch.cat(parts)
    out = torch.zeros_like(state)
    (merge or _gpu_merge)(fold, world, gathered, out)
    return out
