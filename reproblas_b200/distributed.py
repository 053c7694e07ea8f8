"""Multi-GPU reproducible reductions: shard, reduce locally, exchange the binned states.

One process per GPU. Each rank reduces its contiguous shard of a vector into a binned
state (the reference layout) with the library's single-pass kernels; the states are
all-gathered (NCCL over NVLink on GPUs; any torch.distributed backend works) and merged on
every rank with the binned addition on the GPU (rb_*_states, the arithmetic of the
reference's binnedMPI operations). The binned state depends only on the multiset of
deposited values, so every rank obtains the bits a single GPU -- or the reference CPU
library -- computes for the whole vector, whatever the number of ranks or the merge order.
NCCL's built-in sum is not the binned addition and is never used on states.

State kinds and their per-rank record (elements of the state's real type):
  "d"   double_binned, 2*fold doubles            (binnedMPI_DBDBADD,   rb_dbdbadd_states)
  "s"   float_binned, 2*fold floats              (binnedMPI_SBSBADD,   rb_sbsbadd_states)
  "z"   double_complex_binned, 4*fold doubles    (binnedMPI_ZBZBADD,   rb_zbzbadd_states)
  "c"   float_complex_binned, 4*fold floats      (binnedMPI_CBCBADD,   rb_cbcbadd_states)
  "dsq" [scale, double_binned], 1 + 2*fold       (binnedMPI_DBDBADDSQ, rb_dbdbaddsq_states)
  "ssq" [scale, float_binned], 1 + 2*fold        (binnedMPI_SBSBADDSQ, rb_sbsbaddsq_states)
The scaled records carry the sums of squares of the 2-norms (binnedBLAS_dbdssq returns the
scale, the state holds the scaled squares); nrm2 = scale * sqrt(conv(state)).
"""
import torch
import torch.distributed as dist

KINDS = {
    "d": "rb_dbdbadd_states", "s": "rb_sbsbadd_states", "z": "rb_zbzbadd_states",
    "c": "rb_cbcbadd_states", "dsq": "rb_dbdbaddsq_states", "ssq": "rb_sbsbaddsq_states",
}


def record_len(kind, fold):
    """Elements of one state record of `kind` at `fold`."""
    return {"d": 2 * fold, "s": 2 * fold, "z": 4 * fold, "c": 4 * fold,
            "dsq": 1 + 2 * fold, "ssq": 1 + 2 * fold}[kind]


def shard(n, rank, world):
    """Contiguous shard [start, start + length) of n elements for `rank` of `world`."""
    base, rem = divmod(n, world)
    start = rank * base + min(rank, rem)
    return start, base + (1 if rank < rem else 0)


def _gpu_merge(kind):
    def merge(fold, count, gathered, out):
        import reproblas_b200 as rb
        rb.call(KINDS[kind], fold, count, gathered, out)
    return merge


def allgather_merge(state, fold, group=None, merge=None, kind="d"):
    """All-gather the binned `state` record (record_len(kind, fold) elements) of every rank
    and return their binned sum (identical on every rank). `merge(fold, count, gathered,
    out)` adds `count` consecutive records of `gathered` into `out`; by default the GPU merge
    of that kind."""
    if kind not in KINDS:
        raise ValueError("unknown state kind %r" % (kind,))
    if state.numel() != record_len(kind, fold):
        raise ValueError("state has %d elements, a %s record of fold %d has %d"
                         % (state.numel(), kind, fold, record_len(kind, fold)))
    world = dist.get_world_size(group)
    parts = [torch.empty_like(state) for _ in range(world)]
    dist.all_gather(parts, state.contiguous(), group=group)
    gathered = torch.cat(parts)
    out = torch.zeros_like(state)
    (merge or _gpu_merge(kind))(fold, world, gathered, out)
    return out
