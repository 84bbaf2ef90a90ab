"""Sharded MTTKRP over several GPUs (one process per GPU, torch.distributed).

Two decompositions:

* By output rows (the one bench.py runs under torchrun): for each mode n,
  the rows of mode n are cut into W contiguous blocks holding (as nearly as
  whole rows allow) equal nonzero counts (row_blocks), and rank r keeps, for
  mode n, exactly the nonzeros whose mode-n index falls in its block -- its
  own small tensor per mode (select_block), encoded on its GPU alone.  Its
  MTTKRP of mode n then owns every output row it writes, so no reduction is
  needed: each rank's rows go to every other rank (allgather_rows, one
  broadcast per rank's block), which moves half the bytes of an all-reduce
  of the I_n x R output and adds nothing.  This is the reference's
  row-ownership idea (da_mem_pull's per-partition output intervals,
  include/alto.hpp:1544-1634) taken to whole rows per GPU.
* By line range: each rank keeps a contiguous range of the ALTO line -- the
  reference's partition rule for threads (prtn_alto,
  include/alto.hpp:1128-1160) applied to ranks -- runs its MTTKRP into a
  full-size output, and an all-reduce (sum) gives the tensor's MTTKRP.

The factors are replicated on every rank.  Collectives are NCCL over NVLink
on GPUs, gloo on CPUs.

CP-stream serving shards differently: independent streams go to different
GPUs whole (streams_for_rank), each GPU running its own server, and no data
crosses GPUs (one slice's update is too small to split).
"""
from __future__ import annotations


def row_blocks(counts, world):
    """Boundaries b_0 = 0 <= b_1 <= ... <= b_W = len(counts) of W contiguous
    row blocks of one mode: b_r is the first row with at least r/W of the
    nonzeros before it (counts: nonzeros per row; numpy or torch)."""
    import numpy as np

    c = np.asarray(counts.cpu() if hasattr(counts, "cpu") else counts, dtype=np.int64)
    before = np.concatenate([[0], np.cumsum(c)])  # nonzeros in rows < i
    total = int(before[-1])
    b = [int(np.searchsorted(before, -(-r * total // world), side="left")) for r in range(world)]
    b = [min(x, len(c)) for x in b] + [len(c)]
    b[0] = 0
    return b


def select_block(cidx, vals, mode, lo, hi):
    """The nonzeros whose `mode` index lies in [lo, hi) (torch or numpy)."""
    sel = (cidx[mode] >= lo) & (cidx[mode] < hi)
    return cidx[:, sel], vals[sel]


def allgather_rows(out, bounds, group=None):
    """Every rank's block of rows of `out` (rows [b_r, b_{r+1}) written by
    rank r) to every rank, in place: one broadcast per rank's block."""
    import torch.distributed as dist

    for r in range(len(bounds) - 1):
        lo, hi = bounds[r], bounds[r + 1]
        if hi > lo:
            dist.broadcast(out[lo:hi], src=r, group=group)
    return out


def partition_range(nnz, part, nparts):
    """[begin, end) of partition `part` of `nparts` over nnz line entries:
    ceil(nnz / P) entries each, the last ones possibly short or empty
    (include/alto.hpp:1134-1160)."""
    if not 0 <= part < nparts:
        raise ValueError("part outside 0..nparts-1")
    per = (int(nnz) + nparts - 1) // nparts
    return min(part * per, int(nnz)), min((part + 1) * per, int(nnz))


def streams_for_rank(nstreams, rank, world):
    """The serving streams rank `rank` of `world` serves: stream k on rank
    k mod world (round robin, so ranks differ by at most one stream)."""
    if not 0 <= rank < world:
        raise ValueError("rank outside 0..world-1")
    return list(range(rank, int(nstreams), world))


def shard_tensor(tensor, rank, world, stream=None):
    """Restrict an AltoTensor (built from the whole tensor on every rank) to
    this rank's line range."""
    b, e = partition_range(tensor.nnz, rank, world)
    return tensor.restrict(b, e, stream=stream)


def allreduce_output(out, group=None):
    """Sum a rank's partial MTTKRP output over the ranks, in place."""
    import torch.distributed as dist

    dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out


def sharded_mttkrp(shard, mode, factors, rank, out=None, group=None, variant=0, stream=None):
    """MTTKRP of `mode` of the whole tensor from this rank's shard: the local
    MTTKRP, then the all-reduce of the output."""
    out = shard.mttkrp(mode, factors, rank, out=out, variant=variant, stream=stream)
    return allreduce_output(out, group)
