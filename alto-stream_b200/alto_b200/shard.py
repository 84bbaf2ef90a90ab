"""Sharded MTTKRP over several GPUs (one process per GPU, torch.distributed).

Each rank keeps a contiguous range of the tensor's ALTO line -- the
reference's partition rule for threads (prtn_alto, include/alto.hpp:1128-1160)
applied to ranks -- runs its MTTKRP into a full-size output, and an
all-reduce (sum) over the ranks gives the tensor's MTTKRP.  Output rows of
different ranks overlap only where their line ranges share rows, but the
collective is a plain all-reduce of the I_n x R float32 output (NCCL over
NVLink on GPUs, gloo on CPUs).  The factors are replicated on every rank.

CP-stream serving shards differently: independent streams go to different
GPUs whole (streams_for_rank), each GPU running its own server, and no data
crosses GPUs (one slice's update is too small to split).
"""
from __future__ import annotations


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
