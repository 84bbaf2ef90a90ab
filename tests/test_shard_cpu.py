"""Sharded MTTKRP host logic on CPU: two gloo ranks each keep their line
range of the ALTO order (the reference's partition rule), compute their
partial MTTKRP with the FP64 oracle, and the all-reduce of the outputs
equals the whole tensor's MTTKRP."""
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, q):
    import sys

    sys.path.insert(0, os.path.join(ROOT, "alto-stream_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist

    import oracle as O
    from alto_b200 import shard, synth

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dims = np.array([400, 300, 200], np.uint64)
        cidx, vals = synth.powerlaw_coo(dims, 20000, [1.2, None, 1.1], seed=9)
        R = 8
        rng = np.random.default_rng(2)
        F = [rng.uniform(-1, 1, (int(d), R)) for d in dims]
        enc = O.build(dims, cidx, vals)
        b, e = shard.partition_range(enc["nnz"], rank, world)
        part = dict(enc, nnz=e - b, idx=enc["idx"][b:e], vals=enc["vals"][b:e])
        errs = []
        for m in range(3):
            fs = [f.copy() for f in F]
            fs[m][:] = 0
            mine = O.mttkrp(part, m, fs, R)[m]
            out = torch.from_numpy(np.ascontiguousarray(mine))
            shard.allreduce_output(out)
            fs = [f.copy() for f in F]
            fs[m][:] = 0
            full = O.mttkrp(enc, m, fs, R)[m]
            errs.append(float(np.abs(out.numpy() - full).max() / np.abs(full).max()))
        q.put((rank, (b, e), errs))
    finally:
        dist.destroy_process_group()


def test_partition_range_rule():
    from alto_b200 import shard

    assert [shard.partition_range(10, p, 4) for p in range(4)] == [(0, 3), (3, 6), (6, 9), (9, 10)]
    assert [shard.partition_range(5, p, 4) for p in range(4)] == [(0, 2), (2, 4), (4, 5), (5, 5)]
    with pytest.raises(ValueError):
        shard.partition_range(5, 4, 4)


def test_two_rank_sharded_mttkrp_equals_whole():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (_, r0, e0), (_, r1, e1) = res
    assert r0[0] == 0 and r0[1] == r1[0] and r1[1] > r1[0]
    assert max(e0 + e1) <= 1e-12


def test_streams_for_rank_cover_every_stream_once():
    from alto_b200 import shard

    for world in (1, 2, 3, 8):
        got = sorted(k for r in range(world) for k in shard.streams_for_rank(64, r, world))
        assert got == list(range(64))
        sizes = [len(shard.streams_for_rank(64, r, world)) for r in range(world)]
        assert max(sizes) - min(sizes) <= 1
