"""Sharded MTTKRP host logic on CPU, with two gloo ranks and the FP64
oracle as each rank's local MTTKRP:

* by output-row blocks (the multi-GPU bench path): each rank's own tensor
  per mode, disjoint outputs, a row all-gather;
* by line range (the reference's partition rule): partial outputs summed by
  an all-reduce."""
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


def rank_main_rows(rank, world, port, q):
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
        res = []
        for m in range(3):
            counts = np.bincount(cidx[m].astype(np.int64), minlength=int(dims[m]))
            b = shard.row_blocks(counts, world)
            c_r, v_r = shard.select_block(cidx, vals, m, b[rank], b[rank + 1])
            fs = [f.copy() for f in F]
            fs[m][:] = 0
            mine = O.mttkrp(O.build(dims, c_r, v_r), m, fs, R)[m]  # this rank's own tensor
            outside = np.ones(int(dims[m]), bool)
            outside[b[rank]:b[rank + 1]] = False
            untouched = bool(np.all(mine[outside] == 0))
            out = torch.from_numpy(np.ascontiguousarray(mine))
            shard.allgather_rows(out, b)
            fs = [f.copy() for f in F]
            fs[m][:] = 0
            full = O.mttkrp(enc, m, fs, R)[m]
            res.append((b, int(c_r.shape[1]), untouched, bool(np.array_equal(out.numpy(), full)),
                        int(counts.max())))
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_row_blocks_rule():
    from alto_b200 import shard

    assert shard.row_blocks([5, 5, 5, 5], 2) == [0, 2, 4]
    assert shard.row_blocks([10, 0, 0, 0, 10], 2) == [0, 1, 5]
    assert shard.row_blocks([1, 1, 1], 4) == [0, 1, 2, 3, 3]  # more ranks than rows: empty blocks
    assert shard.row_blocks([0, 0], 2) == [0, 0, 2]
    b = shard.row_blocks(np.arange(100), 8)
    assert b[0] == 0 and b[-1] == 100 and all(x <= y for x, y in zip(b, b[1:]))


def test_two_rank_row_block_mttkrp_equals_whole():
    """Each rank encodes only the nonzeros of its row block of each mode;
    its MTTKRP touches only its rows, and after the row all-gather every
    rank holds the whole tensor's MTTKRP bit for bit (each row is summed by
    one rank in the same order as on the whole tensor)."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main_rows, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for m in range(3):
        (b0, n0, u0, eq0, top), (b1, n1, u1, eq1, _) = res[0][m], res[1][m]
        assert b0 == b1
        assert n0 + n1 == 20000 and n0 > 0 and n1 > 0
        assert abs(n0 - 10000) <= top  # equal halves, up to the one row at the cut
        assert u0 and u1 and eq0 and eq1


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
