"""The device stream slicer (alto_slicer_*) against the oracle's restatement
of the reference's StreamingSparseTensor, which the CPU tests pin to the
compiled reference's batches.  Integer work: batches must be identical
(dims, every index, every value bit)."""
import os
import sys

import numpy as np
import pytest

import alto_b200 as A
import oracle as O
from alto_b200 import synth

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402

pytestmark = pytest.mark.gpu


def gpu_batches(dims, cidx, vals, t, thr, lim, device=False):
    if device:
        import torch

        ci = [torch.as_tensor(np.ascontiguousarray(c).astype(np.int64), device="cuda") for c in cidx]
        v = torch.as_tensor(vals, device="cuda")
        sl = A.Slicer(dims, ci, v, t)
    else:
        sl = A.Slicer(dims, cidx, vals, t)
    out = []
    while True:
        b = sl.next(thr, lim)
        if b is None:
            break
        c, v = b.to_host()
        out.append(dict(dims=b.dims.copy(), cidx=c, vals=v))
    assert sl.last_batch()
    return out, sl


def assert_same(gpu, ora):
    assert len(gpu) == len(ora)
    for k, (g, o) in enumerate(zip(gpu, ora)):
        assert np.array_equal(g["dims"], np.asarray(o["dims"], np.uint64)), k
        assert np.array_equal(g["cidx"], np.asarray(o["cidx"], np.uint64)), k
        assert np.array_equal(g["vals"], np.asarray(o["vals"])), k


def test_slicer_golden_digests(golden):
    """The committed digests of the reference's batches (same tensor and cases)."""
    dims = np.array([12, 40, 30, 20], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 2500, seed=3)
    for case in golden["slicer"]:
        b, _ = gpu_batches(dims, cidx, vals, case["stream_mode"], case["nnz_threshold"], case["timeslice_limit"])
        assert len(b) == case["batches"], case
        assert MG.slicer_digest(b) == case["sha256"], case


@pytest.mark.parametrize("t,thr,lim", MG.SLICER_CASES)
@pytest.mark.parametrize("device", [False, True])
def test_slicer_matches_oracle(t, thr, lim, device):
    dims = np.array([12, 40, 30, 20], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 2500, seed=3)
    g, _ = gpu_batches(dims, cidx, vals, t, thr, lim, device=device)
    assert_same(g, O.slice_stream(dims, cidx, vals, t, thr, lim))


def test_slicer_128bit_key_power_law():
    """Key wider than 64 bits (23 + 23 + 22 + 10), power-law indices, float32 values."""
    dims = np.array([1 << 23, 1 << 23, 3_000_000, 1000], np.uint64)
    cidx, vals = synth.powerlaw_coo(dims, 200_000, [1.1, 1.1, 1.2, 0.5], seed=5)
    vals = vals.astype(np.float32)
    # (stream mode 3 puts modes 2, 1, 0 at bits 0, 22, 45: mode 0 straddles the two words)
    for t, thr, lim in [(3, 1, 1), (3, 5000, 50)]:
        g, _ = gpu_batches(dims, cidx, vals, t, thr, lim)
        assert_same(g, O.slice_stream(dims, cidx, vals, t, thr, lim))


def test_slicer_gaps_duplicates_one_row_modes():
    """Empty time steps (batches of nnz 0), repeated coordinates (stable
    order kept), a one-row mode and uint32 input indices."""
    rng = np.random.default_rng(11)
    dims = np.array([30, 1, 17, 9], np.uint64)
    n = 900
    steps = rng.choice(np.array([2, 3, 7, 8, 20, 29], np.uint64), n)
    cidx = np.stack([steps, np.zeros(n, np.uint64), rng.integers(0, 17, n).astype(np.uint64),
                     rng.integers(0, 9, n).astype(np.uint64)])
    cidx[:, 100:200] = cidx[:, 0:100]  # exact duplicates
    vals = rng.random(n)
    for t, thr, lim in [(0, 1, 1), (0, 50, 4), (0, 10**6, 10**6), (2, 1, 1)]:
        g, _ = gpu_batches(dims, cidx.astype(np.uint32), vals, t, thr, lim)
        assert_same(g, O.slice_stream(dims, cidx, vals, t, thr, lim))


def test_slicer_empty_tensor_and_bad_index():
    dims = np.array([5, 6, 7], np.uint64)
    sl = A.Slicer(dims, np.zeros((3, 0), np.uint64), np.zeros(0), 0)
    assert sl.next(1, 1) is None and sl.last_batch()
    sl.close()
    cidx = np.array([[0, 1, 4], [0, 6, 2], [1, 1, 1]], np.uint64)  # 6 >= dims[1]
    with pytest.raises(A.AltoError) as e:
        A.Slicer(dims, cidx, np.ones(3), 0)
    assert e.value.status == A.ERR_INVALID


def test_slicer_iperm_and_stream_prev():
    dims = np.array([12, 40, 30, 20], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 2500, seed=3)
    t = 0
    full = O.slice_stream(dims, cidx, vals, t, 10**9, 10**9)[0]
    sl = A.Slicer(dims, cidx, vals, t)
    # iperm: relabelled index -> original index, over the sorted tensor
    order = np.lexsort([cidx[m] for m in reversed([(t + k) % 4 for k in range(4)])])
    for m in (1, 2, 3):
        ip = sl.iperm(m)
        assert np.array_equal(ip[full["cidx"][m].astype(np.int64)], cidx[m][order])
    assert np.array_equal(sl.iperm(0), np.arange(12, dtype=np.uint64))
    # stream_prev(p) after k single-step batches: the last p steps, relative times
    assert sl.stream_prev(2) is None
    got = []
    for k in range(5):
        got.append(sl.next(1, 1))
    dims_last = got[-1].dims.copy()
    prev = sl.stream_prev(3)
    c, v = prev.to_host()
    want_c = np.concatenate([O.slice_stream(dims, cidx, vals, t, 1, 1)[k]["cidx"] for k in (2, 3, 4)], axis=1)
    want_c[t] = np.concatenate([np.full(O.slice_stream(dims, cidx, vals, t, 1, 1)[k]["cidx"].shape[1], k - 2,
                                        np.uint64) for k in (2, 3, 4)])
    assert np.array_equal(c, want_c)
    assert prev.dims[t] == 3
    assert np.array_equal(np.delete(prev.dims, t), np.delete(dims_last, t))
    sl.close()


@pytest.mark.parametrize("model", [A.CPSTREAM, A.SPCPSTREAM])
def test_cpstream_fed_by_device_slicer_matches_host_batches(model):
    """CP-stream and spCP-stream over the device slicer's batches (device
    memory, uint32 indices) give bit-identical factors to the same batches
    from the host."""
    dims = np.array([12, 40, 30, 20], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 2500, seed=3)
    R, t = 8, 0
    rng = np.random.default_rng(4)
    iv = rng.random(4096 * R)
    host = O.slice_stream(dims, cidx, vals, t, 300, 3)

    def run(feed):
        s = A.CPStream(4, t, R, constraint=A.NONNEG, max_inner=10, epsilon=1e-5)
        s.set_model(model)
        prev = np.zeros(4, np.int64)
        used = 0
        for b in feed():
            d = np.asarray(b.dims if isinstance(b, A.SliceBatch) else b["dims"]).astype(np.int64)
            need = int(np.sum(np.maximum(d - prev, 0))) * R
            if isinstance(b, A.SliceBatch):
                s.push_batch(b, iv[used:used + need])
            else:
                s.push(b["dims"], b["cidx"], b["vals"], iv[used:used + need])
            used += need
            prev = np.maximum(prev, d)
        outs = [s.factor(m, int(prev[m]) if m != t else int(sum(int(b["dims"][t]) for b in host)))
                for m in range(4)]
        s.close()
        return outs

    def dev():
        sl = A.Slicer(dims, cidx, vals, t)
        while True:
            b = sl.next(300, 3)
            if b is None:
                return
            yield b

    a = run(lambda: iter(host))
    b = run(dev)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("model", [A.CPSTREAM, A.SPCPSTREAM])
def test_stream_error_matches_reference(model):
    """cpd_error of the streamed model against the whole tensor and against
    stream_prev's last steps (compute_errorsq), on the device, against the
    oracle and the compiled reference fed the same factor values."""
    dims = np.array([12, 40, 30, 20], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 2500, seed=3)
    R, t = 8, 0
    iv = np.random.default_rng(4).random(4096 * R)
    s = A.CPStream(4, t, R, constraint=A.NONNEG, max_inner=10, epsilon=1e-5)
    s.set_model(model)
    sl = A.Slicer(dims, cidx, vals, t)
    prev, used = np.zeros(4, np.int64), 0
    while (b := sl.next(300, 3)) is not None:
        d = b.dims.astype(np.int64)
        need = int(np.sum(np.maximum(d - prev, 0))) * R
        s.push_batch(b, iv[used:used + need])
        used += need
        prev = np.maximum(prev, d)
    F = [s.factor(0, 12)] + [np.vstack([s.factor(m, int(prev[m])), np.zeros((int(dims[m] - prev[m]), R))])
                             for m in (1, 2, 3)]
    X = sl.tensor()
    c, v = X.to_host()
    err = s.error(X)
    want = O.cpd_error(c, v, F)
    assert abs(err - want) <= 1e-10 * max(1.0, want)
    assert abs(O.ref_cpd_error(dims, c, v, F) - want) <= 1e-12 * max(1.0, want)
    P = sl.stream_prev(3)  # the last three time steps against the last three time rows
    pc, pv = P.to_host()
    e3 = s.error(P)
    want3 = O.cpd_error(pc, pv, [F[0][-3:]] + F[1:])
    assert abs(e3 - want3) <= 1e-10 * max(1.0, want3)
    s.close()
    sl.close()


def test_cut_all_equals_repeated_next():
    """alto_slicer_cut_all makes the cuts repeated next() calls make, with the
    same batch contents, including empty time steps; stream_prev and the end
    state follow."""
    rng = np.random.default_rng(12)
    dims = np.array([40, 30, 20, 10], np.uint64)
    n = 3000
    steps = rng.choice(np.array([0, 1, 4, 5, 6, 9, 17, 30, 31, 39], np.uint64), n)
    cidx = np.stack([steps] + [rng.integers(0, int(d), n).astype(np.uint64) for d in dims[1:]])
    vals = rng.random(n)
    for thr, lim in [(1, 1), (200, 3), (10**9, 7)]:
        want, _ = gpu_batches(dims, cidx, vals, 0, thr, lim)
        sl = A.Slicer(dims, cidx, vals, 0)
        nb = sl.cut_all(thr, lim)
        assert nb == len(want) and sl.last_batch() and sl.next(thr, lim) is None
        for k in range(nb):
            b = sl.batch(k)
            c, v = b.to_host()
            assert np.array_equal(b.dims, want[k]["dims"]) and np.array_equal(c, want[k]["cidx"])
            assert np.array_equal(v, want[k]["vals"])
        p = sl.stream_prev(5)
        assert p is not None and p.dims[0] == 5
        sl.close()
