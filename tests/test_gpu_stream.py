"""GPU CP-stream (unconstrained and non-negative ADMM) against the oracle
and the reference's recorded factor norms.  Bound: final factors within
1e-4 normwise of the FP64 oracle fed the same batches and initial values."""
import numpy as np
import pytest

import alto_b200 as A
import oracle as O
from alto_b200 import synth
from conftest import load_stream_fixture

pytestmark = pytest.mark.gpu


def run_gpu(batches, R, max_iters, eps, nonneg, iv, forgetting=0.99, graph=True):
    N = len(batches[0]["dims"])
    s = A.CPStream(N, 0, R, constraint=A.NONNEG if nonneg else A.UNCONSTRAINED, forgetting=forgetting,
                   max_inner=max_iters, epsilon=eps)
    s.set_graph(graph)
    used = 0
    prev = np.zeros(N, np.int64)
    inner = []
    for b in batches:
        d = b["dims"].astype(np.int64)
        need = int(np.sum(np.maximum(d - prev, 0))) * R
        inner.append(s.push(b["dims"], b["cidx"], b["vals"], iv[used:used + need]))
        used += need
        prev = np.maximum(prev, d)
    outs = []
    for m in range(N):
        rows = int(sum(int(b["dims"][0]) for b in batches)) if m == 0 else int(batches[-1]["dims"][m])
        outs.append(s.factor(m, rows))
    return outs, s.lam(), inner


def normwise(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("nonneg", [0, 1])
def test_small_stream_matches_oracle_and_reference(nonneg, golden):
    g = golden[f"cpstream_small_nonneg{nonneg}"]
    b = load_stream_fixture()
    iv = synth.init_values(g["n_init"], seed=g["init_seed"])
    R = g["rank"]
    outs, lam, inner = run_gpu(b, R, g["max_iters"], g["eps"], nonneg, iv)
    ivo = iv.astype(np.float32).astype(np.float64)
    bo = [dict(dims=x["dims"], cidx=x["cidx"], vals=x["vals"].astype(np.float32).astype(np.float64)) for x in b]
    oo, lo, inner_o = O.cpstream(bo, 0, R, g["max_iters"], g["eps"], nonneg, ivo)
    for a, c in zip(outs, oo):
        assert normwise(a, c) <= 1e-4, normwise(a, c)
    np.testing.assert_allclose([np.linalg.norm(o) for o in outs], g["norms"], rtol=1e-4)
    if nonneg:
        assert all(np.all(o >= 0) for m, o in enumerate(outs) if m != 0)


def test_forgetting_factor_is_a_parameter():
    b = load_stream_fixture()[:3]
    R = 8
    iv = synth.init_values(20000, seed=1)
    o1, _, _ = run_gpu(b, R, 10, 1e-5, 0, iv, forgetting=0.95)
    bo = [dict(dims=x["dims"], cidx=x["cidx"], vals=x["vals"].astype(np.float32).astype(np.float64)) for x in b]
    oo, _, _ = O.cpstream(bo, 0, R, 10, 1e-5, 0, iv.astype(np.float32).astype(np.float64), forgetting=0.95)
    for a, c in zip(o1, oo):
        assert normwise(a, c) <= 1e-4


def test_stream_repeats_bit_for_bit():
    """Two sessions fed the same slices end with identical factors and
    lambda, and take the same inner iterations."""
    b = load_stream_fixture()[:4]
    iv = synth.init_values(20000, seed=3)
    o1, l1, i1 = run_gpu(b, 8, 10, 1e-5, 1, iv, forgetting=0.95)
    o2, l2, i2 = run_gpu(b, 8, 10, 1e-5, 1, iv, forgetting=0.95)
    assert i1 == i2 and np.array_equal(l1, l2)
    for a, c in zip(o1, o2):
        assert np.array_equal(a, c)


@pytest.mark.parametrize("nonneg", [0, 1])
def test_graph_and_direct_launches_agree(nonneg):
    """The session's stream-group graph (all inner iterations of a batch in
    one relaunched graph over the session's descriptor: the grouped kernels,
    device-side inner loop and ADMM chunk loop) and the directly launched
    per-kernel loop give identical factors and iteration counts, bit for
    bit."""
    b = load_stream_fixture()[:4]
    iv = synth.init_values(20000, seed=4)
    og, lg, ig = run_gpu(b, 16, 10, 1e-5, nonneg, iv, forgetting=0.95, graph=True)
    od, ld, id_ = run_gpu(b, 16, 10, 1e-5, nonneg, iv, forgetting=0.95, graph=False)
    assert ig == id_ and np.array_equal(lg, ld)
    for a, c in zip(og, od):
        assert np.array_equal(a, c)


@pytest.mark.parametrize("graph", [True, False])
def test_session_stats_account_for_every_push(graph):
    """alto_stream_stats: the pushes and inner iterations it counts are those
    the pushes returned, the preparation's parts fit inside the preparation,
    and the inner iterations took device time."""
    b = load_stream_fixture()[:4]
    R = 8
    iv = synth.init_values(20000, seed=6)
    N = len(b[0]["dims"])
    s = A.CPStream(N, 0, R, constraint=A.NONNEG, forgetting=0.95, max_inner=10, epsilon=1e-5)
    s.set_graph(graph)
    used, prev, inner = 0, np.zeros(N, np.int64), []
    for x in b:
        d = x["dims"].astype(np.int64)
        need = int(np.sum(np.maximum(d - prev, 0))) * R
        inner.append(s.push(x["dims"], x["cidx"], x["vals"], iv[used:used + need]))
        used += need
        prev = np.maximum(prev, d)
    st = s.stats()
    s.close()
    assert st["pushes"] == len(b) and st["inner_iters"] == sum(inner)
    assert st["inner_device_ms"] > 0 and st["inner_ms"] > 0 and st["finish_ms"] >= 0
    assert st["grow_ms"] + st["encode_ms"] + st["sorted_copies_ms"] <= st["prepare_ms"] + 1e-6


# ------------------------------------------------------------ spCP-stream

def run_sparse(batches, R, max_iters, eps, iv, graph=True, constraint=A.UNCONSTRAINED):
    N = len(batches[0]["dims"])
    s = A.CPStream(N, 0, R, constraint=constraint, forgetting=0.99, max_inner=max_iters, epsilon=eps)
    s.set_model(A.SPCPSTREAM)
    s.set_graph(graph)
    used, prev, inner = 0, np.zeros(N, np.int64), []
    for b in batches:
        d = b["dims"].astype(np.int64)
        need = int(np.sum(np.maximum(d - prev, 0))) * R
        inner.append(s.push(b["dims"], b["cidx"], b["vals"], iv[used:used + need]))
        used += need
        prev = np.maximum(prev, d)
    outs = []
    for m in range(N):
        rows = int(sum(int(b["dims"][0]) for b in batches)) if m == 0 else int(batches[-1]["dims"][m])
        outs.append(s.factor(m, rows))
    s.close()
    return outs, inner


def test_spcpstream_matches_oracle_and_reference(golden):
    """Row-sparse updates (spcpstream_alto_iter) against the FP64 oracle fed
    the same float32 batches and initial values, and the reference's norms."""
    g = golden["spcpstream_small"]
    b = load_stream_fixture()
    iv = synth.init_values(g["n_init"], seed=g["init_seed"])
    outs, inner = run_sparse(b, g["rank"], g["max_iters"], g["eps"], iv)
    bo = [dict(dims=x["dims"], cidx=x["cidx"], vals=x["vals"].astype(np.float32).astype(np.float64)) for x in b]
    oo, _, inner_o = O.spcpstream(bo, 0, g["rank"], g["max_iters"], g["eps"],
                                  iv.astype(np.float32).astype(np.float64))
    assert list(inner) == list(inner_o)
    for a, c in zip(outs, oo):
        assert normwise(a, c) <= 1e-4, normwise(a, c)
    np.testing.assert_allclose([np.linalg.norm(o) for o in outs], g["norms"], rtol=1e-4)


def test_spcpstream_graph_direct_and_server_agree():
    b = load_stream_fixture()[:4]
    iv = synth.init_values(20000, seed=6)
    og, ig = run_sparse(b, 16, 10, 1e-5, iv, graph=True)
    od, id_ = run_sparse(b, 16, 10, 1e-5, iv, graph=False)
    on, in_ = run_sparse(b, 16, 10, 1e-5, iv, graph=True, constraint=A.NONNEG)  # not used by spCP-stream
    assert ig == id_ == in_
    for a, c, d in zip(og, od, on):
        assert np.array_equal(a, c) and np.array_equal(a, d)
    srv = A.Server(4 << 30, workers=2)
    sid = srv.open(4, 0, 16, [len(b)] + [int(x) for x in b[-1]["dims"][1:]], 2000, model=A.SPCPSTREAM)
    used, prev = 0, np.zeros(4, np.int64)
    for x in b:
        d = x["dims"].astype(np.int64)
        need = int(np.sum(np.maximum(d - prev, 0))) * 16
        srv.submit(sid, x["dims"], x["cidx"], x["vals"], iv[used:used + need])
        used += need
        prev = np.maximum(prev, d)
    srv.drain()
    for m in range(4):
        assert np.array_equal(srv.factor(sid, m), og[m])
    srv.destroy()


@pytest.mark.parametrize("model,label", [("cpstream_alto", "CPSTREAM"), ("spcpstream_alto", "spCPSTREAM")])
def test_cpd64_streaming_models(tmp_path, model, label):
    """The rebuilt cpd64 driver runs both streaming models of the reference's
    -l flag on a .tns file (1-based indices, time mode 0)."""
    import os
    import subprocess

    rng = np.random.default_rng(3)
    dims = [5, 40, 30, 20]
    n = 600
    cols = [rng.integers(0, d, n) for d in dims]
    key = cols[0] * 10**6 + cols[1] * 10**4 + cols[2] * 100 + cols[3]
    _, first = np.unique(key, return_index=True)
    path = tmp_path / "s.tns"
    with open(path, "w") as f:
        for q in sorted(first):
            f.write(" ".join(str(int(c[q]) + 1) for c in cols) + " %.6f\n" % rng.random())
    exe = os.path.join(os.path.dirname(A.__file__), "..", "cpd64")
    r = subprocess.run([exe, "-i", str(path), "-r", "8", "-m", "5", "-e", "1e-5", "-l", model, "-a", "0"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert f"{label} (ALTO) on the GPU: 5 batches" in r.stdout
    assert "final fit error: " in r.stdout
