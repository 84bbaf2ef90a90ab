"""The CP-stream server: every stream's result is the same processed alone
and in a mix with other streams -- bit for bit, since CP-stream sessions use
the deterministic MTTKRP and fixed-order reductions throughout (the stated
bound is 1e-4) --, slices of one stream keep their order, admission respects
the HBM budget, and the alone result matches the FP64 oracle within 1e-4."""
import threading
import time

import numpy as np
import pytest

import alto_b200 as A
import oracle as O
from alto_b200 import synth

pytestmark = pytest.mark.gpu


def make_stream(seed, space, nslices, rank):
    b = synth.stream_batches(space, nslices, lambda rng, s: 300 + 40 * s, [1.1, None, 1.2], seed=seed,
                             values="uniform")
    n_init = sum(int(x) for x in b[-1]["dims"]) * rank + 64
    return b, synth.init_values(n_init, seed=seed + 100)


def submit_all(srv, sid, batches, iv, rank):
    used, prev, tickets = 0, np.zeros(len(batches[0]["dims"]), np.int64), []
    for b in batches:
        d = b["dims"].astype(np.int64)
        need = int(np.sum(np.maximum(d - prev, 0))) * rank
        tickets.append(srv.submit(sid, b["dims"], b["cidx"], b["vals"], iv[used:used + need]))
        used += need
        prev = np.maximum(prev, d)
    return tickets


def normwise(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


SPECS = [(11, [150, 200, 40], 8, A.NONNEG), (12, [300, 120, 60], 16, A.UNCONSTRAINED),
         (13, [90, 400, 30], 8, A.UNCONSTRAINED), (14, [250, 250, 50], 16, A.NONNEG)]


def run(specs, workers):
    srv = A.Server(8 << 30, workers=workers)
    sids, streams = [], []
    for seed, space, rank, con in specs:
        b, iv = make_stream(seed, space, 5, rank)
        sid = srv.open(4, 0, rank, [len(b)] + [int(x) for x in b[-1]["dims"][1:]], 2000, constraint=con,
                       forgetting=0.99, max_inner=10, epsilon=1e-5)
        sids.append(sid)
        streams.append((b, iv, rank))
    tickets = [submit_all(srv, sid, b, iv, rank) for sid, (b, iv, rank) in zip(sids, streams)]
    srv.drain()
    out = [[srv.factor(sid, m) for m in range(4)] for sid in sids]
    st = srv.stats()
    srv.destroy()
    return out, st, tickets


def test_each_result_same_alone_and_in_the_mix():
    mix, st, _ = run(SPECS, workers=4)
    assert st["completed"] == 5 * len(SPECS)
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for k, spec in enumerate(SPECS):
        alone, _, _ = run([spec], workers=1)
        for a, m in zip(alone[0], mix[k]):
            assert a.shape == m.shape
            assert np.array_equal(m, a), (k, normwise(m, a))


def test_served_results_equal_the_plain_path():
    """Slices served in stream groups (every kernel over many streams'
    slices) give the same factors, bit for bit, as each stream pushed alone
    through its own session, for several ranks, both constraints and enough
    streams that groups hold several slices at once."""
    specs = SPECS + [(15, [120, 80, 30], 32, A.NONNEG), (16, [60, 300, 20], 32, A.UNCONSTRAINED),
                     (17, [200, 90, 25], 16, A.UNCONSTRAINED), (18, [80, 80, 80], 8, A.NONNEG)]
    mix, st, _ = run(specs, workers=3)
    assert st["completed"] == 5 * len(specs)
    for k, (seed, space, rank, con) in enumerate(specs):
        b, iv = make_stream(seed, space, 5, rank)
        s = A.CPStream(4, 0, rank, constraint=con, forgetting=0.99, max_inner=10, epsilon=1e-5)
        used, prev = 0, np.zeros(4, np.int64)
        for x in b:
            d = x["dims"].astype(np.int64)
            need = int(np.sum(np.maximum(d - prev, 0))) * rank
            s.push(x["dims"], x["cidx"], x["vals"], iv[used:used + need])
            used += need
            prev = np.maximum(prev, d)
        for m in range(4):
            rows = len(b) if m == 0 else int(b[-1]["dims"][m])
            assert np.array_equal(s.factor(m, rows), mix[k][m]), (k, m)
        s.close()


def test_alone_result_matches_oracle():
    seed, space, rank, con = SPECS[0]
    res, _, _ = run([SPECS[0]], workers=1)
    b, iv = make_stream(seed, space, 5, rank)
    bo = [dict(dims=x["dims"], cidx=x["cidx"], vals=x["vals"].astype(np.float32).astype(np.float64)) for x in b]
    oo, _, _ = O.cpstream(bo, 0, rank, 10, 1e-5, con == A.NONNEG, iv.astype(np.float32).astype(np.float64))
    for g, o in zip(res[0], oo):
        assert normwise(g, o) <= 1e-4


def test_admission_waits_for_budget():
    srv = A.Server(1, workers=2)  # room for one stream at a time
    b1, iv1 = make_stream(21, [100, 100, 20], 3, 8)
    b2, iv2 = make_stream(22, [100, 100, 20], 3, 8)
    s1 = srv.open(4, 0, 8, [3, 200, 200, 40], 1000)
    s2 = srv.open(4, 0, 8, [3, 200, 200, 40], 1000)
    st = srv.stats()
    assert st["admitted_streams"] == 1 and st["pending_streams"] == 1
    t2 = submit_all(srv, s2, b2, iv2, 8)
    submit_all(srv, s1, b1, iv1, 8)
    srv.drain()
    assert srv.stats()["completed"] == 3  # only the admitted stream ran
    assert srv.poll(t2[-1]) is None  # queued behind the budget
    srv.close(s1)
    got = srv.wait(t2[-1])
    assert srv.stats()["completed"] == 6
    assert got[0] >= 1
    with pytest.raises(A.AltoError):  # a ticket is handed back once
        srv.poll(t2[-1])
    srv.close(s2)
    srv.destroy()


def test_close_of_pending_stream_wakes_its_waiters():
    srv = A.Server(1, workers=1)  # room for one stream at a time
    b1, iv1 = make_stream(31, [100, 100, 20], 2, 8)
    b2, iv2 = make_stream(32, [100, 100, 20], 2, 8)
    s1 = srv.open(4, 0, 8, [3, 200, 200, 40], 1000)
    s2 = srv.open(4, 0, 8, [3, 200, 200, 40], 1000)
    assert srv.stats()["pending_streams"] == 1
    t2 = submit_all(srv, s2, b2, iv2, 8)
    out = {}

    def waiter():
        try:
            srv.wait(t2[0])
            out["status"] = "ok"
        except A.AltoError as e:
            out["status"] = e.status

    th = threading.Thread(target=waiter)
    th.start()
    time.sleep(0.2)
    assert th.is_alive()  # blocked: s2 is not admitted
    srv.close(s2)  # drops s2's queued slices
    th.join(timeout=30)
    assert not th.is_alive(), "waiter still blocked after close"
    assert out["status"] == A.ERR_INVALID
    with pytest.raises(A.AltoError) as e:
        srv.poll(t2[1])
    assert e.value.status == A.ERR_INVALID
    submit_all(srv, s1, b1, iv1, 8)
    srv.drain()
    srv.close(s1)
    srv.destroy()
