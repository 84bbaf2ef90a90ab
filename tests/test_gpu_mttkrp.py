"""GPU MTTKRP against the FP64 oracle.

The oracle receives the factor values the GPU reads (float32, or bfloat16
for the BF16 path, widened to float64), so the comparison isolates the
float32 accumulation.  Bound: max |gpu - oracle| / max |oracle| <= 1e-5
(normwise) for every mode, rank and variant."""
import numpy as np
import pytest

import alto_b200 as A
import oracle as O
from alto_b200 import synth
from conftest import FIXTURE_NAMES, load_fixture

pytestmark = pytest.mark.gpu
TOL = 1e-5
ALL_VARIANTS = (A.AUTO, A.ATOMIC, A.STAGED, A.SORTED, A.ATOMIC | A.FEED_BULK, A.SORTED | A.FEED_BULK)
# the row-sorted walks that exist for 3-mode tensors only
THREE_MODE_FEEDS = (A.SORTED | A.FEED_DENSE, A.SORTED | A.FEED_FIXED_TARGET)


def to_dev(F, dtype):
    import torch

    return [torch.tensor(f, dtype=torch.float32, device="cuda").to(dtype).contiguous() for f in F]


def seen_by_gpu(Fd):
    return [f.float().cpu().numpy().astype(np.float64) for f in Fd]


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def check_modes(dims, cidx, vals, R, variants=(A.AUTO,), dtype=None, seed=0):
    import torch

    dtype = dtype or torch.float32
    rng = np.random.default_rng(seed)
    F = [rng.uniform(-1.0, 1.0, (int(d), R)) for d in dims]
    Fd = to_dev(F, dtype)
    Fo = seen_by_gpu(Fd)
    t = A.create_alto(dims, cidx, vals)
    vals32 = vals.astype(np.float32).astype(np.float64)
    enc = O.build(dims, cidx, vals32)
    for m in range(len(dims)):
        fs = [f.copy() for f in Fo]
        fs[m][:] = 0
        ref = O.mttkrp(enc, m, fs, R)[m]
        extra = THREE_MODE_FEEDS if len(dims) == 3 and A.SORTED in variants else ()
        for v in tuple(variants) + extra:
            out = t.mttkrp(m, Fd, R, variant=v).cpu().numpy()
            assert rel_err(out, ref) <= TOL, (m, v, rel_err(out, ref))


@pytest.mark.parametrize("name", FIXTURE_NAMES)
def test_fixtures_rank8(name):
    dims, cidx, vals = load_fixture(name)
    check_modes(dims, cidx, vals, 8, variants=ALL_VARIANTS)


@pytest.mark.parametrize("R", [4, 8, 16, 32, 64, 128, 10, 33])
def test_uniform_ranks(R):
    dims = np.array([1000, 1000, 1000], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 150000, seed=R)
    check_modes(dims, cidx, vals, R, variants=ALL_VARIANTS, seed=R)


@pytest.mark.parametrize("R", [8, 16, 32, 64])
def test_bf16_factor_storage(R):
    import torch

    dims = np.array([800, 700, 900], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 100000, seed=R + 1)
    check_modes(dims, cidx, vals, R, variants=(A.AUTO, A.ATOMIC, A.SORTED, A.SORTED | A.FEED_BULK), dtype=torch.bfloat16, seed=R)


def test_power_law_128bit_keys():
    """Zipf-1.2 coordinates with scattered labels and a 65-bit key."""
    dims = np.array([4800000, 1800000, 1800000], np.uint64)
    cidx, vals = synth.powerlaw_coo(dims, 200000, [1.2, 1.2, 1.2], seed=3, values="lognormal")
    check_modes(dims, cidx, vals, 32, variants=ALL_VARIANTS)


def test_five_modes_rank64():
    dims = np.array([100000, 100000, 10000, 1000, 100], np.uint64)
    cidx, vals = synth.powerlaw_coo(dims, 150000, [1.1, 1.1, None, None, None], seed=4)
    check_modes(dims, cidx, vals, 64, variants=ALL_VARIANTS)


def test_stream_mode_single_row():
    dims = np.array([1, 3000, 4000, 500], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 100000, seed=6)
    import torch

    R = 16
    rng = np.random.default_rng(1)
    F = [rng.uniform(-1, 1, (int(d), R)) for d in dims]
    Fd = to_dev(F, torch.float32)
    t = A.init_salto(dims, cidx, vals, 1, stream_mode=0)
    assert t.choose_variant(0, R) == A.STREAM
    enc = O.build(dims, cidx, vals.astype(np.float32).astype(np.float64))
    fs = seen_by_gpu(Fd)
    fs[0][:] = 0
    ref = O.mttkrp(enc, 0, fs, R)[0]
    out = t.mttkrp(0, Fd, R).cpu().numpy()
    assert rel_err(out, ref) <= TOL


def test_accumulate_semantics():
    import torch

    dims = np.array([300, 200, 100], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 30000, seed=8)
    R = 16
    rng = np.random.default_rng(2)
    F = [rng.uniform(-1, 1, (int(d), R)) for d in dims]
    Fd = to_dev(F, torch.float32)
    t = A.create_alto(dims, cidx, vals)
    base = Fd[1].clone()
    A.mttkrp_alto_par(1, Fd, R, t)  # accumulates into Fd[1]
    fresh = t.mttkrp(1, Fd, R).cpu().numpy()
    np.testing.assert_allclose(Fd[1].cpu().numpy(), base.cpu().numpy() + fresh, rtol=1e-5, atol=1e-5)


def test_host_buffer_entry_point():
    dims = np.array([400, 500, 600], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 50000, seed=10)
    R = 16
    rng = np.random.default_rng(3)
    F = [rng.uniform(-1, 1, (int(d), R)) for d in dims]
    t = A.create_alto(dims, cidx, vals)
    for m in range(3):
        fs = [f.copy() for f in F]
        start = fs[m].copy()
        t.mttkrp_host(m, fs, R)
        fo = [f.astype(np.float32).astype(np.float64) for f in F]
        fo[m][:] = 0
        ref = O.mttkrp(O.build(dims, cidx, vals.astype(np.float32).astype(np.float64)), m, fo, R)[m]
        assert rel_err(fs[m] - start, ref) <= TOL


def test_host_buffer_changed_mask_matches_full_copies():
    """A CP-ALS-like sequence of host-buffer MTTKRPs in which the caller
    rewrites the factor it just received (here: halves it) before the next
    call and declares only that factor changed (alto_mttkrp_host_changed):
    every call still matches the oracle on the caller's current arrays
    (a stale device copy would be off by the halving)."""
    dims = np.array([400, 500, 600], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 50000, seed=12)
    R = 16
    rng = np.random.default_rng(4)
    G = [rng.uniform(-1, 1, (int(d), R)) for d in dims]
    t = A.create_alto(dims, cidx, vals)
    enc = O.build(dims, cidx, vals.astype(np.float32).astype(np.float64))
    prev = None
    for it in range(2):
        for m in range(3):
            start = G[m].copy()
            fo = [g.astype(np.float32).astype(np.float64) for g in G]
            fo[m][:] = 0
            ref = O.mttkrp(enc, m, fo, R)[m]
            t.mttkrp_host(m, G, R, changed=range(3) if prev is None else [prev])
            assert rel_err(G[m] - start, ref) <= TOL, (it, m)
            G[m] *= 0.5
            prev = m
    t.close()


def test_launch_counter_advances():
    import torch

    dims = np.array([50, 60, 70], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 1000, seed=1)
    t = A.create_alto(dims, cidx, vals)
    Fd = to_dev([np.ones((int(d), 8)) for d in dims], torch.float32)
    n0 = A.kernel_launches()
    t.mttkrp(0, Fd, 8)
    torch.cuda.synchronize()
    assert A.kernel_launches() > n0


def test_autotune_records_a_choice_per_mode():
    import torch

    dims = np.array([4800000, 1800000, 1800000], np.uint64)
    cidx, vals = synth.powerlaw_coo(dims, 300000, [1.2, 1.2, 1.2], seed=5, values="lognormal")
    R = 32
    rng = np.random.default_rng(4)
    Fd = to_dev([rng.uniform(-1, 1, (int(d), R)) for d in dims], torch.float32)
    t = A.create_alto(dims, cidx, vals)
    chosen = t.autotune(Fd, R)
    assert len(chosen) == 3 and all(c in (A.ATOMIC, A.STAGED, A.SORTED) for c in chosen)
    for m in range(3):
        assert t.choose_variant(m, R) == chosen[m]
    Fo = seen_by_gpu(Fd)
    enc = O.build(dims, cidx, vals.astype(np.float32).astype(np.float64))
    for m in range(3):
        fs = [f.copy() for f in Fo]
        fs[m][:] = 0
        ref = O.mttkrp(enc, m, fs, R)[m]
        assert rel_err(t.mttkrp(m, Fd, R).cpu().numpy(), ref) <= TOL


# ------------------------------------------------- deterministic variant

def check_deterministic(dims, cidx, vals, R, seed=0, stream_mode=-1):
    """DETERMINISTIC against the oracle, and bit-identical on a second run
    with other MTTKRP work (atomic variants) launched in between."""
    import torch

    rng = np.random.default_rng(seed)
    Fd = to_dev([rng.uniform(-1.0, 1.0, (int(d), R)) for d in dims], torch.float32)
    Fo = seen_by_gpu(Fd)
    t = A.init_salto(dims, cidx, vals, 1, stream_mode=stream_mode) if stream_mode >= 0 else \
        A.create_alto(dims, cidx, vals)
    enc = O.build(dims, cidx, vals.astype(np.float32).astype(np.float64))
    for m in range(len(dims)):
        fs = [f.copy() for f in Fo]
        fs[m][:] = 0
        ref = O.mttkrp(enc, m, fs, R)[m]
        first = t.mttkrp(m, Fd, R, variant=A.DETERMINISTIC)
        assert rel_err(first.cpu().numpy(), ref) <= TOL, (m, rel_err(first.cpu().numpy(), ref))
        for v in (A.ATOMIC, A.SORTED):
            t.mttkrp(m, Fd, R, variant=v)
        again = t.mttkrp(m, Fd, R, variant=A.DETERMINISTIC)
        assert torch.equal(first, again), m


@pytest.mark.parametrize("name", FIXTURE_NAMES)
def test_deterministic_fixtures(name):
    dims, cidx, vals = load_fixture(name)
    check_deterministic(dims, cidx, vals, 8)


@pytest.mark.parametrize("R", [8, 16, 32, 64, 128])
def test_deterministic_ranks(R):
    dims = np.array([1000, 1000, 1000], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 150000, seed=R + 40)
    check_deterministic(dims, cidx, vals, R, seed=R)


def test_deterministic_hot_rows_and_128bit_keys():
    """Zipf 2.0: a few rows hold most nonzeros, so their runs span many
    lane-group sub-ranges (the long-chain fix-up)."""
    dims = np.array([4800000, 1800000, 1800000], np.uint64)
    cidx, vals = synth.powerlaw_coo(dims, 200000, [2.0, 1.2, 2.0], seed=13, values="lognormal")
    check_deterministic(dims, cidx, vals, 32)


def test_deterministic_five_modes_and_stream_row():
    dims = np.array([100000, 100000, 10000, 1000, 100], np.uint64)
    cidx, vals = synth.powerlaw_coo(dims, 150000, [1.1, 1.1, None, None, None], seed=14)
    check_deterministic(dims, cidx, vals, 64)
    dims = np.array([1, 3000, 4000, 500], np.uint64)  # every nonzero in one output row
    cidx, vals = synth.uniform_coo(dims, 100000, seed=15)
    check_deterministic(dims, cidx, vals, 16, stream_mode=0)


def test_deterministic_accumulates_and_rejects_unsupported():
    import torch

    dims = np.array([300, 200, 100], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 30000, seed=16)
    R = 16
    rng = np.random.default_rng(5)
    Fd = to_dev([rng.uniform(-1, 1, (int(d), R)) for d in dims], torch.float32)
    t = A.create_alto(dims, cidx, vals)
    base = torch.ones((200, R), device="cuda")
    out = base.clone()
    t.mttkrp(1, Fd, R, out=out, accumulate=True, variant=A.DETERMINISTIC)
    fresh = t.mttkrp(1, Fd, R, variant=A.DETERMINISTIC)
    np.testing.assert_allclose(out.cpu().numpy(), base.cpu().numpy() + fresh.cpu().numpy(), rtol=1e-6, atol=1e-6)
    Fd10 = to_dev([rng.uniform(-1, 1, (int(d), 10)) for d in dims], torch.float32)
    with pytest.raises(A.AltoError):
        t.mttkrp(0, Fd10, 10, variant=A.DETERMINISTIC)
    with pytest.raises(A.AltoError):
        t.mttkrp(0, [f.to(torch.bfloat16) for f in Fd], R, variant=A.DETERMINISTIC)


# ------------------------------------------------------------ shards

@pytest.mark.parametrize("nparts", [1, 3, 8])
def test_shards_sum_to_the_whole(nparts):
    """alto_tensor_restrict: the shards' MTTKRPs add up to the whole
    tensor's, and each shard keeps the exact keys of its line range."""
    import torch

    from alto_b200 import shard

    dims = np.array([4800000, 1800000, 1800000], np.uint64)
    cidx, vals = synth.powerlaw_coo(dims, 100000, [1.2, 1.2, 1.2], seed=21, values="lognormal")
    R = 32
    rng = np.random.default_rng(7)
    Fd = to_dev([rng.uniform(-1, 1, (int(d), R)) for d in dims], torch.float32)
    whole = A.create_alto(dims, cidx, vals)
    keys = whole.export()
    parts = [shard.shard_tensor(A.create_alto(dims, cidx, vals), p, nparts) for p in range(nparts)]
    assert sum(p.nnz for p in parts) == whole.nnz
    off = 0
    for p in parts:
        k = p.export()
        assert np.array_equal(k["idx"], keys["idx"][off:off + p.nnz])
        off += p.nnz
    for m in range(3):
        ref = whole.mttkrp(m, Fd, R).cpu().numpy()
        tot = sum(p.mttkrp(m, Fd, R, variant=v).cpu().numpy() for p in parts for v in (A.AUTO,))
        assert rel_err(tot, ref) <= 1e-5
