"""Every workload configuration against the FP64 oracle, at its own size or a
stated scale-down, with the oracle fed the ORIGINAL float64 inputs (values,
initial model, factors) rather than the float32 / bfloat16 values the device
holds -- so each bound below is the end-to-end error of the device path, not
only of its accumulation.

  * CP-ALS on 1000^3 with 1,000,000 uniform nonzeros, rank 16, 20
    iterations, plus 100 standalone mode-0 MTTKRPs (that workload at its
    full size).
  * CP-ALS at rank 64 on the 5-mode shape 100k x 100k x 10k x 1k x 100 with
    Zipf(1.1) on modes 0-1 and uniform values, with float32 and with bfloat16
    factor storage (2,000,000 nonzeros against the workload's 50M: the
    oracle is single-threaded).
  * The bfloat16 MTTKRP's error against the oracle given the original
    float32 factors (what halving the gather bytes costs).
  * Three slices of the CP-stream configuration (100k x 100k x 10k,
    Zipf(1.1), Poisson(3) values, rank 16, non-negative ADMM, forgetting
    0.95, up to 50 inner iterations), against the oracle's cpstream.

The 140M-nonzero power-law MTTKRP is checked by bench.py itself, which
recomputes sampled output rows in float64 from the COO it generated."""
import os
import sys

import numpy as np
import pytest

import alto_b200 as A
import oracle as O
from alto_b200 import synth

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def init_model(dims, R, seed):
    init = synth.init_values(int(np.sum(dims)) * R, seed=seed)
    U0, off = [], 0
    for d in dims:
        U0.append(init[off:off + int(d) * R].reshape(int(d), R).copy())
        off += int(d) * R
    return U0


def normwise(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_cpals_1000cubed_1M_nonzeros_20_iterations():
    """Fits within 1e-5 relative at every one of the 20 iterations; factors
    within 1e-3 normwise; 100 mode-0 MTTKRPs each within 1e-5."""
    import torch

    dims = np.array([1000, 1000, 1000], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 1_000_000, seed=55)
    R = 16
    U0 = init_model(dims, R, 55)
    t = A.create_alto(dims, cidx, vals)
    enc = O.build(dims, cidx, vals)
    U, lam, fits, it = A.cpd_alto(t, U0, np.ones(R), R, 20, 1e-12)
    Uo, lo, fo, ito = O.cpd_als(enc, U0, np.ones(R), R, 20, 1e-12)
    assert it == ito == 20
    np.testing.assert_allclose(fits, fo, rtol=1e-5)
    for a, b in zip(U, Uo):
        assert normwise(a, b) <= 1e-3, normwise(a, b)
    # 100 standalone MTTKRPs of mode 0 with float32 factors (the oracle reads
    # the same float32 factor values, widened)
    rng = np.random.default_rng(5)
    F = [rng.uniform(-1, 1, (int(d), R)).astype(np.float32) for d in dims]
    Fd = [torch.tensor(f, device="cuda") for f in F]
    fo64 = [f.astype(np.float64) for f in F]
    fo64[0][:] = 0
    ref = O.mttkrp(enc, 0, fo64, R)[0]
    worst = 0.0
    for _ in range(100):
        out = t.mttkrp(0, Fd, R).cpu().numpy()
        worst = max(worst, normwise(out, ref))
    assert worst <= 1e-5, worst
    t.close()


@pytest.fixture(scope="module")
def five_mode_case():
    dims = np.array([100000, 100000, 10000, 1000, 100], np.uint64)
    cidx, vals = synth.powerlaw_coo(dims, 2_000_000, [1.1, 1.1, None, None, None], seed=3)
    R = 64
    U0 = init_model(dims, R, 3)
    enc = O.build(dims, cidx, vals)
    Uo, lo, fo, ito = O.cpd_als(enc, U0, np.ones(R), R, 3, 1e-12)
    return dims, cidx, vals, R, U0, (Uo, lo, fo, ito)


@pytest.mark.parametrize("storage,fit_tol,factor_tol", [(A.F32, 1e-5, 1e-3), (A.BF16, 1e-4, 5e-2)],
                         ids=["f32", "bf16"])
def test_cpals_five_modes_rank64(five_mode_case, storage, fit_tol, factor_tol):
    """Rank 64 runs the specialised rank-64 MTTKRP (the reference's
    runtime-rank path, include/cpd.hpp:47-191); float64 Grams and Cholesky.
    Bounds: fits within fit_tol relative, factors within factor_tol
    normwise (bfloat16 storage rounds every factor to 8 significant bits
    after each update)."""
    dims, cidx, vals, R, U0, (Uo, lo, fo, ito) = five_mode_case
    t = A.create_alto(dims, cidx, vals)
    U, lam, fits, it = A.cpd_alto(t, U0, np.ones(R), R, 3, 1e-12, storage=storage)
    assert it == ito == 3
    np.testing.assert_allclose(fits, fo, rtol=fit_tol)
    for a, b in zip(U, Uo):
        assert normwise(a, b) <= factor_tol, normwise(a, b)
    t.close()


@pytest.mark.parametrize("R", [16, 32, 64])
def test_bf16_mttkrp_error_against_original_factors(R):
    """The bfloat16 factor path against the oracle given the float32 factors
    before rounding: the rounding of two gathered rows to 8 significant bits
    bounds it (2 x 2^-9 per product); measured about 2e-3 normwise."""
    import torch

    dims = np.array([4800000, 1800000, 1800000], np.uint64)
    cidx, vals = synth.powerlaw_coo(dims, 300000, [1.2, 1.2, 1.2], seed=R, values="lognormal")
    rng = np.random.default_rng(R)
    F = [rng.uniform(-1, 1, (int(d), R)).astype(np.float32) for d in dims]
    Fd = [torch.tensor(f, device="cuda").to(torch.bfloat16) for f in F]
    t = A.create_alto(dims, cidx, vals)
    enc = O.build(dims, cidx, vals)
    for m in range(3):
        fs = [f.astype(np.float64) for f in F]
        fs[m][:] = 0
        ref = O.mttkrp(enc, m, fs, R)[m]
        out = t.mttkrp(m, Fd, R).cpu().numpy()
        assert normwise(out, ref) <= 1e-2, (m, normwise(out, ref))
    t.close()


def test_cpstream_three_slices_of_the_workload():
    """Three slices of the CP-stream configuration (the first three of
    bench.py's stream, 92k-133k nonzeros each) through the session API
    against the oracle's cpstream with the original float64 values and
    initial model: factors within 1e-4 normwise, the same inner-iteration
    counts, non-negative factors."""
    import bench

    R = 16
    b = bench.c4_batches(3)
    need = bench.stream_need(b, R)
    iv = synth.init_values(sum(need), seed=11)
    N = len(b[0]["dims"])
    s = A.CPStream(N, 0, R, constraint=A.NONNEG, forgetting=0.95, max_inner=50, epsilon=1e-5)
    used, inner = 0, []
    for x, n in zip(b, need):
        inner.append(s.push(x["dims"], x["cidx"], x["vals"], iv[used:used + n]))
        used += n
    oo, lo, inner_o = O.cpstream(b, 0, R, 50, 1e-5, 1, iv, forgetting=0.95)
    assert list(inner) == list(inner_o)
    for m in range(N):
        rows = len(b) if m == 0 else int(b[-1]["dims"][m])
        g = s.factor(m, rows)
        assert normwise(g, oo[m]) <= 1e-4, (m, normwise(g, oo[m]))
        if m:
            assert np.all(g >= 0)
    s.close()
