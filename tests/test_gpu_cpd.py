"""GPU CP-ALS against the oracle and the reference's recorded fits.

Factors are float32 on the device (MTTKRP accumulates in float32, Grams /
Cholesky / fit in float64), so the bound is relative: |fit - fit_ref| <=
1e-5 * fit_ref per iteration, and the final factors within 1e-3
(normwise) of the FP64 oracle."""
import numpy as np
import pytest

import alto_b200 as A
import oracle as O
from alto_b200 import synth
from conftest import load_fixture

pytestmark = pytest.mark.gpu


def init_model(dims, R, seed):
    init = synth.init_values(int(np.sum(dims)) * R, seed=seed)
    U0, off = [], 0
    for d in dims:
        U0.append(init[off:off + int(d) * R].reshape(int(d), R).copy())
        off += int(d) * R
    return U0


def test_med_fits_match_reference(golden):
    g = golden["cpd_als_med"]
    dims, cidx, vals = load_fixture("med")
    R = g["rank"]
    U0 = init_model(dims, R, g["init_seed"])
    t = A.create_alto(dims, cidx, vals)
    U, lam, fits, it = A.cpd_alto(t, U0, np.ones(R), R, 8, 1e-12)
    assert it == g["iters"]
    np.testing.assert_allclose(fits, g["fits"], rtol=1e-5)


@pytest.mark.parametrize("R,fit_mode", [(8, A.FIT_REFERENCE), (16, A.FIT_EXACT), (32, A.FIT_REFERENCE)])
def test_random_against_oracle(R, fit_mode):
    dims = np.array([60, 70, 80], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 20000, seed=R)
    vals = vals.astype(np.float32).astype(np.float64)
    U0 = [u.astype(np.float32).astype(np.float64) for u in init_model(dims, R, R)]
    t = A.create_alto(dims, cidx, vals)
    U, lam, fits, it = A.cpd_alto(t, U0, np.ones(R), R, 6, 1e-12, fit_mode=fit_mode)
    Uo, lo, fo, ito = O.cpd_als(O.build(dims, cidx, vals), U0, np.ones(R), R, 6, 1e-12,
                                fit_exact=fit_mode == A.FIT_EXACT)
    assert it == ito == 6
    np.testing.assert_allclose(fits, fo, rtol=1e-5)
    for a, b in zip(U, Uo):
        assert np.abs(a - b).max() <= 1e-3 * np.abs(b).max()
    np.testing.assert_allclose(lam, lo, rtol=1e-3)


def test_five_modes_and_bf16_storage():
    dims = np.array([500, 400, 300, 50, 20], np.uint64)
    cidx, vals = synth.powerlaw_coo(dims, 60000, [1.1, 1.1, None, None, None], seed=2)
    R = 16
    U0 = init_model(dims, R, 1)
    t = A.create_alto(dims, cidx, vals)
    _, _, f32, _ = A.cpd_alto(t, U0, np.ones(R), R, 5, 1e-12, storage=A.F32)
    _, _, fb, _ = A.cpd_alto(t, U0, np.ones(R), R, 5, 1e-12, storage=A.BF16)
    _, _, fo, _ = O.cpd_als(O.build(dims, cidx, vals), U0, np.ones(R), R, 5, 1e-12)
    np.testing.assert_allclose(f32, fo, rtol=1e-4)
    np.testing.assert_allclose(fb, fo, rtol=5e-3)


def test_early_stop_matches_epsilon():
    dims = np.array([40, 50, 60], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 8000, seed=5)
    vals = vals.astype(np.float32).astype(np.float64)
    R = 8
    U0 = [u.astype(np.float32).astype(np.float64) for u in init_model(dims, R, 2)]
    t = A.create_alto(dims, cidx, vals)
    _, _, fits, it = A.cpd_alto(t, U0, np.ones(R), R, 50, 1e-3)
    _, _, fo, ito = O.cpd_als(O.build(dims, cidx, vals), U0, np.ones(R), R, 50, 1e-3)
    assert it == ito
