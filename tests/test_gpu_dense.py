"""GPU float64 Gram (update_gram) through the C ABI against numpy float64."""
import numpy as np
import pytest

import alto_b200 as A

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows,rank", [(1, 1), (7, 3), (1000, 8), (4096, 16), (100000, 32), (33333, 64),
                                       (5000, 100), (2000, 128), (0, 16)])
def test_gram_matches_float64(rows, rank):
    import torch

    rng = np.random.default_rng(rows + rank)
    U = rng.uniform(-1, 1, (rows, rank)).astype(np.float32)
    G = A.gram(torch.tensor(U, device="cuda")).cpu().numpy()
    ref = U.astype(np.float64).T @ U.astype(np.float64)
    np.testing.assert_allclose(G, ref, rtol=1e-12, atol=1e-12 * max(1.0, np.abs(ref).max()))
    assert np.array_equal(G, G.T)


def test_gram_rejects_large_rank():
    import torch

    with pytest.raises(A.AltoError) as e:
        A.gram(torch.zeros((4, 129), device="cuda"))
    assert e.value.status == A.ERR_UNSUPPORTED
