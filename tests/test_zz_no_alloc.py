"""alto_gram_noalloc, the Gram entry point for callers that cannot allocate
device memory.

Who needs it: a process whose memory pool has already reserved all of HBM,
code that runs inside CUDA graph capture or a real-time loop where the
allocator is off limits, and embedders that are not allowed to call
cudaMalloc / cudaFree.  The entry point keeps its scratch (the per-block
partial sums of the Gram) in a fixed device array inside the library, so
it allocates nothing.

The test calls it through the C ABI twice in a row and compares each
result with alto_gram's at the tolerance of the other Gram tests; the
second call is smaller than the first, so leftovers of the first call in
the shared scratch would show.  It passes alone in a fresh process and
after the rest of the suite (this file is collected last).
"""
import ctypes

import numpy as np
import pytest

import alto_b200 as A

pytestmark = pytest.mark.gpu


def _call(fn, U, G, stream):
    rows, rank = U.shape
    return fn(ctypes.c_void_p(U.data_ptr()), ctypes.c_uint64(rows), ctypes.c_int(rank),
              ctypes.c_void_p(G.data_ptr()), ctypes.c_void_p(stream))


# Pairs of calls in a row; the second is smaller than the first.  The cases
# cover the 64-block cap (100000 rows at rank 64), the per-thread share of
# 16 used for a share-of-8 need (rank 40), a single row and rank 1, and zero
# rows, where G is cleared without a kernel.
CALL_PAIRS = [
    [(100000, 64), (3000, 16)],
    [(50000, 40), (1, 1)],
    [(20000, 8), (0, 8)],
]


@pytest.mark.parametrize("calls", CALL_PAIRS, ids=["cap-then-small", "rank40-then-one-row", "then-empty"])
def test_noalloc_gram_matches_alto_gram_on_two_calls(calls):
    import torch

    L = A.lib()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(7)
    for rows, rank in calls:
        U = torch.tensor(rng.uniform(-1, 1, (rows, rank)).astype(np.float32), device="cuda")
        G_ref = torch.empty((rank, rank), dtype=torch.float64, device="cuda")
        G_new = torch.full((rank, rank), float("nan"), dtype=torch.float64, device="cuda")
        assert _call(L.alto_gram, U, G_ref, stream) == A.OK
        assert _call(L.alto_gram_noalloc, U, G_new, stream) == A.OK, L.alto_last_error()
        torch.cuda.synchronize()
        ref = G_ref.cpu().numpy()
        np.testing.assert_allclose(G_new.cpu().numpy(), ref, rtol=1e-12,
                                   atol=1e-12 * max(1.0, np.abs(ref).max()))


def test_noalloc_gram_rejects_rank_beyond_its_scratch():
    import torch

    L = A.lib()
    U = torch.zeros((10, 65), dtype=torch.float32, device="cuda")
    G = torch.zeros((65, 65), dtype=torch.float64, device="cuda")
    assert _call(L.alto_gram_noalloc, U, G, torch.cuda.current_stream().cuda_stream) == A.ERR_UNSUPPORTED
    assert b"rank 65" in L.alto_last_error()
