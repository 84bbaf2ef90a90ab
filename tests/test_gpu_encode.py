"""GPU ALTO encoding (linearise, radix sort, partition) is bit-exact against
the oracle: keys, order, values, partition pointers and intervals."""
import numpy as np
import pytest

import alto_b200 as A
import oracle as O
from alto_b200 import synth
from conftest import FIXTURE_NAMES, load_fixture

pytestmark = pytest.mark.gpu


def check_same(t, dims, cidx, vals, P):
    e = t.export()
    o = O.build(dims, cidx, vals, nprtn=P)
    assert np.array_equal(e["masks"], o["masks"])
    assert np.array_equal(e["alto_mask"], o["alto_mask"])
    assert np.array_equal(e["idx"], o["idx"]), "ALTO keys or order differ"
    assert np.array_equal(e["perm"], o["perm"])
    np.testing.assert_array_equal(e["vals"], o["vals"].astype(np.float32).astype(np.float64))
    assert np.array_equal(e["prtn_ptr"], o["prtn_ptr"])
    assert np.array_equal(e["intervals"], o["intervals"])
    assert t.alto_bits == o["alto_bits"]


@pytest.mark.parametrize("name", FIXTURE_NAMES)
@pytest.mark.parametrize("P", [1, 3, 8])
def test_fixture_encoding_bit_exact(name, P):
    dims, cidx, vals = load_fixture(name)
    t = A.create_alto(dims, cidx, vals, nprtn=P)
    check_same(t, dims, cidx, vals, P)


@pytest.mark.parametrize("dims,nnz,key_bits", [
    ([1000, 1000, 1000], 200000, 0),
    ([1000, 1000, 1000], 50000, 128),
    ([2 ** 21 + 5, 2 ** 21 + 7, 2 ** 22 + 1], 150000, 0),
    ([100000, 100000, 10000, 1000, 100], 120000, 0),
    ([3, 5, 7, 11, 13, 17, 19, 23], 60000, 0),
])
def test_random_encoding_bit_exact(dims, nnz, key_bits):
    dims = np.array(dims, np.uint64)
    cidx, vals = synth.uniform_coo(dims, nnz, seed=len(dims))
    t = A.create_alto(dims, cidx, vals, nprtn=7, key_bits=key_bits)
    check_same(t, dims, cidx, vals, 7)


def test_device_coo_input():
    import torch

    dims = np.array([3000, 2000, 500], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 100000, seed=9)
    for dt in (torch.int64, torch.int32):
        c = torch.tensor(cidx.astype(np.int64), dtype=dt, device="cuda")
        v = torch.tensor(vals, dtype=torch.float32, device="cuda")
        t = A.AltoTensor(dims, c, v, nprtn=5)
        check_same(t, dims, cidx, vals.astype(np.float32).astype(np.float64), 5)


def test_update_reuses_tensor():
    dims = np.array([500, 400, 300], np.uint64)
    c1, v1 = synth.uniform_coo(dims, 80000, seed=1)
    t = A.init_salto(dims, c1, v1, 4, stream_mode=0)
    check_same(t, dims, c1, v1, 4)
    dims2 = np.array([1, 4000, 300], np.uint64)
    c2, v2 = synth.uniform_coo(dims2, 20000, seed=2)
    A.update_salto(dims2, c2, v2, t, nprtn=3)
    check_same(t, dims2, c2, v2, 3)
    dims3 = np.array([1, 5000, 9000], np.uint64)
    c3, v3 = synth.uniform_coo(dims3, 200000, seed=3)
    A.update_salto(dims3, c3, v3, t, nprtn=9)
    check_same(t, dims3, c3, v3, 9)


@pytest.mark.parametrize("dims,nnz", [([5, 6, 7], 1), ([1, 50, 60], 400), ([1, 1, 9], 9), ([4, 4, 4], 0)])
def test_edge_shapes(dims, nnz):
    dims = np.array(dims, np.uint64)
    if nnz:
        cidx, vals = synth.uniform_coo(dims, nnz, seed=3)
    else:
        cidx, vals = np.zeros((3, 0), np.uint64), np.zeros(0)
    t = A.create_alto(dims, cidx, vals, nprtn=4)
    check_same(t, dims, cidx, vals, 4)


def test_large_one_million_nonzeros():
    """The 1000^3, 1M-nonzero CP-ALS workload: encoding bit-exact."""
    dims = np.array([1000, 1000, 1000], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 1000000, seed=55)
    t = A.create_alto(dims, cidx, vals, nprtn=8)
    check_same(t, dims, cidx, vals, 8)
