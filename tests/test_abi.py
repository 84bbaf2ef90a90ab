"""The C-ABI library loads and exports every entry point that
include/alto_b200.h declares; host-only entry points and argument checks
work without a GPU (no device work is requested here)."""
import ctypes
import os
import re

import numpy as np
import pytest

import alto_b200 as A
import oracle as O
from alto_b200 import synth
from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "alto_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(alto_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_expected_surface():
    names = declared_functions()
    assert "alto_tensor_create" in names and "alto_mttkrp" in names and "alto_cpd_als" in names
    assert set(names) == set(A.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = A.lib()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_mirror_constants_match_the_header():
    """The Python mirror's variant, feed, dtype and constraint values are
    the header's (a mismatch would run a different kernel than asked for)."""
    text = open(HEADER).read()
    defines = {k: int(v, 0) for k, v in re.findall(r"#define\s+(ALTO_[A-Z0-9_]+)\s+(0x[0-9a-fA-F]+|\d+)", text)}
    for name in ("FEED_BULK", "FEED_DENSE", "FEED_FIXED_TARGET"):
        assert getattr(A, name) == defines["ALTO_MTTKRP_" + name], name
    enums = {k: int(v) for k, v in re.findall(r"\b(ALTO_[A-Z0-9_]+)\s*=\s*(\d+)", text)}
    for name in ("AUTO", "ATOMIC", "STAGED", "STREAM", "SORTED", "DETERMINISTIC"):
        assert getattr(A, name) == enums["ALTO_MTTKRP_" + name], name
    assert A.F32 == enums["ALTO_F32"] and A.BF16 == enums["ALTO_BF16"]


def test_status_strings_and_version():
    L = A.lib()
    assert L.alto_version() == 100
    for s in range(7):
        assert L.alto_status_string(s)


@pytest.mark.parametrize("dims", [[2, 3, 2], [2425, 10816, 29567], [1, 8, 1, 3], [4800000, 1800000, 1800000],
                                  [100000, 100000, 10000, 1000, 100], [7], [2 ** 32 - 1, 2 ** 32 - 1]])
def test_host_masks_match_oracle(dims):
    masks, am, bits = A.compute_masks(dims, 128)
    ref = O.setup_masks(np.array(dims, np.uint64))
    assert np.array_equal(masks, ref["masks"])
    assert np.array_equal(am, ref["alto_mask"])
    assert bits == ref["alto_bits"]


def test_mask_width_rejected():
    with pytest.raises(A.AltoError) as e:
        A.compute_masks([4800000, 1800000, 1800000], 64)
    assert e.value.status == A.ERR_UNSUPPORTED


def test_bad_arguments_rejected_before_device_work():
    L = A.lib()
    out = ctypes.c_void_p()
    assert L.alto_tensor_create(None, 0, 1, -1, None, ctypes.byref(out)) == A.ERR_INVALID
    dims = np.array([4, 4], np.uint64)
    cidx = np.array([[0, 1], [2, 9]], np.uint64)  # 9 >= dims[1]
    coo = A._Coo(dims, cidx, np.ones(2))
    assert L.alto_tensor_create(ctypes.byref(coo.c), 0, 1, -1, None, ctypes.byref(out)) == A.ERR_INVALID
    assert b"cidx[1][1]" in L.alto_last_error()
    coo = A._Coo(dims, np.array([[0, 1], [2, 3]], np.uint64), np.ones(2))
    assert L.alto_tensor_create(ctypes.byref(coo.c), 0, 0, -1, None, ctypes.byref(out)) == A.ERR_INVALID
    assert L.alto_tensor_create(ctypes.byref(coo.c), 32, 1, -1, None, ctypes.byref(out)) == A.ERR_INVALID
    assert L.alto_stream_open(3, 5, 8, 0, ctypes.c_double(0.99), 10, ctypes.c_double(1e-5), None, ctypes.byref(out)) == A.ERR_INVALID
    assert L.alto_stream_open(3, 0, 0, 0, ctypes.c_double(0.99), 10, ctypes.c_double(1e-5), None, ctypes.byref(out)) == A.ERR_UNSUPPORTED


def test_synthetic_generators_unique_and_in_range():
    dims = [50, 60, 70]
    cidx, vals = synth.uniform_coo(dims, 5000, seed=4)
    assert cidx.shape == (3, 5000)
    assert len({tuple(c) for c in cidx.T.tolist()}) == 5000
    assert all(int(cidx[m].max()) < d for m, d in enumerate(dims))
    c2, v2 = synth.powerlaw_coo([1000, 500, 200], 3000, [1.2, 1.2, None], seed=1, values="lognormal")
    assert len({tuple(c) for c in c2.T.tolist()}) == c2.shape[1] == 3000
    assert np.all(v2 > 0)


def test_stream_batches_follow_the_reference_slicer():
    b = synth.stream_batches([200, 300, 50], 5, lambda rng, s: 300, [1.1, 1.1, None], seed=5)
    prev = None
    for x in b:
        assert int(x["dims"][0]) == 1 and np.all(x["cidx"][0] == 0)
        assert np.all(x["vals"] != 0)
        if prev is not None:
            assert np.all(x["dims"] >= prev)
        for m in (1, 2, 3):
            assert int(x["cidx"][m].max()) < int(x["dims"][m])
        prev = x["dims"]


def test_new_entry_points_reject_bad_arguments_without_device_work(tmp_path):
    """Argument checks of the slicer, tensor-file, error and poll entry
    points (each fails before any device work)."""
    L = A.lib()
    c = ctypes.c_int()
    u = ctypes.c_uint64()
    coo = A.alto_coo()
    assert L.alto_slicer_next(None, ctypes.c_uint64(1), ctypes.c_uint64(1), ctypes.byref(coo), ctypes.byref(c)) \
        == A.ERR_INVALID
    assert L.alto_slicer_cut_all(None, ctypes.c_uint64(1), ctypes.c_uint64(1), ctypes.byref(u)) == A.ERR_INVALID
    assert L.alto_slicer_batch(None, ctypes.c_uint64(0), ctypes.byref(coo)) == A.ERR_INVALID
    assert L.alto_slicer_last_batch(None, ctypes.byref(c)) == A.ERR_INVALID
    assert L.alto_slicer_tensor(None, ctypes.byref(coo)) == A.ERR_INVALID
    assert L.alto_slicer_destroy(None) == A.OK
    h = ctypes.c_void_p()
    assert L.alto_read_tensor(str(tmp_path / "missing.tns").encode(), 0, 0, None, ctypes.byref(h)) == A.ERR_INVALID
    (tmp_path / "empty.tns").write_bytes(b"")
    assert L.alto_read_tensor(str(tmp_path / "empty.tns").encode(), 0, 0, None, ctypes.byref(h)) == A.ERR_INVALID
    assert L.alto_read_tensor(str(tmp_path / "x.tns").encode(), 7, 0, None, ctypes.byref(h)) == A.ERR_INVALID
    assert L.alto_dcoo_view(None, ctypes.byref(coo)) == A.ERR_INVALID
    assert L.alto_dcoo_destroy(None) == A.OK
    assert L.alto_server_poll(None, ctypes.c_uint64(0), ctypes.byref(c), None, None) == A.ERR_INVALID
    assert L.alto_stream_error(None, ctypes.byref(coo), None) == A.ERR_INVALID
    dims = np.array([3, 3], np.uint64)
    with pytest.raises(A.AltoError) as e:  # the reference asserts nnz > 0 on export
        A.write_tensor(tmp_path / "e.tns", dims, np.zeros((2, 0), np.uint64), np.zeros(0))
    assert e.value.status == A.ERR_INVALID
