"""The oracle (C restatement in oracle/alto_oracle.c) against the golden
vectors that the compiled reference produced (tests/golden/make_golden.py),
and against the compiled reference itself when oracle/_ref is built."""
import hashlib
import os

import numpy as np
import pytest

import oracle as O
from alto_b200 import synth
from conftest import FIXTURE_NAMES, load_fixture, load_stream_fixture

# Known answers from a debug build of the reference (ALTO_DEBUG prints the
# masks): small.tns, small4.tns and med.tns.
KNOWN_MASKS = {
    "small": [0x1, 0xC, 0x2],
    "small4": [0x1, 0x2, 0x14, 0x28],
    "med": [0x249249249, 0x5492492492, 0x1A924924924],
}


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", list(KNOWN_MASKS))
def test_known_masks(name):
    dims, _, _ = load_fixture(name)
    m = O.setup_masks(dims)
    assert O.join128(m["masks"]) == KNOWN_MASKS[name]


@pytest.mark.parametrize("name", FIXTURE_NAMES)
def test_encoding_matches_reference_digests(name, golden):
    dims, cidx, vals = load_fixture(name)
    g = golden[name]
    for P in (1, 3, 8):
        enc = O.build(dims, cidx, vals, nprtn=P, max_bits=g["bits"])
        assert [[int(a), int(b)] for a, b in enc["masks"]] == g["masks"]
        assert [int(x) for x in enc["alto_mask"]] == g["alto_mask"]
        assert digest(enc["idx"]) == g[f"P{P}"]["idx"]
        assert digest(enc["vals"]) == g[f"P{P}"]["vals"]
        assert enc["prtn_ptr"].tolist() == g[f"P{P}"]["prtn_ptr"]
        assert digest(enc["intervals"].reshape(-1)) == g[f"P{P}"]["intervals"]


@pytest.mark.parametrize("name", FIXTURE_NAMES)
def test_decode_roundtrip(name):
    dims, cidx, vals = load_fixture(name)
    enc = O.build(dims, cidx, vals)
    dec = O.decode(enc)
    assert np.array_equal(dec, cidx[:, enc["perm"].astype(np.int64)])


@pytest.mark.parametrize("name", FIXTURE_NAMES)
def test_mttkrp_matches_reference(name, golden):
    dims, cidx, vals = load_fixture(name)
    enc = O.build(dims, cidx, vals)
    rng = np.random.default_rng(11)
    F = [rng.uniform(-1.0, 1.0, (int(d), 8)) for d in dims]
    for m, g in enumerate(golden[name]["mttkrp"]):
        fs = [f.copy() for f in F]
        fs[m][:] = 0
        out = O.mttkrp(enc, m, fs, 8)[m]
        if "full" in g:
            np.testing.assert_allclose(out, np.array(g["full"]), rtol=1e-12, atol=1e-12)
        else:
            np.testing.assert_allclose(out.sum(0), g["colsum"], rtol=1e-10, atol=1e-9)
            np.testing.assert_allclose(np.linalg.norm(out), g["fro"], rtol=1e-12)
            np.testing.assert_allclose(out[g["rows"]], np.array(g["sample"]), rtol=1e-10, atol=1e-12)
        # the COO MTTKRP (src/mttkrp.cpp) agrees with the ALTO one
        coo = O.coo_mttkrp(cidx, vals, m, [f.copy() if i != m else np.zeros_like(f) for i, f in enumerate(F)], 8)[m]
        np.testing.assert_allclose(out, coo, rtol=1e-10, atol=1e-10)


def test_cpd_als_matches_reference(golden):
    g = golden["cpd_als_med"]
    dims, cidx, vals = load_fixture("med")
    R = g["rank"]
    init = synth.init_values(int(dims.sum()) * R, seed=g["init_seed"])
    U0, off = [], 0
    for n in dims:
        U0.append(init[off:off + int(n) * R].reshape(int(n), R))
        off += int(n) * R
    enc = O.build(dims, cidx, vals)
    _, lam, fits, it = O.cpd_als(enc, U0, np.ones(R), R, 8, 1e-12)
    assert it == g["iters"]
    np.testing.assert_allclose(fits, g["fits"], rtol=1e-10)
    np.testing.assert_allclose(lam, g["lambda"], rtol=1e-8)


@pytest.mark.parametrize("nonneg", [0, 1])
def test_cpstream_matches_reference(nonneg, golden):
    g = golden[f"cpstream_small_nonneg{nonneg}"]
    b = load_stream_fixture()
    iv = synth.init_values(g["n_init"], seed=g["init_seed"])
    outs, lam, inner = O.cpstream(b, 0, g["rank"], g["max_iters"], g["eps"], nonneg, iv)
    np.testing.assert_allclose([np.linalg.norm(o) for o in outs], g["norms"], rtol=1e-9)
    for o, cs in zip(outs, g["colsums"]):
        np.testing.assert_allclose(o.sum(0), cs, rtol=1e-7, atol=1e-9)


def test_spcpstream_matches_reference(golden):
    """The spCP-stream restatement against the compiled reference's
    spcpstream_alto_iter on the small stream (row-sparse updates, closed-form
    untouched rows, c/h Gram bookkeeping)."""
    g = golden["spcpstream_small"]
    b = load_stream_fixture()
    iv = synth.init_values(g["n_init"], seed=g["init_seed"])
    outs, lam, inner = O.spcpstream(b, 0, g["rank"], g["max_iters"], g["eps"], iv)
    np.testing.assert_allclose([np.linalg.norm(o) for o in outs], g["norms"], rtol=1e-9)
    for o, cs in zip(outs, g["colsums"]):
        np.testing.assert_allclose(o.sum(0), cs, rtol=1e-7, atol=1e-9)


def test_partition_rules():
    """prtn_alto: equal-nnz partitions, empty tail partitions, clamped intervals."""
    dims = np.array([4, 5, 6], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 10, seed=2)
    enc = O.build(dims, cidx, vals, nprtn=4)
    assert enc["prtn_ptr"].tolist() == [0, 3, 6, 9, 10]
    enc = O.build(dims, cidx[:, :5], vals[:5], nprtn=4)
    assert enc["prtn_ptr"].tolist() == [0, 2, 4, 5, 5]
    assert np.all(enc["intervals"][3] == 0)  # empty partition: start = stop = 0


def test_length_one_mode_takes_no_bits():
    m = O.setup_masks(np.array([1, 8, 1, 3], np.uint64))
    assert m["alto_bits"] == 5
    assert O.join128(m["masks"])[0] == 0 and O.join128(m["masks"])[2] == 0


@pytest.mark.skipif(not (O.ref_available(64) and O.ref_available(128)), reason="oracle/_ref not built")
class TestAgainstCompiledReference:
    def test_random_encodings(self):
        for seed, dims in enumerate([[1000, 1000, 1000], [4800, 1800, 18000], [100, 100, 10, 7, 3],
                                     [2 ** 21 + 5, 2 ** 21 + 7, 2 ** 22 + 1]]):
            dims = np.array(dims, np.uint64)
            cidx, vals = synth.uniform_coo(dims, 20000, seed=seed)
            for P in (1, 5, 37):
                t = O.RefTensor(dims, cidx, vals, P)
                e = t.export()
                o = O.build(dims, cidx, vals, nprtn=P)
                assert np.array_equal(e["masks"], o["masks"])
                assert np.array_equal(e["idx"], o["idx"])
                assert np.array_equal(e["vals"], o["vals"])
                assert np.array_equal(e["prtn_ptr"], o["prtn_ptr"])
                assert np.array_equal(e["intervals"], o["intervals"])
                t.close()

    def test_mttkrp_random_power_law_and_five_modes(self):
        """The oracle's MTTKRP (float64) against the reference's
        mttkrp_alto_par (include/alto.hpp:826-908 and the variant it picks)
        on a Zipf 3-mode tensor with a 65-bit key (the 128-bit build) and a
        5-mode tensor, every mode, at several partition counts.  The
        reference sums in a thread-dependent order, so the bound is
        normwise 1e-12."""
        cases = [(np.array([4800000, 1800000, 1800000], np.uint64), 40000, [1.2, 1.2, 1.2], 32),
                 (np.array([100000, 100000, 10000, 1000, 100], np.uint64), 30000, [1.1, 1.1, None, None, None], 16)]
        for k, (dims, nnz, zipf, R) in enumerate(cases):
            cidx, vals = synth.powerlaw_coo(dims, nnz, zipf, seed=11 + k)
            rng = np.random.default_rng(k)
            F = [rng.uniform(-1, 1, (int(d), R)) for d in dims]
            enc = O.build(dims, cidx, vals)
            for P in (1, 7):
                t = O.RefTensor(dims, cidx, vals, P)
                for m in range(len(dims)):
                    fs = [f.copy() for f in F]
                    fs[m][:] = 0
                    ref = t.mttkrp(m, fs, R)[m]
                    fo = [f.copy() for f in F]
                    fo[m][:] = 0
                    out = O.mttkrp(enc, m, fo, R)[m]
                    err = np.abs(out - ref).max() / np.abs(ref).max()
                    assert err <= 1e-12, (k, P, m, err)
                t.close()

    @pytest.mark.parametrize("nonneg", [0, 1])
    def test_cpstream_random_slices(self, nonneg):
        """The oracle's CP-stream against the reference's cpstream
        (src/streaming_cpd.cpp:26-366, 1198-1519) on four random slices
        drawn like the CP-stream workload (Zipf 1.1 coordinates with
        first-seen labels, Poisson(3) values) at a reduced size, rank 8, ten
        inner iterations at most, forgetting 0.99 (the reference's fixed
        value); the reference single-threaded.  Bound: 1e-10 normwise per
        factor, identical lambda."""
        space = [3000, 3000, 500]
        b = synth.stream_batches(space, 4, lambda rng, s: int(np.clip(rng.lognormal(np.log(4000), 0.5), 1500, 12000)),
                                 [1.1, 1.1, 1.1], seed=5, values="poisson3")
        R, need, prev = 8, 0, np.zeros(4, np.int64)
        for x in b:
            d = x["dims"].astype(np.int64)
            need += int(np.sum(np.maximum(d - prev, 0))) * R
            prev = np.maximum(prev, d)
        iv = synth.init_values(need, seed=9)
        L = O.ref_lib(64)
        L.ref_set_threads(1)
        try:
            outs, lam, inner = O.cpstream(b, 0, R, 10, 1e-5, nonneg, iv)
            routs, rlam, _ = O.ref_cpstream(b, 0, R, 10, 1e-5, nonneg, iv)
        finally:
            L.ref_set_threads(os.cpu_count() or 1)
        for o, r in zip(outs, routs):
            assert np.abs(o - r).max() <= 1e-10 * np.abs(r).max()
        np.testing.assert_allclose(lam, rlam, rtol=1e-12)

    def test_spcpstream_random_slices(self):
        """The oracle's spCP-stream against the reference's
        spcpstream_alto_iter (src/streaming_cpd.cpp:466-1085) on four random
        slices of the CP-stream workload's distribution at a reduced size,
        rank 8, the reference single-threaded.  Bound: 1e-10 normwise per
        factor, identical lambda."""
        space = [3000, 3000, 500]
        b = synth.stream_batches(space, 4, lambda rng, s: int(np.clip(rng.lognormal(np.log(4000), 0.5), 1500, 12000)),
                                 [1.1, 1.1, 1.1], seed=6, values="poisson3")
        R, need, prev = 8, 0, np.zeros(4, np.int64)
        for x in b:
            d = x["dims"].astype(np.int64)
            need += int(np.sum(np.maximum(d - prev, 0))) * R
            prev = np.maximum(prev, d)
        iv = synth.init_values(need, seed=10)
        L = O.ref_lib(64)
        L.ref_set_threads(1)
        try:
            outs, lam, inner = O.spcpstream(b, 0, R, 10, 1e-5, iv)
            routs, rlam, _ = O.ref_spcpstream(b, 0, R, 10, 1e-5, iv)
        finally:
            L.ref_set_threads(os.cpu_count() or 1)
        for o, r in zip(outs, routs):
            assert np.abs(o - r).max() <= 1e-10 * np.abs(r).max()
        np.testing.assert_allclose(lam, rlam, rtol=1e-12)

    @pytest.mark.parametrize("dims,zipf,R", [([65537, 65539, 65541, 70000], [1.2, 1.2, 1.2, None], 16),
                                             ([2000, 2000, 300, 50, 10], [1.1, 1.1, None, None, None], 10)],
                             ids=["128bit-4mode-r16", "5mode-r10"])
    def test_cpd_als_wide_keys_and_runtime_rank(self, dims, zipf, R):
        """The oracle's CP-ALS against the reference's cpd_alto
        (include/cpd.hpp:47-191) on a 4-mode tensor with a 68-bit key (the
        128-bit build) at a specialised rank and a 5-mode tensor at a
        runtime rank (10, outside the reference's 8/16/100 specialisers);
        six iterations, the reference single-threaded."""
        dims = np.array(dims, np.uint64)
        cidx, vals = synth.powerlaw_coo(dims, 20000, zipf, seed=3)
        init = synth.init_values(int(dims.sum()) * R, seed=4)
        U0, off = [], 0
        for d in dims:
            U0.append(init[off:off + int(d) * R].reshape(int(d), R))
            off += int(d) * R
        t = O.RefTensor(dims, cidx, vals, 4)
        L = O.ref_lib(t.bits)
        L.ref_set_threads(1)
        try:
            Ur, lr, fr, itr = t.cpd_als(U0, np.ones(R), R, 6, 1e-12)
        finally:
            L.ref_set_threads(os.cpu_count() or 1)
            t.close()
        Uo, lo, fo, ito = O.cpd_als(O.build(dims, cidx, vals), U0, np.ones(R), R, 6, 1e-12)
        assert itr == ito
        np.testing.assert_allclose(fo, fr, rtol=1e-12)
        for a, b in zip(Ur, Uo):
            assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()

    def test_slicer_random_power_law(self):
        """The slicer restatement against the reference's
        StreamingSparseTensor (src/streaming_sptensor.cpp:69-327) on a
        tensor shaped like the CP-stream workload (a uniform time mode of 60
        steps, Zipf 1.1 on the other three, Poisson(3) values), whole
        batches compared: dims, every index and value.  The time mode is
        uniform so that no step is empty: the reference asserts on an empty
        step."""
        dims = np.array([60, 3000, 3000, 500], np.uint64)
        cidx, vals = synth.powerlaw_coo(dims, 30000, [None, 1.1, 1.1, 1.1], seed=8, values="poisson3")
        assert len(np.unique(cidx[0])) == 60
        for thr, lim in [(1, 1), (2000, 5), (1, 7)]:
            a = O.slice_stream(dims, cidx, vals, 0, thr, lim)
            b = O.ref_slice_stream(dims, cidx, vals, 0, thr, lim)
            assert len(a) == len(b)
            for x, y in zip(a, b):
                assert np.array_equal(x["dims"], y["dims"])
                assert np.array_equal(x["cidx"], y["cidx"])
                assert np.array_equal(x["vals"], y["vals"])

    def test_cpd_als_random(self):
        dims = np.array([30, 40, 50], np.uint64)
        cidx, vals = synth.uniform_coo(dims, 3000, seed=1)
        R = 8
        init = synth.init_values(int(dims.sum()) * R, seed=3)
        U0, off = [], 0
        for d in dims:
            U0.append(init[off:off + int(d) * R].reshape(int(d), R))
            off += int(d) * R
        t = O.RefTensor(dims, cidx, vals, 4)
        Ur, lr, fr, itr = t.cpd_als(U0, np.ones(R), R, 10, 1e-12)
        Uo, lo, fo, ito = O.cpd_als(O.build(dims, cidx, vals), U0, np.ones(R), R, 10, 1e-12)
        assert itr == ito
        np.testing.assert_allclose(fo, fr, rtol=1e-10)
        for a, b in zip(Ur, Uo):
            np.testing.assert_allclose(b, a, rtol=1e-8, atol=1e-10)


def test_slicer_matches_reference(golden):
    """The stream slicer restatement against the reference's
    StreamingSparseTensor batches (sort order, first-seen labels, batch cuts,
    growing dims), by digest."""
    import sys
    import os

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden as MG

    dims = np.array([12, 40, 30, 20], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 2500, seed=3)
    for case in golden["slicer"]:
        b = O.slice_stream(dims, cidx, vals, case["stream_mode"], case["nnz_threshold"], case["timeslice_limit"])
        assert len(b) == case["batches"]
        assert MG.slicer_digest(b) == case["sha256"], case
