"""Tensor files on the device (alto_read_tensor): every value and index
equal to the reference's ImportSparseTensor (digests of the compiled
reference's reads) and to the oracle's restatement; binary files byte for
byte; text round trips through the writer."""
import os
import sys

import numpy as np
import pytest

import alto_b200 as A
import oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402

pytestmark = pytest.mark.gpu


def test_read_cases_match_reference(golden, tmp_path):
    for name, data in MG.tns_cases().items():
        path = tmp_path / f"{name}.tns"
        path.write_bytes(data)
        for zb in (0, 1):
            t = A.read_tensor(path, zero_based=bool(zb))
            c, v = t.to_host()
            want = golden["tns"][f"{name}_zb{zb}"]
            assert t.nmodes == want["nmodes"] and t.nnz == want["nnz"], name
            assert [int(x) for x in t.dims] == want["dims"], name
            assert MG.tns_digest(t.dims, c, v) == want["sha256"], (name, zb)
            st = t.stats()
            assert st["file_bytes"] == len(data)
            if name == "value_forms":
                assert st["host_values"] > 0  # hexadecimal, inf/nan, long significands
            if name in ("basic", "crlf_tabs", "comments_blank"):
                assert st["host_values"] == 0  # plain decimals stay on the device
            t.close()


def test_read_matches_oracle_random(tmp_path):
    """A larger file with mixed value forms and comment blocks, against the restatement."""
    rng = np.random.default_rng(8)
    lines = []
    for k in range(200_000):
        if k % 5003 == 0:
            lines.append("# comment %d\n\n" % k)
        lines.append("%d %d %d %s\n" % (rng.integers(1, 5000), rng.integers(1, 300), rng.integers(1, 40),
                                        MG._fmt_val(rng)))
    data = "".join(lines).encode()
    path = tmp_path / "r.tns"
    path.write_bytes(data)
    t = A.read_tensor(path)
    c, v = t.to_host()
    d0, c0, v0 = O.read_tns(data, 0)
    assert np.array_equal(t.dims, d0) and np.array_equal(c, c0)
    assert np.array_equal(v.view(np.uint64), v0.view(np.uint64))


def test_binary_round_trip(tmp_path):
    import torch

    rng = np.random.default_rng(9)
    dims = np.array([100, 200, 300, 7], np.uint64)
    c = np.stack([rng.integers(0, d, 50_000).astype(np.uint64) for d in dims])
    v = rng.normal(size=50_000)
    (tmp_path / "o.bin").write_bytes(O.write_bin(dims, c, v))
    t = A.read_tensor(tmp_path / "o.bin", binary=True)
    c1, v1 = t.to_host()
    assert np.array_equal(t.dims, dims) and np.array_equal(c1, c) and np.array_equal(v1, v)
    # the reference's own binary files carry stray bytes above the int nmodes
    raw = bytearray(O.write_bin(dims, c, v))
    raw[4:8] = b"\x9b\x7f\x00\x00"
    (tmp_path / "r.bin").write_bytes(bytes(raw))
    t2 = A.read_tensor(tmp_path / "r.bin", binary=True)
    assert t2.nmodes == 4 and np.array_equal(t2.to_host()[0], c)
    t2.close()
    idx, vals = t.tensors()  # device COO written back out
    A.write_tensor(tmp_path / "w.bin", t.dims, idx, vals, binary=True)
    assert (tmp_path / "w.bin").read_bytes() == (tmp_path / "o.bin").read_bytes()
    t.close()
    torch.cuda.synchronize()


def test_text_round_trip_large(tmp_path):
    """2M nonzeros from device memory, written (%g) and read back."""
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    n = 2_000_000
    dims = [4_000_000, 70_000, 900]
    idx = [torch.randint(0, d, (n,), generator=g, device="cuda", dtype=torch.int64) for d in dims]
    vals = torch.randn(n, generator=g, device="cuda", dtype=torch.float64).exp()
    A.write_tensor(tmp_path / "big.tns", dims, idx, vals)
    t = A.read_tensor(tmp_path / "big.tns")
    c, v = t.to_host()
    hc = np.stack([x.cpu().numpy().astype(np.uint64) for x in idx])
    assert np.array_equal(c, hc)
    want = np.array([float("%g" % x) for x in vals.cpu().numpy()])
    assert np.array_equal(v, want)
    assert np.array_equal(t.dims, hc.max(1) + 1)
    assert t.stats()["host_values"] == 0
    t.close()


def test_read_errors(tmp_path):
    (tmp_path / "empty.tns").write_bytes(b"")
    (tmp_path / "comments.tns").write_bytes(b"# only\n#\n\n")
    (tmp_path / "wide.tns").write_bytes(b"1 2 3 4 5 6 7 8 9 1.0\n")
    (tmp_path / "short.bin").write_bytes(O.write_bin([5, 5], np.zeros((2, 10), np.uint64), np.ones(10))[:-8])
    for name, binary, status in (("missing.tns", False, A.ERR_INVALID), ("empty.tns", False, A.ERR_INVALID),
                                 ("comments.tns", False, A.ERR_INVALID), ("wide.tns", False, A.ERR_UNSUPPORTED),
                                 ("short.bin", True, A.ERR_INVALID)):
        with pytest.raises(A.AltoError) as e:
            A.read_tensor(tmp_path / name, binary=binary)
        assert e.value.status == status, name


def test_read_feeds_encoder_and_slicer(tmp_path):
    """A file read to the device goes to the encoder and the slicer as it is."""
    rng = np.random.default_rng(2)
    dims = np.array([30, 50, 40, 20], np.uint64)
    c = np.stack([rng.integers(0, d, 3000).astype(np.uint64) for d in dims])
    v = rng.integers(1, 9, 3000).astype(np.float64)
    (tmp_path / "t.tns").write_bytes(O.write_tns(c, v))
    t = A.read_tensor(tmp_path / "t.tns")
    idx, vals = t.tensors()
    at = A.AltoTensor(t.dims, idx, vals, nprtn=1)
    assert at.nnz == 3000
    sl = A.Slicer(t.dims, idx, vals, 0)
    got = []
    while (b := sl.next(1, 1)) is not None:
        got.append(b.to_host())
    want = O.slice_stream(t.dims, c, v, 0, 1, 1)
    assert len(got) == len(want)
    for (gc, gv), w in zip(got, want):
        assert np.array_equal(gc, w["cidx"]) and np.array_equal(gv, w["vals"])


@pytest.mark.parametrize("binary", [False, True])
def test_cpd64_reads_files(tmp_path, binary):
    """The rebuilt cpd64 driver reads -i (text) and -b (binary) files through
    the device reader and checks its MTTKRP against the COO ground truth."""
    import subprocess

    rng = np.random.default_rng(6)
    dims = np.array([300, 200, 100], np.uint64)
    c = np.stack([rng.integers(0, d, 5000).astype(np.uint64) for d in dims])
    v = rng.random(5000)
    path = tmp_path / ("t.bin" if binary else "t.tns")
    path.write_bytes(O.write_bin(dims, c, v) if binary else O.write_tns(c, v))
    exe = os.path.join(os.path.dirname(A.__file__), "..", "cpd64")
    r = subprocess.run([exe, "-b" if binary else "-i", str(path), "-r", "8", "-c"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "tensor: 3 modes, 5000 nonzeros" in r.stdout
    assert r.stdout.count("correct") == 3 and "INCORRECT" not in r.stdout


@pytest.mark.parametrize("binary", [False, True])
def test_cpd64_takes_the_reference_flags(tmp_path, binary):
    """The reference's own flag strings, unchanged: -f 1 writes the tensor back
    in the other format as <N>D_<nnz>.bin / .tns in the working directory
    (src/main.cpp:268-289), -o names an output file, -x seeds, -e and -m set
    epsilon and iterations, and -l als runs CP-ALS."""
    import subprocess

    rng = np.random.default_rng(16)
    dims = np.array([60, 50, 40], np.uint64)
    c = np.stack([rng.integers(0, d, 3000).astype(np.uint64) for d in dims])
    key = (c[0] * 50 + c[1]) * 40 + c[2]
    _, first = np.unique(key, return_index=True)
    c = c[:, np.sort(first)]
    v = rng.integers(1, 9, c.shape[1]).astype(np.float64)  # (exact in %g)
    nnz = c.shape[1]
    path = tmp_path / ("t.bin" if binary else "t.tns")
    path.write_bytes(O.write_bin(dims, c, v) if binary else O.write_tns(c, v))
    exe = os.path.abspath(os.path.join(os.path.dirname(A.__file__), "..", "cpd64"))
    args = [exe, "-b" if binary else "-i", str(path), "-r", "4", "-m", "3", "-x", "5", "-e", "1e-5", "-f", "1",
            "-o", str(tmp_path / "out.tns"), "-l", "als"]
    r = subprocess.run(args, capture_output=True, text=True, timeout=120, cwd=tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "it: 2" in r.stdout
    back = tmp_path / ("3D_%d.%s" % (nnz, "tns" if binary else "bin"))
    read_dims = dims if binary else c.max(axis=1) + 1  # (text files: largest index + 1)
    assert back.read_bytes() == (O.write_tns(c, v) if binary else O.write_bin(read_dims, c, v))
    assert (tmp_path / "out.tns").read_bytes() == O.write_tns(c, v)


def test_many_values_left_to_host(tmp_path):
    """More than 2^20 values outside the device's fast path (17 significant
    digits): the listed lines overflow their first buffer and are listed
    again; every value still equals the C library's conversion."""
    rng = np.random.default_rng(10)
    n = 1_300_000  # (about 9 in 10 of these values need all 17 digits)
    c = np.stack([rng.integers(1, 500, n), rng.integers(1, 400, n), rng.integers(1, 300, n)])
    v = rng.normal(size=n) * 1e-3
    text = "".join("%d %d %d %.17g\n" % (a, b, d, x) for a, b, d, x in zip(c[0], c[1], c[2], v))
    (tmp_path / "long.tns").write_text(text)
    t = A.read_tensor(tmp_path / "long.tns")
    got_c, got_v = t.to_host()
    assert t.stats()["host_values"] > (1 << 20)
    assert np.array_equal(got_c, (c - 1).astype(np.uint64))
    want = np.array([float(ln.rsplit(" ", 1)[1]) for ln in text.splitlines()])
    assert np.array_equal(got_v, want)
    t.close()


def test_host_values_long_texts_and_numpy_style(tmp_path):
    """Values in numpy's savetxt style (%.18e: every one converted on the
    host from the text copied back) and value texts longer than the 64-byte
    copy (re-read from the file): each equals the C library's conversion."""
    rng = np.random.default_rng(14)
    n = 50_000
    v = rng.normal(size=n) * 10.0 ** rng.integers(-8, 8, n)
    vt = ["%.18e" % x for x in v]
    for k in range(0, n, 997):  # texts past the 64-byte copy
        vt[k] = "0." + "0" * (70 + k % 9) + "123456789012345678901234"
    lines = ["%d %d %d %s\n" % (k % 100 + 1, k % 37 + 1, k % 11 + 1, t) for k, t in enumerate(vt)]
    (tmp_path / "np.tns").write_text("".join(lines))
    t = A.read_tensor(tmp_path / "np.tns")
    _, got = t.to_host()
    assert t.stats()["host_values"] == n
    want = np.array([float(x) for x in vt])
    assert np.array_equal(got, want)
    t.close()
