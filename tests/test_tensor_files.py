"""Tensor files on the CPU: the oracle's restatement of the reference's
ImportSparseTensor against the digests of the compiled reference's reads
(tests/golden/make_golden.py), and the library's writer (host formatting,
no device work) against the reference's ExportSparseTensor bytes."""
import hashlib
import os
import sys

import numpy as np

import alto_b200 as A
import oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402


def test_reader_restatement_matches_reference(golden):
    """Comments, blank and whitespace-only lines, CRLF and tabs, a trailing
    space that adds a mode, no final newline, a one-byte last line, signed,
    overflowing and missing indices, and every strtod form (hexadecimal,
    inf/nan, long significands, over- and underflow), 1- and 0-based."""
    for name, data in MG.tns_cases().items():
        for zb in (0, 1):
            dims, c, v = O.read_tns(data, zb)
            want = golden["tns"][f"{name}_zb{zb}"]
            assert len(dims) == want["nmodes"] and c.shape[1] == want["nnz"], name
            assert MG.tns_digest(dims, c, v) == want["sha256"], (name, zb)


def test_writer_matches_reference(golden, tmp_path):
    dims, c, v = MG.export_tensor()
    for binary, key in ((False, "text"), (True, "binary")):
        path = tmp_path / f"x_{key}"
        A.write_tensor(path, dims, c, v, binary=binary)
        data = path.read_bytes()
        assert hashlib.sha256(data).hexdigest() == golden["tns_export"][key]
        assert data == (O.write_bin(dims, c, v) if binary else O.write_tns(c, v))


def test_writer_uint32_float32_inputs(tmp_path):
    """Narrow inputs are widened as the reference's IType and FType hold them."""
    rng = np.random.default_rng(5)
    dims = np.array([9, 8, 7, 6], np.uint64)
    c = np.stack([rng.integers(0, d, 500) for d in dims]).astype(np.uint32)
    v = (rng.random(500) * 100).astype(np.float32)
    A.write_tensor(tmp_path / "n.tns", dims, c, v)
    assert (tmp_path / "n.tns").read_bytes() == O.write_tns(c.astype(np.uint64), v.astype(np.float64))


def test_cpd_error_restatement_matches_reference(golden):
    dims, c, v, F = MG.cpd_error_case()
    assert abs(O.cpd_error(c, v, F) - golden["cpd_error"]["err"]) <= 1e-13


def test_cpd64_parses_the_reference_flags_without_a_gpu():
    """cpd64's option string is the reference's (src/main.cpp:93): -h prints
    the usage, -f takes the reference's integer (not a forgetting factor),
    and a generated tensor (-d/-s) is refused with a clear message before
    any device work."""
    import subprocess

    exe = os.path.join(os.path.dirname(A.__file__), "..", "cpd64")
    r = subprocess.run([exe, "-h"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "-f N" in r.stderr and "--forgetting" in r.stderr
    r = subprocess.run([exe, "-d", "10,10,10", "-s", "0.1", "-r", "4", "-f", "1"], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 1 and "-d/-s" in r.stderr
    r = subprocess.run([exe, "-q"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
