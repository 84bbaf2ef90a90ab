"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run where the reference sources exist (the machines that run the GPU tests
have no copy):

    make -C oracle ref REF=<reference dir>   # oracle/_ref/libaltoref{64,128}.so
    python tests/golden/make_golden.py [path-to-reference]
    python tests/golden/make_golden.py only tns tns_export cpd_error   # refresh some parts

Inputs are the reference's own fixture tensors (tests/tensors/*.tns in the
reference project, 1-based text format, src/sptensor.cpp:74-158) plus seeded
synthetic cases.  Every output below comes from the compiled reference
(oracle/ref/ref_harness.cpp driving the reference's functions), so the
fixtures pin both the C restatement in oracle/ and the CUDA path:

* per tensor: the inputs (0-based cidx, values) as compressed arrays; the
  mode masks and alto_mask; SHA-256 digests of the sorted key array, the
  sorted values, prtn_ptr and prtn_intervals at P = 1, 3 and 8;
* MTTKRP (rank 8, factors from a seeded numpy generator) per mode: the full
  output for tensors under 1000 rows, else column sums, Frobenius norm and
  16 sampled rows;
* CP-ALS: fits of 8 iterations on med.tns at rank 8;
* CP-stream: final factor norms of a small seeded stream, unconstrained and
  non-negative; spCP-stream on the same stream;
* the stream slicer (StreamingSparseTensor): digests of the batches of a
  seeded 4-mode tensor for six (stream mode, nnz_threshold, timeslice_limit)
  cases;
* tensor files: digests of ImportSparseTensor's reads of ten edge-case
  .tns files (1- and 0-based) and of ExportSparseTensor's text and binary
  output;
* cpd_error of a seeded model against a seeded tensor.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "alto-stream_b200"))

import oracle as O  # noqa: E402
from alto_b200 import synth  # noqa: E402

FIXTURES = ["small.tns", "small4.tns", "small4_zeroidx.tns", "med.tns", "med4.tns", "med5.tns"]
RANK = 8


def load_tns(path, zero_based=False):
    rows = [ln.split() for ln in open(path) if ln.strip() and not ln.startswith("#")]
    a = np.array(rows, dtype=np.float64)
    idx = a[:, :-1].astype(np.int64)
    if not zero_based:
        idx -= 1
    return np.ascontiguousarray(idx.T.astype(np.uint64)), a[:, -1].copy()


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def factors_for(dims, seed=11):
    rng = np.random.default_rng(seed)
    return [rng.uniform(-1.0, 1.0, (int(d), RANK)) for d in dims]


def mttkrp_summary(out):
    if out.shape[0] < 1000:
        return {"full": out.tolist()}
    rows = np.linspace(0, out.shape[0] - 1, 16).astype(int)
    return {"colsum": out.sum(0).tolist(), "fro": float(np.linalg.norm(out)),
            "rows": rows.tolist(), "sample": out[rows].tolist()}


def main(ref_root):
    out_json = {}
    for fn in FIXTURES:
        zero = "zeroidx" in fn
        cidx, vals = load_tns(os.path.join(ref_root, "tests", "tensors", fn), zero_based=zero)
        dims = (cidx.max(1) + 1).astype(np.uint64)
        name = fn[:-4]
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), cidx=cidx.astype(np.uint32), vals=vals, dims=dims)
        rec = {"dims": dims.tolist(), "nnz": int(cidx.shape[1])}
        for P in (1, 3, 8):
            t = O.RefTensor(dims, cidx, vals, P)
            e = t.export()
            rec[f"P{P}"] = {"idx": digest(e["idx"]), "vals": digest(e["vals"]),
                            "prtn_ptr": e["prtn_ptr"].tolist(), "intervals": digest(e["intervals"])}
            if P == 1:
                rec["bits"] = t.bits
                rec["masks"] = [[int(a), int(b)] for a, b in e["masks"]]
                rec["alto_mask"] = [int(x) for x in e["alto_mask"]]
                F = factors_for(dims)
                rec["mttkrp"] = []
                for m in range(len(dims)):
                    fs = [f.copy() for f in F]
                    fs[m][:] = 0
                    res = t.mttkrp(m, fs, RANK)
                    rec["mttkrp"].append(mttkrp_summary(res[m]))
            t.close()
        out_json[name] = rec
        print(fn, "done", file=sys.stderr)

    # CP-ALS on med.tns
    d = np.load(os.path.join(HERE, "med.npz"))
    dims = d["dims"]
    init = synth.init_values(int(dims.sum()) * RANK, seed=3)
    U0, off = [], 0
    for n in dims:
        U0.append(init[off:off + int(n) * RANK].reshape(int(n), RANK))
        off += int(n) * RANK
    t = O.RefTensor(dims, d["cidx"], d["vals"], 4)
    _, lam, fits, it = t.cpd_als(U0, np.ones(RANK), RANK, 8, 1e-12)
    out_json["cpd_als_med"] = {"rank": RANK, "iters": it, "fits": fits.tolist(), "init_seed": 3,
                               "lambda": lam.tolist()}
    t.close()

    # CP-stream on a small seeded stream
    b = synth.stream_batches([200, 300, 50], 6, lambda rng, s: 400 + 50 * s, [1.1, 1.1, None], seed=5)
    np.savez_compressed(os.path.join(HERE, "stream_small.npz"),
                        **{f"dims{s}": x["dims"] for s, x in enumerate(b)},
                        **{f"cidx{s}": x["cidx"] for s, x in enumerate(b)},
                        **{f"vals{s}": x["vals"] for s, x in enumerate(b)})
    ntot = sum(int(x) for x in b[-1]["dims"]) * RANK + 1000
    iv = synth.init_values(ntot, seed=7)
    for nonneg in (0, 1):
        outs, lam, _ = O.ref_cpstream(b, 0, RANK, 20, 1e-5, nonneg, iv)
        out_json[f"cpstream_small_nonneg{nonneg}"] = {
            "rank": RANK, "max_iters": 20, "eps": 1e-5, "init_seed": 7, "n_init": ntot,
            "norms": [float(np.linalg.norm(o)) for o in outs],
            "colsums": [o.sum(0).tolist() for o in outs]}

    out_json["spcpstream_small"] = spcpstream_golden(b, iv, ntot)
    out_json["slicer"] = slicer_golden()
    out_json["tns"] = tns_golden()
    out_json["tns_export"] = export_golden()
    out_json["cpd_error"] = cpd_error_golden()

    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out_json, f, indent=1)


SLICER_CASES = [(0, 1, 1), (0, 300, 3), (0, 10**9, 4), (2, 1, 1), (2, 300, 3), (3, 50, 100)]


def slicer_digest(batches):
    h = hashlib.sha256()
    for x in batches:
        h.update(np.ascontiguousarray(x["dims"], np.uint64).tobytes())
        h.update(np.ascontiguousarray(x["cidx"], np.uint64).tobytes())
        h.update(np.ascontiguousarray(x["vals"], np.float64).tobytes())
    return h.hexdigest()


def slicer_golden():
    """The reference's StreamingSparseTensor batches of a seeded 4-mode tensor."""
    dims = np.array([12, 40, 30, 20], np.uint64)
    cidx, vals = synth.uniform_coo(dims, 2500, seed=3)
    out = []
    for t, thr, lim in SLICER_CASES:
        b = O.ref_slice_stream(dims, cidx, vals, t, thr, lim)
        out.append({"stream_mode": t, "nnz_threshold": thr, "timeslice_limit": lim, "batches": len(b),
                    "sha256": slicer_digest(b)})
    return out


def spcpstream_golden(b, iv, ntot):
    """spCP-stream (the reference's row-sparse model) on the small stream."""
    outs, lam, _ = O.ref_spcpstream(b, 0, RANK, 10, 1e-5, iv)
    return {"rank": RANK, "max_iters": 10, "eps": 1e-5, "init_seed": 7, "n_init": ntot,
            "norms": [float(np.linalg.norm(o)) for o in outs], "colsums": [o.sum(0).tolist() for o in outs]}


def _fmt_val(rng):
    r = rng.random()
    if r < 0.6:
        return "%g" % (rng.random() * 10.0 ** int(rng.integers(-6, 7)))
    if r < 0.8:
        return "%d" % rng.integers(0, 100)
    if r < 0.9:
        return "%.10e" % rng.normal()
    return "%.17g" % rng.normal()


def tns_cases():
    """Text tensor files covering the reader's edge cases, as bytes."""
    cases = {
        "basic": b"1 1 1 1.5\n2 3 1 2\n3 2 4 -0.25\n",
        "comments_blank": b"# header\n\n1 2 3 4\n#mid\n\n2 2 2 5e-1\n   \n3 1 1 7\n",
        "crlf_tabs": b"1\t2\t3\t1.25\r\n 4  5 6   2.5\r\n7 8 9 3\r\n",
        "trailing_space_first": b"1 2 3 4.5 \n2 3 4 5.5\n3 1 1 6.25\n",
        "no_final_newline": b"1 2 3 4\n5 6 7 8",
        "single_char_last": b"1 2 3 4\n2 2 2 9\n5",
        "index_forms": (b"+3 2 1 1\n-1 2 2 2\n18446744073709551615 1 1 3\n18446744073709551616 1 1 4\n"
                        b"0 1 1 5\nabc 1 2 3\n4 5 6\n"),
    }
    forms = ["1e-3", "2.5E+02", "-0.0", "+7", ".5", "5.", "1e", "0x1.8p1", "inf", "-INF", "nan",
             "1.7976931348623157e308", "4.9e-324", "123456789012345678901234567890", "0.1",
             "3.14159265358979323846", "1e400", "1e-400", "007", "9007199254740993", "12345678901234567e-5",
             "1.0000000000000000000000001", "0e5", "1e22", "1e23", "123e20", "5e-22", "0x", "-.5e+1", "1.e2",
             "9007199254740992", "0.000000000000000000000000000001234", "1E+0010"]
    cases["value_forms"] = "".join("%d %d %d %s\n" % (k + 1, k % 5 + 1, k % 3 + 1, f)
                                   for k, f in enumerate(forms)).encode()
    rng = np.random.default_rng(21)
    cases["five_modes"] = "".join(" ".join(str(int(x)) for x in rng.integers(1, 40, 5)) + " " + _fmt_val(rng) + "\n"
                                  for _ in range(300)).encode()
    lines = []
    for k in range(20000):
        if k % 997 == 0:
            lines.append("# block %d\n" % k)
        sep = " " if k % 7 else "\t"
        lines.append(sep.join(str(int(x)) for x in rng.integers(1, 1000, 3)) + sep + _fmt_val(rng) + "\n")
    cases["random_mixed"] = "".join(lines).encode()
    return cases


def tns_digest(dims, cidx, vals):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(dims, np.uint64).tobytes())
    h.update(np.ascontiguousarray(cidx, np.uint64).tobytes())
    h.update(np.ascontiguousarray(vals, np.float64).tobytes())
    return h.hexdigest()


def tns_golden():
    """The reference's ImportSparseTensor of every case, 1- and 0-based, by digest."""
    import tempfile

    out = {}
    with tempfile.TemporaryDirectory() as d:
        for name, data in tns_cases().items():
            path = os.path.join(d, name + ".tns")
            with open(path, "wb") as f:
                f.write(data)
            for zb in (0, 1):
                dims, c, v = O.ref_import(path, 0, zb)
                out[f"{name}_zb{zb}"] = {"nmodes": len(dims), "nnz": int(c.shape[1]), "dims": [int(x) for x in dims],
                                         "sha256": tns_digest(dims, c, v)}
    return out


def export_tensor():
    """A seeded tensor whose values exercise %g (signed zero, 1e6, tiny, inf, nan)."""
    rng = np.random.default_rng(31)
    dims = np.array([50, 60, 70], np.uint64)
    c = np.stack([rng.integers(0, d, 1000).astype(np.uint64) for d in dims])
    v = np.concatenate([rng.random(500) * 10, rng.integers(-5, 5, 500).astype(float)])
    v[3:11] = [-0.0, 1e6, 123456.0, 1e-5, np.inf, -np.nan, 0.0, 999999.0]
    return dims, c, v


def export_golden():
    """SHA-256 of the reference's ExportSparseTensor output, text and binary.
    The binary header's first word is written from the struct's int nmodes
    with sizeof(IType) = 8 bytes (src/sptensor.cpp:59), so its upper four
    bytes are whatever follows the int in memory; they are zeroed before
    hashing."""
    import tempfile

    dims, c, v = export_tensor()
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for fmt, name in ((0, "text"), (1, "binary")):
            path = os.path.join(d, "x")
            O.ref_export(path, fmt, dims, c, v)
            with open(path, "rb") as f:
                data = bytearray(f.read())
            if fmt == 1:
                data[4:8] = bytes(4)
            out[name] = hashlib.sha256(bytes(data)).hexdigest()
    return out


def cpd_error_case():
    """A seeded tensor and model for cpd_error."""
    rng = np.random.default_rng(41)
    dims = np.array([30, 40, 20, 10], np.uint64)
    c = np.stack([rng.integers(0, d, 2000).astype(np.uint64) for d in dims])
    v = rng.random(2000)
    F = [rng.random((int(d), 8)) * 0.3 for d in dims]
    return dims, c, v, F


def cpd_error_golden():
    dims, c, v, F = cpd_error_case()
    return {"err": O.ref_cpd_error(dims, c, v, F)}


PARTS = {"tns": tns_golden, "tns_export": export_golden, "cpd_error": cpd_error_golden}

if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[1] == "only":  # refresh the named parts of golden.json
        with open(os.path.join(HERE, "golden.json")) as f:
            g = json.load(f)
        for part in sys.argv[2:]:
            g[part] = PARTS[part]()
        with open(os.path.join(HERE, "golden.json"), "w") as f:
            json.dump(g, f, indent=1)
    else:
        default = os.environ.get("ALTO_REFERENCE",
                                 os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference"))
        main(sys.argv[1] if len(sys.argv) > 1 else default)
