"""ctypes wrappers for the ALTO oracle (test infrastructure only).

Two test libraries are wrapped here:

* ``liboracle.so`` -- the single-threaded FP64 C restatement of the reference
  algorithm (``oracle/alto_oracle.c``), the oracle the CUDA path's parity
  tests compare against;
* ``_ref/libaltoref{64,128}.so`` -- the reference implementation itself,
  compiled from its own sources by ``oracle/ref/Makefile`` and driven by
  ``oracle/ref/ref_harness.cpp``; it pins the restatement and is the timed
  CPU baseline of ``bench.py``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its CPU
baseline and reference arm) import this module.  The product library never
does: it has no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = {}


def _ptr(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


def _dptrs(arrs):
    """double** over a list of contiguous float64 arrays."""
    arr = (POINTER(c_double) * len(arrs))()
    for i, a in enumerate(arrs):
        assert a.dtype == np.float64 and a.flags.c_contiguous
        arr[i] = a.ctypes.data_as(POINTER(c_double))
    return arr


def lib():
    """Load (building if needed) the C restatement."""
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            import subprocess

            subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        L = ctypes.CDLL(path)
        L.ora_setup_masks.restype = c_int
        L.ora_alto_build.restype = c_int
        L.ora_cpd_als.restype = c_int
        L.ora_cpstream.restype = c_int
        _LIB = L
    return _LIB


def ref_available(bits=64):
    return os.path.exists(os.path.join(HERE, "_ref", f"libaltoref{bits}.so"))


def ref_lib(bits=64):
    """Load the compiled reference (64- or 128-bit ALTO keys)."""
    if bits not in _REF:
        path = os.path.join(HERE, "_ref", f"libaltoref{bits}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref REF=<reference dir>` where the reference sources exist")
        L = ctypes.CDLL(path)
        L.ref_alto_create.restype = c_void_p
        L.ref_alto_destroy.argtypes = [c_void_p]
        L.ref_alto_export.argtypes = [c_void_p] + [c_void_p] * 6
        L.ref_alto_nprtn.argtypes = [c_void_p]
        L.ref_mttkrp.argtypes = [c_void_p, c_int, c_void_p, c_int]
        L.ref_coo_mttkrp.argtypes = [c_void_p, c_int, c_void_p, c_int]
        L.ref_mttkrp_time.argtypes = [c_void_p, c_int, c_void_p, c_int, c_int]
        L.ref_mttkrp_time.restype = c_double
        L.ref_cpd_als.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_int, c_double, c_void_p]
        L.ref_cpd_als.restype = c_int
        L.ref_cpstream.restype = c_int
        L.ref_get_num_ptrn.argtypes = [c_uint64]
        L.ref_get_num_ptrn.restype = c_int
        L.ref_max_threads.restype = c_int
        L.ref_set_threads.argtypes = [c_int]
        _REF[bits] = L
    return _REF[bits]


def join128(lohi):
    """(n, 2) uint64 lo/hi pairs -> list of Python ints."""
    lohi = np.asarray(lohi, dtype=np.uint64).reshape(-1, 2)
    return [int(lo) | (int(hi) << 64) for lo, hi in lohi]


def mode_bits(dim):
    return 0 if dim <= 1 else int(dim - 1).bit_length()


# ------------------------------------------------------------ restatement

def setup_masks(dims, max_bits=128):
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    N = len(dims)
    masks = np.zeros(2 * N, np.uint64)
    am = np.zeros(2, np.uint64)
    pos = np.zeros(N, np.int32)
    bits = lib().ora_setup_masks(c_int(N), _ptr(dims), c_int(max_bits), _ptr(masks), _ptr(am), _ptr(pos))
    if bits < 0:
        raise ValueError("index bits exceed key width")
    return dict(masks=masks.reshape(N, 2), alto_mask=am, mode_pos=pos, alto_bits=bits)


def build(dims, cidx, vals, nprtn=1, max_bits=128):
    """Encode, sort and partition a COO tensor the way create_alto does."""
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    cidx = np.ascontiguousarray(cidx, dtype=np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    N, nnz = cidx.shape
    masks = np.zeros(2 * N, np.uint64)
    am = np.zeros(2, np.uint64)
    idx = np.zeros(2 * max(nnz, 1), np.uint64)
    sv = np.zeros(max(nnz, 1), np.float64)
    perm = np.zeros(max(nnz, 1), np.uint64)
    pp = np.zeros(nprtn + 1, np.uint64)
    iv = np.zeros(2 * nprtn * N, np.uint64)
    bits = lib().ora_alto_build(c_int(N), _ptr(dims), c_uint64(nnz), _ptr(cidx), _ptr(vals),
                                c_int(max_bits), c_int(nprtn), _ptr(masks), _ptr(am), _ptr(idx),
                                _ptr(sv), _ptr(perm), _ptr(pp), _ptr(iv))
    if bits < 0:
        raise ValueError("index bits exceed key width")
    return dict(dims=dims, nmodes=N, nnz=nnz, masks=masks.reshape(N, 2), alto_mask=am,
                idx=idx[: 2 * nnz].reshape(nnz, 2), vals=sv[:nnz], perm=perm[:nnz],
                prtn_ptr=pp, intervals=iv.reshape(nprtn, N, 2), alto_bits=bits)


def partition(enc, nprtn):
    N, nnz = enc["nmodes"], enc["nnz"]
    pp = np.zeros(nprtn + 1, np.uint64)
    iv = np.zeros(2 * nprtn * N, np.uint64)
    lib().ora_partition(c_int(N), _ptr(enc["dims"]), c_uint64(nnz), _ptr(np.ascontiguousarray(enc["idx"])),
                        _ptr(np.ascontiguousarray(enc["masks"])), c_int(nprtn), _ptr(pp), _ptr(iv))
    return pp, iv.reshape(nprtn, N, 2)


def decode(enc):
    N, nnz = enc["nmodes"], enc["nnz"]
    out = np.zeros((N, max(nnz, 1)), np.uint64)
    lib().ora_decode(c_int(N), c_uint64(nnz), _ptr(np.ascontiguousarray(enc["idx"])),
                     _ptr(np.ascontiguousarray(enc["masks"])), _ptr(out))
    return out[:, :nnz]


def mttkrp(enc, mode, factors, rank):
    """Accumulate the ALTO MTTKRP of `mode` into factors[mode] (FP64)."""
    fs = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
    lib().ora_mttkrp(c_int(enc["nmodes"]), c_uint64(enc["nnz"]), _ptr(np.ascontiguousarray(enc["idx"])),
                     _ptr(np.ascontiguousarray(enc["vals"], dtype=np.float64)),
                     _ptr(np.ascontiguousarray(enc["masks"])), c_int(mode), _dptrs(fs), c_int(rank))
    return fs


def coo_mttkrp(cidx, vals, mode, factors, rank):
    cidx = np.ascontiguousarray(cidx, dtype=np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    fs = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
    lib().ora_coo_mttkrp(c_int(cidx.shape[0]), c_uint64(cidx.shape[1]), _ptr(cidx), _ptr(vals),
                         c_int(mode), _dptrs(fs), c_int(rank))
    return fs


def cpd_als(enc, U, lam, rank, max_iters, eps, fit_exact=False):
    Us = [np.array(u, dtype=np.float64, copy=True, order="C") for u in U]
    lam = np.array(lam, dtype=np.float64, copy=True)
    fits = np.zeros(max(max_iters, 1), np.float64)
    it = lib().ora_cpd_als(c_int(enc["nmodes"]), _ptr(enc["dims"]), c_uint64(enc["nnz"]),
                           _ptr(np.ascontiguousarray(enc["idx"])), _ptr(np.ascontiguousarray(enc["vals"])),
                           _ptr(np.ascontiguousarray(enc["masks"])), _dptrs(Us), _ptr(lam), c_int(rank),
                           c_int(max_iters), c_double(eps), c_int(1 if fit_exact else 0), _ptr(fits))
    return Us, lam, fits[: abs(it)], it


def _stream_args(batches):
    dims = np.ascontiguousarray(np.concatenate([np.asarray(b["dims"], np.uint64) for b in batches]))
    nnz = np.ascontiguousarray([b["cidx"].shape[1] for b in batches], dtype=np.uint64)
    cidx = np.ascontiguousarray(np.concatenate([np.asarray(b["cidx"], np.uint64).ravel() for b in batches]))
    vals = np.ascontiguousarray(np.concatenate([np.asarray(b["vals"], np.float64) for b in batches]))
    return dims, nnz, cidx, vals


def _stream_outputs(batches, stream_mode, rank):
    last = batches[-1]["dims"]
    total_t = int(sum(int(b["dims"][stream_mode]) for b in batches))
    outs = []
    for m, d in enumerate(last):
        n = total_t if m == stream_mode else int(d)
        outs.append(np.zeros((max(n, 1), rank), np.float64))
    return outs


def cpstream(batches, stream_mode, rank, max_iters, eps, nonneg, init_vals, forgetting=0.99):
    """CP-stream over a list of batches {dims, cidx (N x nnz), vals}."""
    N = len(batches[0]["dims"])
    dims, nnz, cidx, vals = _stream_args(batches)
    init_vals = np.ascontiguousarray(init_vals, dtype=np.float64)
    outs = _stream_outputs(batches, stream_mode, rank)
    lam = np.zeros(rank, np.float64)
    inner = np.zeros(len(batches), np.int32)
    tt = lib().ora_cpstream(c_int(N), c_int(stream_mode), c_int(len(batches)), _ptr(dims), _ptr(nnz),
                            _ptr(cidx), _ptr(vals), c_int(rank), c_int(max_iters), c_double(eps),
                            c_int(1 if nonneg else 0), c_double(forgetting), _ptr(init_vals),
                            c_uint64(len(init_vals)), _dptrs(outs), _ptr(lam), _ptr(inner))
    if tt < 0:
        raise RuntimeError("oracle CP-stream: factorisation failed")
    return outs, lam, inner


def spcpstream(batches, stream_mode, rank, max_iters, eps, init_vals, forgetting=0.99):
    """spCP-stream (row-sparse updates) over a list of batches."""
    N = len(batches[0]["dims"])
    dims, nnz, cidx, vals = _stream_args(batches)
    init_vals = np.ascontiguousarray(init_vals, dtype=np.float64)
    outs = _stream_outputs(batches, stream_mode, rank)
    lam = np.zeros(rank, np.float64)
    inner = np.zeros(len(batches), np.int32)
    tt = lib().ora_spcpstream(c_int(N), c_int(stream_mode), c_int(len(batches)), _ptr(dims), _ptr(nnz),
                              _ptr(cidx), _ptr(vals), c_int(rank), c_int(max_iters), c_double(eps),
                              c_double(forgetting), _ptr(init_vals), c_uint64(len(init_vals)), _dptrs(outs),
                              _ptr(lam), _ptr(inner))
    if tt < 0:
        raise RuntimeError("oracle spCP-stream failed")
    return outs, lam, inner


def slice_stream(dims, cidx, vals, stream_mode, nnz_threshold=1, timeslice_limit=1):
    """The reference's stream slicer (StreamingSparseTensor,
    src/streaming_sptensor.cpp:69-264), restated: sort by the stream mode and
    then the following modes cyclically (tt_sort, src/sort.cpp:477-519),
    relabel every other mode in first-seen order over the sorted tensor, and
    cut batches of whole time steps (next_dynamic_batch): a batch grows by
    one time step at a time while it holds fewer than nnz_threshold nonzeros
    and fewer than timeslice_limit steps.  Batch time indices are local;
    the other dims are the running maximum of index + 1.  Returns a list of
    {dims, cidx, vals}."""
    cidx = np.asarray(cidx, np.uint64)
    vals = np.asarray(vals, np.float64)
    N, nnz = cidx.shape
    t = stream_mode
    prio = [(t + m) % N for m in range(N)]
    perm = np.lexsort([cidx[m] for m in reversed(prio)])
    c = cidx[:, perm].copy()
    v = vals[perm]
    for m in range(N):
        if m == t:
            continue
        u, first = np.unique(c[m], return_index=True)
        lab = np.zeros(int(dims[m]) if len(dims) else 0, np.uint64)
        lab[u[np.argsort(first)]] = np.arange(len(u), dtype=np.uint64)
        c[m] = lab[c[m]]
    time = c[t]
    out, batch, ptr = [], 0, 0
    prev = np.zeros(N, np.uint64)
    while ptr < nnz:
        first_batch = batch
        start = int(np.searchsorted(time, batch, side="left")) if ptr == 0 else ptr
        start = max(start, ptr)
        end = start
        local = []
        while end - start < nnz_threshold and end < nnz:
            e2 = int(np.searchsorted(time, batch + 1, side="left"))
            local.extend([batch - first_batch] * (e2 - end))
            end = e2
            batch += 1
            if batch - first_batch >= timeslice_limit:
                break
        bd = np.zeros(N, np.uint64)
        bc = c[:, start:end].copy()
        bc[t] = np.asarray(local, np.uint64)
        for m in range(N):
            if m == t:
                bd[m] = batch - first_batch
            else:
                # an empty batch counts as max index 0 (dim = 0 + 1): the
                # reference asserts nnz > 0 first (:229), so this is its
                # behaviour with assertions compiled out
                mx = int(bc[m].max()) + 1 if end > start else 1
                bd[m] = max(mx, int(prev[m]))
                prev[m] = bd[m]
        out.append(dict(dims=bd, cidx=bc, vals=v[start:end].copy()))
        ptr = end
    return out


def ref_slice_stream(dims, cidx, vals, stream_mode, nnz_threshold=1, timeslice_limit=1, bits=64):
    """The compiled reference's slicer over the same tensor (see the harness)."""
    L = ref_lib(bits)
    dims = np.ascontiguousarray(dims, np.uint64)
    cidx = np.ascontiguousarray(cidx, np.uint64)
    vals = np.ascontiguousarray(vals, np.float64)
    N, nnz = cidx.shape
    maxb = int(dims[stream_mode]) + 1
    bdims = np.zeros(maxb * N, np.uint64)
    bnnz = np.zeros(maxb, np.uint64)
    oc = np.zeros(N * nnz, np.uint64)
    ov = np.zeros(nnz, np.float64)
    nb = L.ref_slice_stream(c_int(N), _ptr(dims), c_uint64(nnz), _ptr(cidx), _ptr(vals), c_int(stream_mode),
                            c_uint64(nnz_threshold), c_uint64(timeslice_limit), c_int(maxb), _ptr(bdims),
                            _ptr(bnnz), _ptr(oc), _ptr(ov))
    out, oi, ovv = [], 0, 0
    for b in range(nb):
        n = int(bnnz[b])
        out.append(dict(dims=bdims[b * N:(b + 1) * N].copy(), cidx=oc[oi:oi + N * n].reshape(N, n).copy(),
                        vals=ov[ovv:ovv + n].copy()))
        oi += N * n
        ovv += n
    return out


def cpd_error(cidx, vals, factors):
    """cpd_error (src/streaming_cpd.cpp:368-464), restated: with unit
    weights, inner = sum_k v_k sum_r prod_m U_m[i_m(k), r] (the reference
    forms it as an MTTKRP of the shortest mode followed by a dot product),
    ||X||^2 = sum v^2, ||M||^2 = sum_ij prod_m (U_m^T U_m)_ij
    (kruskal_norm, src/kruskal_model.cpp:400-443); the result is
    sqrt(||X||^2 + ||M||^2 - 2 inner) / ||X||."""
    cidx = np.asarray(cidx, np.int64)
    vals = np.asarray(vals, np.float64)
    R = factors[0].shape[1]
    prod = np.ones((len(vals), R))
    for m, U in enumerate(factors):
        prod *= U[cidx[m]]
    inner = float(vals @ prod.sum(1))
    xx = float(vals @ vals)
    G = np.ones((R, R))
    for U in factors:
        G *= U.T @ U
    z = abs(float(G.sum()))
    return float(np.sqrt(xx + z - 2 * inner) / np.sqrt(xx))


def ref_cpd_error(dims, cidx, vals, factors):
    """The compiled reference's cpd_error of the given model against the tensor."""
    L = ref_lib(64)
    L.ref_cpd_error.restype = c_double
    dims = np.ascontiguousarray(dims, np.uint64)
    cidx = np.ascontiguousarray(cidx, np.uint64)
    vals = np.ascontiguousarray(vals, np.float64)
    F = [np.ascontiguousarray(f, np.float64) for f in factors]
    ptrs = (c_void_p * len(F))(*[f.ctypes.data for f in F])
    return L.ref_cpd_error(c_int(len(F)), _ptr(dims), c_uint64(cidx.shape[1]), _ptr(cidx), _ptr(vals), ptrs,
                           c_int(F[0].shape[1]))


# ------------------------------------------------------------- tensor files

_SPACE = b" \t\n\v\f\r"
_U64 = (1 << 64) - 1


def _strtoull(line, p):
    """C strtoull(line + p, &end, 10) on one NUL-terminated line: (value, end)."""
    q = p
    n = len(line)
    while q < n and line[q] in _SPACE:
        q += 1
    neg = False
    if q < n and line[q] in b"+-":
        neg = line[q] == ord("-")
        q += 1
    s = q
    while q < n and 48 <= line[q] <= 57:
        q += 1
    if q == s:
        return 0, p  # no conversion: end = start
    v = int(line[s:q])
    if v > _U64:
        return _U64, q
    return ((-v) & _U64 if neg else v), q


def _strtod(line, p):
    """C strtod(line + p, &end) on one line: decimal, hexadecimal, inf and nan
    forms (the shortest-round-trip decimal conversion is correctly rounded
    in both C and Python)."""
    import re

    q = p
    n = len(line)
    while q < n and line[q] in _SPACE:
        q += 1
    rest = line[q:].decode("latin-1")
    m = re.match(r"[+-]?0[xX](?:[0-9a-fA-F]+\.?[0-9a-fA-F]*|\.[0-9a-fA-F]+)(?:[pP][+-]?[0-9]+)?", rest)
    if m:
        txt = m.group(0)
        sign = -1.0 if txt[0] == "-" else 1.0
        body = txt.lstrip("+-")
        if not re.search(r"[pP]", body):
            body += "p0"
        return sign * float.fromhex(body), q + len(txt)
    m = re.match(r"[+-]?(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?", rest)
    if m:
        return float(m.group(0)), q + len(m.group(0))
    m = re.match(r"[+-]?(?:inf(?:inity)?|nan(?:\([0-9A-Za-z_]*\))?)", rest, re.IGNORECASE)
    if m:
        txt = m.group(0)
        neg = txt[0] == "-"
        body = txt.lstrip("+-").lower()
        v = float("inf") if body.startswith("inf") else float("nan")
        return (-v if neg else v), q + len(txt)
    return 0.0, p


def _tns_lines(data):
    """getline over the file: each line with its newline; the valid ones
    (more than one byte read and not starting with '#')."""
    out = []
    pos = 0
    n = len(data)
    while pos < n:
        e = data.find(b"\n", pos)
        e = n if e < 0 else e + 1
        line = data[pos:e]
        if len(line) > 1 and line[0] != ord("#"):
            out.append(line)
        pos = e
    return out


def read_tns(data, zero_based=0):
    """ImportSparseTensor(TEXT_FORMAT) (src/sptensor.cpp:74-158), restated on
    the file's bytes: the mode count is the first valid line's token count
    (strtok on space and tab) minus one; every valid line gives a nonzero
    from nmodes strtoull calls and one strtod; dims[m] is the maximum of
    index + zero_based, and the stored index is index - (1 - zero_based),
    all in uint64 arithmetic.  Returns (dims, cidx [nmodes, nnz], vals)."""
    import re

    lines = _tns_lines(data)
    if not lines:
        return np.zeros(0, np.uint64), np.zeros((0, 0), np.uint64), np.zeros(0)
    first = lines[0].split(b"\0")[0]
    nmodes = len([t for t in re.split(rb"[ \t]+", first) if t]) - 1
    one_based = 0 if zero_based else 1
    dims = [0] * nmodes
    cidx = np.zeros((max(nmodes, 0), len(lines)), np.uint64)
    vals = np.zeros(len(lines))
    for k, line in enumerate(lines):
        line = line.split(b"\0")[0]
        p = 0
        for m in range(nmodes):
            v, p = _strtoull(line, p)
            dims[m] = max(dims[m], (v + zero_based) & _U64)
            cidx[m, k] = (v - one_based) & _U64
        vals[k], p = _strtod(line, p)
    return np.array(dims, np.uint64), cidx, vals


def _fmt_g(v):
    """printf("%g") as glibc writes it."""
    import math

    if math.isnan(v):
        return "-nan" if math.copysign(1.0, v) < 0 else "nan"
    return "%g" % v


def write_tns(cidx, vals):
    """ExportSparseTensor(TEXT_FORMAT) (src/sptensor.cpp:48-56): per nonzero
    "%llu " of index + 1 for every mode, then "%g\n" of the value."""
    cidx = np.asarray(cidx, np.uint64)
    out = []
    for k in range(len(vals)):
        out.append("".join("%d " % ((int(cidx[m, k]) + 1) & _U64) for m in range(cidx.shape[0]))
                   + _fmt_g(float(vals[k])) + "\n")
    return "".join(out).encode()


def write_bin(dims, cidx, vals):
    """ExportSparseTensor(BINARY_FORMAT) (src/sptensor.cpp:57-69): uint64
    nmodes, dims, nnz, the index arrays mode by mode, float64 values."""
    cidx = np.asarray(cidx, np.uint64)
    head = np.array([cidx.shape[0]] + [int(d) for d in dims] + [cidx.shape[1]], np.uint64)
    return head.tobytes() + np.ascontiguousarray(cidx).tobytes() + np.asarray(vals, np.float64).tobytes()


def ref_import(path, fmt=0, zero_based=0):
    """The compiled reference's ImportSparseTensor of `path`."""
    L = ref_lib(64)
    nm, nnz = c_uint64(), c_uint64()
    dims = np.zeros(16, np.uint64)
    p = str(path).encode()
    if L.ref_import_info(p, c_int(fmt), c_uint64(zero_based), ctypes.byref(nm), _ptr(dims), ctypes.byref(nnz)):
        raise FileNotFoundError(path)
    c = np.zeros((nm.value, nnz.value), np.uint64)
    v = np.zeros(nnz.value)
    L.ref_import_data(p, c_int(fmt), c_uint64(zero_based), _ptr(c), _ptr(v))
    return dims[: nm.value].copy(), c, v


def ref_export(path, fmt, dims, cidx, vals):
    """The compiled reference's ExportSparseTensor to `path`."""
    L = ref_lib(64)
    dims = np.ascontiguousarray(dims, np.uint64)
    cidx = np.ascontiguousarray(cidx, np.uint64)
    vals = np.ascontiguousarray(vals, np.float64)
    L.ref_export(str(path).encode(), c_int(fmt), c_int(cidx.shape[0]), _ptr(dims), c_uint64(cidx.shape[1]),
                 _ptr(cidx), _ptr(vals))


# ------------------------------------------------------ compiled reference

class RefTensor:
    """The reference's AltoTensor, built by create_alto (or init/update_salto)."""

    def __init__(self, dims, cidx, vals, nprtn, stream_mode=-1, bits=None):
        dims = np.ascontiguousarray(dims, dtype=np.uint64)
        self.cidx = np.ascontiguousarray(cidx, dtype=np.uint64)
        self.vals_in = np.ascontiguousarray(vals, dtype=np.float64)
        if bits is None:
            bits = 64 if sum(mode_bits(int(d)) for d in dims) <= 64 else 128
        self.bits = bits
        self.L = ref_lib(bits)
        self.dims = dims
        self.N = len(dims)
        self.nnz = self.cidx.shape[1]
        self.h = self.L.ref_alto_create(c_int(self.N), _ptr(dims), c_uint64(self.nnz), _ptr(self.cidx),
                                        _ptr(self.vals_in), c_int(nprtn), c_int(stream_mode))
        self.nprtn = self.L.ref_alto_nprtn(self.h)

    def export(self):
        N, nnz, P = self.N, self.nnz, self.nprtn
        masks = np.zeros(2 * N, np.uint64)
        am = np.zeros(2, np.uint64)
        idx = np.zeros(2 * max(nnz, 1), np.uint64)
        vals = np.zeros(max(nnz, 1), np.float64)
        pp = np.zeros(P + 1, np.uint64)
        iv = np.zeros(2 * P * N, np.uint64)
        self.L.ref_alto_export(self.h, _ptr(masks), _ptr(am), _ptr(idx), _ptr(vals), _ptr(pp), _ptr(iv))
        return dict(masks=masks.reshape(N, 2), alto_mask=am, idx=idx[: 2 * nnz].reshape(nnz, 2),
                    vals=vals[:nnz], prtn_ptr=pp, intervals=iv.reshape(P, N, 2))

    def mttkrp(self, mode, factors, rank):
        fs = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
        self.L.ref_mttkrp(self.h, mode, ctypes.cast(_dptrs(fs), c_void_p), rank)
        return fs

    def coo_mttkrp(self, mode, factors, rank):
        fs = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
        self.L.ref_coo_mttkrp(self.h, mode, ctypes.cast(_dptrs(fs), c_void_p), rank)
        return fs

    def mttkrp_time(self, mode, factors, rank, reps):
        fs = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
        return self.L.ref_mttkrp_time(self.h, mode, ctypes.cast(_dptrs(fs), c_void_p), rank, reps)

    def cpd_als(self, U, lam, rank, max_iters, eps):
        Us = [np.array(u, dtype=np.float64, copy=True, order="C") for u in U]
        lam = np.array(lam, dtype=np.float64, copy=True)
        fits = np.zeros(max(max_iters, 1), np.float64)
        it = self.L.ref_cpd_als(self.h, ctypes.cast(_dptrs(Us), c_void_p), _ptr(lam), rank, max_iters,
                                eps, _ptr(fits))
        return Us, lam, fits[:it], it

    def close(self):
        if self.h:
            self.L.ref_alto_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_spcpstream(batches, stream_mode, rank, max_iters, eps, init_vals, bits=64):
    """The reference's spCP-stream (ALTO) over the same batches (forgetting 0.99)."""
    L = ref_lib(bits)
    N = len(batches[0]["dims"])
    dims, nnz, cidx, vals = _stream_args(batches)
    init_vals = np.ascontiguousarray(init_vals, dtype=np.float64)
    outs = _stream_outputs(batches, stream_mode, rank)
    lam = np.zeros(rank, np.float64)
    secs = np.zeros(len(batches), np.float64)
    L.ref_spcpstream(c_int(N), c_int(stream_mode), c_int(len(batches)), _ptr(dims), _ptr(nnz), _ptr(cidx),
                     _ptr(vals), c_int(rank), c_int(max_iters), c_double(eps), _ptr(init_vals),
                     c_uint64(len(init_vals)), _dptrs(outs), _ptr(lam), _ptr(secs))
    return outs, lam, secs


def ref_cpstream(batches, stream_mode, rank, max_iters, eps, nonneg, init_vals, bits=64):
    """The reference's CP-stream (ALTO) over the same batches (forgetting 0.99)."""
    L = ref_lib(bits)
    N = len(batches[0]["dims"])
    dims, nnz, cidx, vals = _stream_args(batches)
    init_vals = np.ascontiguousarray(init_vals, dtype=np.float64)
    outs = _stream_outputs(batches, stream_mode, rank)
    lam = np.zeros(rank, np.float64)
    secs = np.zeros(len(batches), np.float64)
    tt = L.ref_cpstream(c_int(N), c_int(stream_mode), c_int(len(batches)), _ptr(dims), _ptr(nnz),
                        _ptr(cidx), _ptr(vals), c_int(rank), c_int(max_iters), c_double(eps),
                        c_int(1 if nonneg else 0), _ptr(init_vals), c_uint64(len(init_vals)),
                        _dptrs(outs), _ptr(lam), _ptr(secs))
    return outs, lam, secs
