"""alto_b200 -- Python host side of the B200 ALTO library.

Mirrors the reference's operator interface for the hot path
(jeewhanchoi/ALTO-stream, include/alto.hpp, include/cpd.hpp,
src/streaming_cpd.cpp) over the C ABI in ``include/alto_b200.h``:

* ``create_alto`` / ``init_salto`` + ``update_salto`` / ``destroy_alto``
  (include/alto.hpp:151-604) -> :class:`AltoTensor`;
* ``mttkrp_alto_par`` (include/alto.hpp:902) -> :func:`mttkrp_alto_par`
  (accumulates into ``factors[target_mode]`` like the reference);
* ``cpd_alto`` (include/cpd.hpp:47) -> :func:`cpd_alto`;
* ``cpstream`` (src/streaming_cpd.cpp:26) -> :class:`CPStream`;
* ``ImportSparseTensor`` / ``ExportSparseTensor`` (src/sptensor.cpp:22-249)
  -> :func:`read_tensor` (parsed on the device) / :func:`write_tensor`;
* ``StreamingSparseTensor`` (include/streaming_sptensor.hpp:10-44) ->
  :class:`Slicer`, whose batches :meth:`CPStream.push_batch` takes as they
  lie in device memory.

The library is the CUDA build ``libalto_b200.so`` next to this file.  There
is no CPU fallback: importing works anywhere, but every call that needs the
library raises :class:`AltoError` when it is missing or no GPU is usable.
Device buffers are torch CUDA tensors (torch is plumbing here: memory and
streams); host buffers are numpy arrays.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, byref, c_char_p, c_double, c_int, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libalto_b200.so")

OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_NOT_SPD, ERR_UNSUPPORTED, ERR_TIMEOUT = range(7)
F32, BF16, F64 = 0, 1, 2
AUTO, ATOMIC, STAGED, STREAM, SORTED, DETERMINISTIC = range(6)
FEED_BULK = 0x100  # OR with ATOMIC / SORTED: line streamed through shared memory by bulk copy
FEED_DENSE = 0x200  # OR with SORTED (3 modes): the walk compiled for five blocks per SM
FEED_FIXED_TARGET = 0x400  # OR with SORTED (3 modes): as FEED_DENSE, compiled once per target mode
UNCONSTRAINED, NONNEG, LASSO = range(3)
CPSTREAM, SPCPSTREAM = range(2)  # streaming models (alto_stream_set_model)
FIT_REFERENCE, FIT_EXACT = 0, 1

EXPORTED = [
    "alto_status_string", "alto_last_error", "alto_version", "alto_kernel_launches",
    "alto_compute_masks", "alto_tensor_create", "alto_tensor_update", "alto_tensor_export", "alto_tensor_info",
    "alto_tensor_device_bytes", "alto_tensor_restrict", "alto_tensor_destroy", "alto_mttkrp", "alto_mttkrp_variant_run",
    "alto_mttkrp_choose", "alto_mttkrp_autotune", "alto_mttkrp_host", "alto_mttkrp_host_changed", "alto_gram",
    "alto_gram_noalloc", "alto_cpd_als", "alto_stream_open",
    "alto_stream_push", "alto_stream_factor", "alto_stream_lambda", "alto_stream_set_model", "alto_stream_set_graph", "alto_stream_stats", "alto_stream_error",
    "alto_stream_close",
    "alto_read_tensor", "alto_dcoo_view", "alto_dcoo_stats", "alto_dcoo_to_host", "alto_dcoo_destroy", "alto_write_tensor",
    "alto_slicer_create", "alto_slicer_next", "alto_slicer_cut_all", "alto_slicer_batch", "alto_slicer_last_batch", "alto_slicer_stream_prev",
    "alto_slicer_iperm", "alto_slicer_tensor", "alto_slicer_destroy",
    "alto_server_create", "alto_server_open", "alto_server_submit", "alto_server_wait", "alto_server_poll",
    "alto_server_drain", "alto_server_stats", "alto_server_factor", "alto_server_close", "alto_server_destroy",
]


class AltoError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"alto status {status}: {msg}")
        self.status = status


class alto_coo(ctypes.Structure):
    _fields_ = [("nmodes", c_int), ("dims", POINTER(c_uint64)), ("nnz", c_uint64),
                ("cidx", POINTER(c_void_p)), ("index_bytes", c_int), ("vals", c_void_p),
                ("val_dtype", c_int), ("on_device", c_int)]


_lib = None


def lib():
    """The loaded CUDA library (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AltoError(ERR_CUDA, f"{LIB_PATH} is not built (run `make -C alto-stream_b200`)")
        L = ctypes.CDLL(LIB_PATH)
        L.alto_status_string.restype = c_char_p
        L.alto_last_error.restype = c_char_p
        L.alto_kernel_launches.restype = c_uint64
        for name in EXPORTED:
            if name not in ("alto_status_string", "alto_last_error", "alto_kernel_launches", "alto_version"):
                getattr(L, name).restype = c_int
        _lib = L
    return _lib


def check(status):
    if status != OK:
        L = lib()
        raise AltoError(status, f"{L.alto_status_string(status).decode()}: {L.alto_last_error().decode()}")


def kernel_launches():
    return int(lib().alto_kernel_launches())


def _stream_handle(stream):
    if stream is None:
        try:
            import torch

            if torch.cuda.is_available():
                return c_void_p(torch.cuda.current_stream().cuda_stream)
        except ImportError:
            pass
        return c_void_p(0)
    if isinstance(stream, int):
        return c_void_p(stream)
    return c_void_p(stream.cuda_stream)


def _is_torch(x):
    return type(x).__module__.startswith("torch")


class _Coo:
    """Holds an alto_coo and keeps its buffers alive."""

    def __init__(self, dims, cidx, vals):
        self.dims = np.ascontiguousarray(dims, dtype=np.uint64)
        N = len(self.dims)
        keep = []
        ptrs = (c_void_p * N)()
        if _is_torch(cidx) or (isinstance(cidx, (list, tuple)) and len(cidx) and _is_torch(cidx[0])):
            cols = [cidx[m] for m in range(N)]
            ib = cols[0].element_size()
            for m, c in enumerate(cols):
                c = c.contiguous()
                keep.append(c)
                ptrs[m] = c.data_ptr()
            on_dev = 1
            nnz = cols[0].numel()
            v = vals.contiguous()
            keep.append(v)
            vptr = v.data_ptr()
            vdt = F64 if v.element_size() == 8 else F32
        else:
            cidx = np.ascontiguousarray(cidx)
            if cidx.dtype not in (np.uint64, np.int64, np.uint32, np.int32):
                cidx = cidx.astype(np.uint64)
            ib = cidx.dtype.itemsize
            nnz = cidx.shape[1] if cidx.ndim == 2 else 0
            for m in range(N):
                row = np.ascontiguousarray(cidx[m])
                keep.append(row)
                ptrs[m] = row.ctypes.data
            v = np.ascontiguousarray(vals)
            if v.dtype not in (np.float64, np.float32):
                v = v.astype(np.float64)
            keep.append(v)
            vptr = v.ctypes.data
            vdt = F64 if v.dtype == np.float64 else F32
            on_dev = 0
        self.keep = keep
        self.ptrs = ptrs
        self.c = alto_coo(N, self.dims.ctypes.data_as(POINTER(c_uint64)), nnz,
                          ctypes.cast(ptrs, POINTER(c_void_p)), ib, c_void_p(vptr), vdt, on_dev)
        self.nnz = nnz


def compute_masks(dims, key_bits=128):
    """setup_packed_alto on the host (no GPU needed): (masks [N, 2], alto_mask [2], bits)."""
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    N = len(dims)
    masks = np.zeros(2 * N, np.uint64)
    am = np.zeros(2, np.uint64)
    bits = c_int()
    check(lib().alto_compute_masks(c_int(N), dims.ctypes.data_as(c_void_p), c_int(key_bits),
                                   masks.ctypes.data_as(c_void_p), am.ctypes.data_as(c_void_p), byref(bits)))
    return masks.reshape(N, 2), am, bits.value


class AltoTensor:
    """A device-resident ALTO tensor (the reference's AltoTensor<LIT>).

    dims: mode lengths; cidx: [nmodes, nnz] 0-based indices (numpy host array
    or torch CUDA tensor); vals: nnz values.  nprtn is the reference's
    partition count (used for exported prtn_ptr / prtn_intervals);
    stream_mode >= 0 marks the streaming mode (init_salto)."""

    def __init__(self, dims, cidx, vals, nprtn=1, stream_mode=-1, key_bits=0, stream=None):
        L = lib()
        coo = _Coo(dims, cidx, vals)
        h = c_void_p()
        check(L.alto_tensor_create(byref(coo.c), c_int(key_bits), c_int(nprtn), c_int(stream_mode),
                                   _stream_handle(stream), byref(h)))
        self.h = h
        self._refresh()

    def _refresh(self):
        L = lib()
        n = c_int()
        dims = (c_uint64 * 8)()
        nnz = c_uint64()
        kb, ab, np_, sm = c_int(), c_int(), c_int(), c_int()
        check(L.alto_tensor_info(self.h, byref(n), dims, byref(nnz), byref(kb), byref(ab), byref(np_), byref(sm)))
        self.nmodes = n.value
        self.dims = np.array(dims[: n.value], np.uint64)
        self.nnz = nnz.value
        self.key_bits = kb.value
        self.alto_bits = ab.value
        self.nprtn = np_.value
        self.stream_mode = sm.value

    def update(self, dims, cidx, vals, nprtn=1, stream=None):
        """update_salto: re-encode a new slice into this tensor."""
        coo = _Coo(dims, cidx, vals)
        check(lib().alto_tensor_update(self.h, byref(coo.c), c_int(nprtn), _stream_handle(stream)))
        self._refresh()

    def export(self):
        N, nnz, P = self.nmodes, self.nnz, self.nprtn
        masks = np.zeros(2 * N, np.uint64)
        am = np.zeros(2, np.uint64)
        idx = np.zeros(2 * max(nnz, 1), np.uint64)
        vals = np.zeros(max(nnz, 1), np.float64)
        perm = np.zeros(max(nnz, 1), np.uint64)
        pp = np.zeros(P + 1, np.uint64)
        iv = np.zeros(2 * P * N, np.uint64)
        p = lambda a: a.ctypes.data_as(c_void_p)
        check(lib().alto_tensor_export(self.h, p(masks), p(am), p(idx), p(vals), p(perm), p(pp), p(iv)))
        return dict(masks=masks.reshape(N, 2), alto_mask=am, idx=idx[: 2 * nnz].reshape(nnz, 2),
                    vals=vals[:nnz], perm=perm[:nnz], prtn_ptr=pp, intervals=iv.reshape(P, N, 2))

    def restrict(self, begin, end, stream=None):
        """Keep line entries [begin, end) of the ALTO order (a shard; alto_tensor_restrict)."""
        check(lib().alto_tensor_restrict(self.h, c_uint64(int(begin)), c_uint64(int(end)), _stream_handle(stream)))
        self._refresh()
        return self

    def device_bytes(self):
        b = c_uint64()
        check(lib().alto_tensor_device_bytes(self.h, byref(b)))
        return b.value

    def mttkrp(self, mode, factors, rank, out=None, accumulate=False, variant=AUTO, stream=None):
        """MTTKRP of `mode` into `out` (float32 torch CUDA tensor, allocated if None)."""
        import torch

        N = self.nmodes
        if out is None:
            ref = next(f for i, f in enumerate(factors) if i != mode)
            out = torch.empty((int(self.dims[mode]), rank), dtype=torch.float32, device=ref.device)
            accumulate = False
        dt = None
        ptrs = (c_void_p * N)()
        for m in range(N):
            if m == mode:
                ptrs[m] = None
                continue
            f = factors[m]
            if not f.is_contiguous():
                raise ValueError("factor matrices must be contiguous")
            fdt = BF16 if f.dtype == torch.bfloat16 else F32
            if f.dtype not in (torch.float32, torch.bfloat16):
                raise ValueError("factors must be float32 or bfloat16")
            if dt is not None and fdt != dt:
                raise ValueError("all factors must share one dtype")
            dt = fdt
            ptrs[m] = f.data_ptr()
        if out.dtype != torch.float32 or not out.is_contiguous():
            raise ValueError("out must be a contiguous float32 tensor")
        check(lib().alto_mttkrp_variant_run(self.h, c_int(mode), ptrs, c_int(dt), c_int(rank),
                                            c_void_p(out.data_ptr()), c_int(1 if accumulate else 0),
                                            c_int(variant), _stream_handle(stream)))
        return out

    def choose_variant(self, mode, rank, fdtype=F32):
        v = c_int()
        check(lib().alto_mttkrp_choose(self.h, c_int(mode), c_int(rank), c_int(fdtype), byref(v)))
        return v.value

    def autotune(self, factors, rank, stream=None):
        """Time the MTTKRP variants per mode and make AUTO use the fastest.
        Returns the chosen variant per mode."""
        import torch

        N = self.nmodes
        ptrs = (c_void_p * N)(*[f.data_ptr() for f in factors])
        dt = BF16 if factors[0].dtype == torch.bfloat16 else F32
        out = (c_int * N)()
        check(lib().alto_mttkrp_autotune(self.h, ptrs, c_int(dt), c_int(rank), _stream_handle(stream), out))
        return list(out)

    def mttkrp_host(self, mode, factors, rank, stream=None, changed=None):
        """The reference calling convention on host float64 arrays:
        factors[mode] is accumulated into, in place.  changed: the modes
        whose arrays the caller modified since this thread's previous
        host-buffer MTTKRP (alto_mttkrp_host_changed; the others are not
        copied again), or None to copy every factor."""
        arrs = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
        for a, f in zip(arrs, factors):
            if a is not f:
                raise ValueError("host factors must be C-contiguous float64 arrays")
        ptrs = (POINTER(c_double) * self.nmodes)(*[a.ctypes.data_as(POINTER(c_double)) for a in arrs])
        if changed is None:
            check(lib().alto_mttkrp_host(self.h, c_int(mode), ptrs, c_int(rank), _stream_handle(stream)))
        else:
            mask = 0
            for m in changed:
                mask |= 1 << int(m)
            check(lib().alto_mttkrp_host_changed(self.h, c_int(mode), ptrs, c_int(rank), c_uint32(mask),
                                                 _stream_handle(stream)))
        return factors

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().alto_tensor_destroy(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gram(U, out=None, stream=None):
    """update_gram: G = U^T U (float64, full symmetric) of a float32 CUDA tensor."""
    import torch

    if U.dtype != torch.float32 or not U.is_contiguous() or U.dim() != 2:
        raise ValueError("U must be a contiguous 2-D float32 tensor")
    rows, rank = U.shape
    if out is None:
        out = torch.empty((rank, rank), dtype=torch.float64, device=U.device)
    check(lib().alto_gram(c_void_p(U.data_ptr()), c_uint64(rows), c_int(rank), c_void_p(out.data_ptr()),
                          _stream_handle(stream)))
    return out


# ------------------------------------------------- reference-named mirrors

def create_alto(dims, cidx, vals, nprtn=1, key_bits=0, stream=None):
    """create_alto (include/alto.hpp:436): build the ALTO tensor."""
    return AltoTensor(dims, cidx, vals, nprtn=nprtn, stream_mode=-1, key_bits=key_bits, stream=stream)


def init_salto(dims, cidx, vals, max_nprtn, stream_mode, key_bits=0, stream=None):
    """init_salto + the first update_salto (include/alto.hpp:151-299)."""
    return AltoTensor(dims, cidx, vals, nprtn=max_nprtn, stream_mode=stream_mode, key_bits=key_bits,
                      stream=stream)


def update_salto(dims, cidx, vals, at, nprtn=1, stream=None):
    at.update(dims, cidx, vals, nprtn=nprtn, stream=stream)
    return at


def destroy_alto(at):
    at.close()


def mttkrp_alto_par(target_mode, factors, rank, at, stream=None):
    """mttkrp_alto_par (include/alto.hpp:902): accumulates the MTTKRP of
    target_mode into factors[target_mode] (torch float32 CUDA tensors)."""
    at.mttkrp(target_mode, factors, rank, out=factors[target_mode], accumulate=True, stream=stream)
    return factors[target_mode]


def cpd_alto(at, U, lam, rank, max_iters, epsilon, fit_mode=FIT_REFERENCE, storage=F32, stream=None):
    """cpd_alto (include/cpd.hpp:47): CP-ALS on the device.

    U: list of host float64 arrays (dims[n] x rank), lam: host float64
    (rank); both hold the initial model and are returned updated (copies).
    Returns (U, lam, fits, iterations)."""
    Us = [np.array(u, dtype=np.float64, copy=True, order="C") for u in U]
    lam = np.array(lam, dtype=np.float64, copy=True)
    fits = np.zeros(max(max_iters, 1), np.float64)
    it = c_int()
    ptrs = (POINTER(c_double) * len(Us))(*[u.ctypes.data_as(POINTER(c_double)) for u in Us])
    check(lib().alto_cpd_als(at.h, c_int(rank), ptrs, lam.ctypes.data_as(POINTER(c_double)),
                             c_int(max_iters), c_double(epsilon), c_int(fit_mode), c_int(storage),
                             fits.ctypes.data_as(POINTER(c_double)), byref(it), _stream_handle(stream)))
    return Us, lam, fits[: it.value], it.value


class CPStream:
    """A CP-stream session (cpstream, src/streaming_cpd.cpp:26) whose model,
    Grams and ADMM state stay on the device between time batches."""

    def __init__(self, nmodes, stream_mode, rank, constraint=UNCONSTRAINED, forgetting=0.99,
                 max_inner=10, epsilon=1e-5, stream=None):
        h = c_void_p()
        check(lib().alto_stream_open(c_int(nmodes), c_int(stream_mode), c_int(rank), c_int(constraint),
                                     c_double(forgetting), c_int(max_inner), c_double(epsilon),
                                     _stream_handle(stream), byref(h)))
        self.h = h
        self.nmodes = nmodes
        self.stream_mode = stream_mode
        self.rank = rank

    def push(self, dims, cidx, vals, init_vals=None):
        """Process one time batch; init_vals feeds the rows the model gains."""
        coo = _Coo(dims, cidx, vals)
        iv = np.ascontiguousarray(init_vals if init_vals is not None else np.zeros(0), dtype=np.float64)
        inner = c_int()
        check(lib().alto_stream_push(self.h, byref(coo.c), iv.ctypes.data_as(c_void_p), c_uint64(len(iv)),
                                     byref(inner)))
        return inner.value

    def push_batch(self, batch, init_vals=None):
        """Process one :class:`SliceBatch` (device memory, no copy)."""
        iv = np.ascontiguousarray(init_vals if init_vals is not None else np.zeros(0), dtype=np.float64)
        inner = c_int()
        check(lib().alto_stream_push(self.h, byref(batch.coo), iv.ctypes.data_as(c_void_p), c_uint64(len(iv)),
                                     byref(inner)))
        return inner.value

    def factor(self, mode, max_rows):
        out = np.zeros((max(max_rows, 1), self.rank), np.float64)
        rows = c_uint64()
        check(lib().alto_stream_factor(self.h, c_int(mode), out.ctypes.data_as(c_void_p), byref(rows)))
        return out[: rows.value]

    def set_model(self, model):
        """CPSTREAM (default) or SPCPSTREAM, before the first push (alto_stream_set_model)."""
        check(lib().alto_stream_set_model(self.h, c_int(model)))

    def set_graph(self, enable):
        """A batch's inner iterations as one launch of the session's CUDA
        graph (default) or launched one by one (alto_stream_set_graph)."""
        check(lib().alto_stream_set_graph(self.h, c_int(1 if enable else 0)))

    def stats(self):
        """Where the pushes spent their time (alto_stream_stats), summed:
        host ms preparing, from the inner iterations' launch to their
        outcome, and finishing; device ms of the inner iterations."""
        out = (c_double * 9)()
        check(lib().alto_stream_stats(self.h, out))
        return {"pushes": int(out[0]), "prepare_ms": out[1], "inner_ms": out[2], "inner_device_ms": out[3],
                "finish_ms": out[4], "inner_iters": int(out[5]), "grow_ms": out[6], "encode_ms": out[7],
                "sorted_copies_ms": out[8]}

    def error(self, X):
        """cpd_error of the current model against X: a :class:`SliceBatch`
        (e.g. :meth:`Slicer.tensor` or :meth:`Slicer.stream_prev`) or a
        (dims, cidx, vals) tuple in the session's indexing."""
        coo = X if isinstance(X, SliceBatch) else _Coo(*X)
        err = c_double()
        check(lib().alto_stream_error(self.h, byref(coo.coo if isinstance(X, SliceBatch) else coo.c), byref(err)))
        return err.value

    def lam(self):
        out = np.zeros(self.rank, np.float64)
        check(lib().alto_stream_lambda(self.h, out.ctypes.data_as(c_void_p)))
        return out

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().alto_stream_close(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------- tensor files

TEXT, BINARY = 0, 1  # the reference's FileFormat


class DeviceCoo:
    """A tensor read from a file into device memory (alto_read_tensor):
    uint64 indices and float64 values, the reference's IType and FType."""

    def __init__(self, path, binary=False, zero_based=False, stream=None):
        h = c_void_p()
        check(lib().alto_read_tensor(str(path).encode(), c_int(BINARY if binary else TEXT),
                                     c_int(1 if zero_based else 0), _stream_handle(stream), byref(h)))
        self.h = h
        self.coo = alto_coo()
        check(lib().alto_dcoo_view(self.h, byref(self.coo)))
        self.nmodes = int(self.coo.nmodes)
        self.nnz = int(self.coo.nnz)
        self.dims = np.array([self.coo.dims[m] for m in range(self.nmodes)], np.uint64)

    def tensors(self):
        """(list of int64 index tensors, float64 value tensor): torch views."""
        import torch

        idx = [torch.as_tensor(_DeviceArray(self.coo.cidx[m], self.nnz, "<i8"), device="cuda")
               for m in range(self.nmodes)]
        return idx, torch.as_tensor(_DeviceArray(self.coo.vals, self.nnz, "<f8"), device="cuda")

    def to_host(self):
        """(cidx uint64 [nmodes, nnz], vals float64) as numpy arrays (alto_dcoo_to_host)."""
        c = np.zeros((self.nmodes, self.nnz), np.uint64)
        v = np.zeros(self.nnz)
        check(lib().alto_dcoo_to_host(self.h, c.ctypes.data_as(c_void_p), v.ctypes.data_as(c_void_p)))
        return c, v

    def stats(self):
        r, p, fb, hv = c_double(), c_double(), c_uint64(), c_uint64()
        check(lib().alto_dcoo_stats(self.h, byref(r), byref(p), byref(fb), byref(hv)))
        return {"read_ms": r.value, "parse_ms": p.value, "file_bytes": fb.value, "host_values": hv.value}

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().alto_dcoo_destroy(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_tensor(path, binary=False, zero_based=False, stream=None):
    """ImportSparseTensor into device memory: a :class:`DeviceCoo`."""
    return DeviceCoo(path, binary, zero_based, stream)


def write_tensor(path, dims, cidx, vals, binary=False):
    """ExportSparseTensor of a host (numpy) or device (torch) COO tensor."""
    coo = _Coo(dims, cidx, vals)
    check(lib().alto_write_tensor(str(path).encode(), c_int(BINARY if binary else TEXT), byref(coo.c)))


# ------------------------------------------------------------ stream slicer

class _DeviceArray:
    """A device pointer described for torch.as_tensor (no copy)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class SliceBatch:
    """One batch of a :class:`Slicer`: dims (host), nnz and an alto_coo of
    device views into the slicer's arrays, valid while the slicer lives (the
    host-side dims and pointers are copied here)."""

    def __init__(self, coo, nmodes):
        self.nmodes = nmodes
        self.nnz = int(coo.nnz)
        self.dims = np.array([coo.dims[m] for m in range(nmodes)], np.uint64)
        self._ptrs = (c_void_p * nmodes)(*[coo.cidx[m] for m in range(nmodes)])
        self.coo = alto_coo(coo.nmodes, self.dims.ctypes.data_as(POINTER(c_uint64)), coo.nnz,
                            ctypes.cast(self._ptrs, POINTER(c_void_p)), coo.index_bytes, coo.vals, coo.val_dtype,
                            coo.on_device)

    def tensors(self):
        """(list of uint32 index tensors, value tensor): torch views of the batch."""
        import torch

        if self.nnz == 0:
            return ([torch.zeros(0, dtype=torch.int32, device="cuda") for _ in range(self.nmodes)],
                    torch.zeros(0, dtype=torch.float64, device="cuda"))
        idx = [torch.as_tensor(_DeviceArray(self.coo.cidx[m], self.nnz, "<i4"), device="cuda")
               for m in range(self.nmodes)]
        vt = "<f8" if self.coo.val_dtype == F64 else "<f4"
        return idx, torch.as_tensor(_DeviceArray(self.coo.vals, self.nnz, vt), device="cuda")

    def to_host(self):
        """(cidx uint64 [nmodes, nnz], vals) as numpy arrays."""
        import torch

        torch.cuda.synchronize()
        idx, v = self.tensors()
        c = np.zeros((self.nmodes, self.nnz), np.uint64)
        for m in range(self.nmodes):
            c[m] = idx[m].cpu().numpy().view(np.uint32)
        return c, v.cpu().numpy()


class Slicer:
    """The reference's StreamingSparseTensor on the device (alto_slicer_*):
    the whole tensor sorted by the stream mode and relabelled once, then cut
    into batches of whole time steps with :meth:`next`."""

    def __init__(self, dims, cidx, vals, stream_mode, stream=None):
        self.coo_in = _Coo(dims, cidx, vals)
        self.nmodes = len(self.coo_in.dims)
        self.stream_mode = stream_mode
        h = c_void_p()
        check(lib().alto_slicer_create(byref(self.coo_in.c), c_int(stream_mode), _stream_handle(stream), byref(h)))
        self.h = h
        self.coo_in = None  # the slicer keeps its own copy

    def next(self, nnz_threshold=1, timeslice_limit=1):
        """next_dynamic_batch: a :class:`SliceBatch`, or None at the end."""
        c = alto_coo()
        got = c_int()
        check(lib().alto_slicer_next(self.h, c_uint64(nnz_threshold), c_uint64(timeslice_limit), byref(c),
                                     byref(got)))
        return SliceBatch(c, self.nmodes) if got.value else None

    def cut_all(self, nnz_threshold=1, timeslice_limit=1):
        """Every remaining batch at once (alto_slicer_cut_all); returns the
        count, and :meth:`batch` gives each one."""
        n = c_uint64()
        check(lib().alto_slicer_cut_all(self.h, c_uint64(nnz_threshold), c_uint64(timeslice_limit), byref(n)))
        return n.value

    def batch(self, b):
        """Batch b of the last :meth:`cut_all`."""
        c = alto_coo()
        check(lib().alto_slicer_batch(self.h, c_uint64(b), byref(c)))
        return SliceBatch(c, self.nmodes)

    def last_batch(self):
        last = c_int()
        check(lib().alto_slicer_last_batch(self.h, byref(last)))
        return bool(last.value)

    def stream_prev(self, previous):
        """The nonzeros of the last `previous` time steps returned (or None)."""
        c = alto_coo()
        got = c_int()
        check(lib().alto_slicer_stream_prev(self.h, c_uint64(previous), byref(c), byref(got)))
        return SliceBatch(c, self.nmodes) if got.value else None

    def tensor(self):
        """The whole sorted, relabelled tensor with global time indices."""
        c = alto_coo()
        check(lib().alto_slicer_tensor(self.h, byref(c)))
        return SliceBatch(c, self.nmodes)

    def iperm(self, mode):
        """Original index of every label of `mode` (numpy uint64)."""
        n = c_uint64()
        check(lib().alto_slicer_iperm(self.h, c_int(mode), None, byref(n)))
        out = np.zeros(max(n.value, 1), np.uint64)
        check(lib().alto_slicer_iperm(self.h, c_int(mode), out.ctypes.data_as(c_void_p), byref(n)))
        return out[: n.value]

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().alto_slicer_destroy(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ serving

class alto_stream_config(ctypes.Structure):
    _fields_ = [("nmodes", c_int), ("stream_mode", c_int), ("rank", c_int), ("constraint", c_int),
                ("forgetting", c_double), ("max_inner_iters", c_int), ("epsilon", c_double), ("model", c_int)]


class alto_serving_stats(ctypes.Structure):
    _fields_ = [("submitted", c_uint64), ("completed", c_uint64), ("p50_ms", c_double), ("p99_ms", c_double),
                ("max_ms", c_double), ("slices_per_s", c_double), ("reserved_bytes", c_uint64),
                ("admitted_streams", c_int), ("pending_streams", c_int), ("prepare_ms", c_double),
                ("step_ms", c_double), ("finish_ms", c_double), ("steps", c_uint64), ("step_slices", c_uint64)]


class Server:
    """Many CP-stream tensors served concurrently (alto_server_*): slices are
    queued per stream and processed by `workers` threads on their own CUDA
    streams; streams are admitted under an HBM budget."""

    def __init__(self, hbm_budget_bytes, workers=8):
        h = c_void_p()
        check(lib().alto_server_create(c_uint64(int(hbm_budget_bytes)), c_int(workers), byref(h)))
        self.h = h
        self.rank = {}

    def open(self, nmodes, stream_mode, rank, max_dims, max_slice_nnz, constraint=UNCONSTRAINED,
             forgetting=0.99, max_inner=10, epsilon=1e-5, model=0):
        cfg = alto_stream_config(nmodes, stream_mode, rank, constraint, forgetting, max_inner, epsilon, model)
        md = np.ascontiguousarray(max_dims, dtype=np.uint64)
        sid = c_int()
        check(lib().alto_server_open(self.h, byref(cfg), md.ctypes.data_as(c_void_p), c_uint64(int(max_slice_nnz)),
                                     byref(sid)))
        self.rank[sid.value] = rank
        return sid.value

    def submit(self, sid, dims, cidx, vals, init_vals=None):
        coo = _Coo(dims, cidx, vals)
        iv = np.ascontiguousarray(init_vals if init_vals is not None else np.zeros(0), dtype=np.float64)
        t = c_uint64()
        check(lib().alto_server_submit(self.h, c_int(sid), byref(coo.c), iv.ctypes.data_as(c_void_p),
                                       c_uint64(len(iv)), byref(t)))
        return t.value

    def wait(self, ticket):
        inner, lat = c_int(), c_double()
        check(lib().alto_server_wait(self.h, c_uint64(ticket), byref(inner), byref(lat)))
        return inner.value, lat.value

    def poll(self, ticket):
        """None while the slice is queued or running, else (inner iterations, latency ms)."""
        done, inner, lat = c_int(), c_int(), c_double()
        check(lib().alto_server_poll(self.h, c_uint64(ticket), byref(done), byref(inner), byref(lat)))
        return (inner.value, lat.value) if done.value else None

    def drain(self):
        check(lib().alto_server_drain(self.h))

    def stats(self):
        st = alto_serving_stats()
        check(lib().alto_server_stats(self.h, byref(st)))
        return {f: getattr(st, f) for f, _ in alto_serving_stats._fields_}

    def factor(self, sid, mode):
        rows = c_uint64()
        check(lib().alto_server_factor(self.h, c_int(sid), c_int(mode), None, byref(rows)))
        out = np.zeros((max(rows.value, 1), self.rank[sid]), np.float64)
        check(lib().alto_server_factor(self.h, c_int(sid), c_int(mode), out.ctypes.data_as(c_void_p), byref(rows)))
        return out[: rows.value]

    def close(self, sid):
        check(lib().alto_server_close(self.h, c_int(sid)))

    def destroy(self):
        if getattr(self, "h", None) and self.h.value:
            lib().alto_server_destroy(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
