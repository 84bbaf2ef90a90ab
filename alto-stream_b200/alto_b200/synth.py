"""Seeded synthetic sparse tensors with the shapes and value distributions of
the workloads this library is measured on.

No public dataset is used: every tensor is generated from a seed.  All
generators return unique coordinates (the ALTO sort order is only a total
order for unique coordinates), drawn with oversampling, de-duplicated,
shuffled and truncated.

Host generators (numpy) serve tests and CPU-side references; the device
generator ``zipf_coo_device`` produces the 140M-nonzero power-law tensor
directly in HBM with torch's CUDA generator.
"""
from __future__ import annotations

import math

import numpy as np


def _dedup_shuffle(cidx, rng, nnz):
    """Drop repeated coordinates, shuffle, keep the first nnz."""
    N, n = cidx.shape
    # lexicographic unique over the columns
    order = np.lexsort(cidx[::-1])
    s = cidx[:, order]
    keep = np.ones(n, bool)
    keep[1:] = np.any(s[:, 1:] != s[:, :-1], axis=0)
    s = s[:, keep]
    perm = rng.permutation(s.shape[1])
    return np.ascontiguousarray(s[:, perm[:nnz]])


def uniform_coo(dims, nnz, seed=0, values="uniform"):
    """Coordinates i.i.d. uniform per mode, duplicates removed; values U(0,1)."""
    rng = np.random.default_rng(seed)
    dims = [int(d) for d in dims]
    space = math.prod(dims)
    nnz = int(min(nnz, space))
    draw = int(nnz * 1.3) + 64
    while True:
        cidx = np.stack([rng.integers(0, d, draw, dtype=np.uint64) for d in dims])
        cidx = _dedup_shuffle(cidx, rng, nnz)
        if cidx.shape[1] >= nnz or draw > 8 * nnz + 1024:
            break
        draw *= 2
    vals = _values(rng, cidx.shape[1], values)
    return cidx, vals


class ZipfSampler:
    """Draws from a Zipf(s) law truncated to ranks 1..dim, as 0-based indices
    whose labels are randomly permuted once (so hot rows are scattered, and
    stay the same rows across calls)."""

    def __init__(self, rng, dim, s, permute=True):
        ranks = np.arange(1, dim + 1, dtype=np.float64)
        cdf = np.cumsum(ranks ** (-float(s)))
        self.cdf = cdf / cdf[-1]
        self.dim = dim
        self.labels = rng.permutation(dim).astype(np.uint64) if permute else None

    def sample(self, rng, n):
        r = np.searchsorted(self.cdf, rng.random(n), side="right").astype(np.uint64)
        r = np.minimum(r, self.dim - 1)
        return self.labels[r] if self.labels is not None else r


def zipf_indices(rng, dim, s, n, permute=True):
    """n draws from a Zipf(s) law truncated to ranks 1..dim (one label
    permutation per call; use ZipfSampler to keep labels across calls)."""
    return ZipfSampler(rng, dim, s, permute).sample(rng, n)


def _values(rng, n, kind):
    if kind == "uniform":
        return rng.random(n)
    if kind == "lognormal":
        return rng.lognormal(0.0, 1.0, n)
    if kind == "poisson3":
        v = rng.poisson(3.0, n).astype(np.float64)
        return v
    raise ValueError(kind)


def powerlaw_coo(dims, nnz, exponents, seed=0, values="uniform"):
    """Per-mode Zipf coordinates (exponent None = uniform), unique, with the
    given value distribution ("uniform", "lognormal", "poisson3")."""
    rng = np.random.default_rng(seed)
    dims = [int(d) for d in dims]
    nnz = int(nnz)
    draw = int(nnz * 1.5) + 64
    for _ in range(8):
        cols = []
        for d, s in zip(dims, exponents):
            if s is None:
                cols.append(rng.integers(0, d, draw, dtype=np.uint64))
            else:
                cols.append(zipf_indices(rng, d, s, draw))
        cidx = _dedup_shuffle(np.stack(cols), rng, nnz)
        if cidx.shape[1] >= nnz:
            break
        draw *= 2
    vals = _values(rng, cidx.shape[1], values)
    if values == "poisson3":  # zero draws are not stored as nonzeros
        keep = vals != 0
        cidx, vals = np.ascontiguousarray(cidx[:, keep]), vals[keep]
    return cidx, vals


def stream_batches(space_dims, nslices, nnz_fn, exponents, seed=0, values="poisson3",
                   time_mode=0, relabel=True):
    """A CP-stream input: nslices batches of one time step each.

    Every batch is {dims, cidx, vals} as the reference's
    StreamingSparseTensor.next_dynamic_batch hands it over
    (src/streaming_sptensor.cpp:69-264): the batch's nonzeros are in the
    slicer's sorted order (lexicographic over the modes that follow the time
    mode), the time mode has extent 1 and index 0, the other modes carry
    first-seen relabelled indices (first seen in that order, over the whole
    stream) and their extents grow monotonically (max index + 1, never
    shrinking).  nnz_fn(rng, s) gives the number of coordinate draws for
    slice s; zero values are dropped.
    """
    rng = np.random.default_rng(seed)
    nsp = len(space_dims)
    nmodes = nsp + 1
    samplers = [ZipfSampler(rng, int(d), e) if e is not None else None for d, e in zip(space_dims, exponents)]
    maps = [np.full(int(d), -1, np.int64) for d in space_dims]
    nxt = [0] * nsp
    prev = [0] * nmodes
    batches = []
    for s in range(nslices):
        n = int(nnz_fn(rng, s))
        cols = []
        for d, zs in zip(space_dims, samplers):
            cols.append(zs.sample(rng, n) if zs is not None else rng.integers(0, int(d), n, dtype=np.uint64))
        c = _dedup_shuffle(np.stack(cols), rng, n)
        v = _values(rng, c.shape[1], values)
        keep = v != 0
        c, v = c[:, keep], v[keep]
        order = np.lexsort(c[::-1])  # sorted by (mode 1, mode 2, ...) as the slicer's tt_sort
        c, v = np.ascontiguousarray(c[:, order]), v[order]
        if relabel:
            for m in range(nsp):
                col = c[m].astype(np.int64)
                mp = maps[m]
                unseen = mp[col] < 0
                if unseen.any():
                    u, first = np.unique(col[unseen], return_index=True)
                    newv = u[np.argsort(first)]
                    mp[newv] = np.arange(nxt[m], nxt[m] + len(newv))
                    nxt[m] += len(newv)
                c[m] = mp[col].astype(np.uint64)
        full = np.zeros((nmodes, c.shape[1]), np.uint64)
        dims = [0] * nmodes
        k = 0
        for m in range(nmodes):
            if m == time_mode:
                dims[m] = 1
            else:
                full[m] = c[k]
                dims[m] = max(int(c[k].max()) + 1 if c.shape[1] else 0, prev[m])
                k += 1
        prev = dims
        batches.append(dict(dims=np.array(dims, np.uint64), cidx=np.ascontiguousarray(full), vals=v))
    return batches


def init_values(n, seed=0):
    """Initial model values in [-3, 3] with random sign, the range of the
    reference's rand_val (src/util.cpp:28-35); drawn from numpy, not rand()."""
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 3.0, n) * np.where(rng.random(n) < 0.5, -1.0, 1.0)


def zipf_coo_device(dims, nnz, exponents, seed=0, values="lognormal", device="cuda"):
    """Power-law COO generated on the device (torch), unique coordinates.

    Returns (cidx int64 [N, nnz], vals float32 [nnz]) on `device`: draws
    repeat until nnz distinct coordinates exist (at most 64 rounds, else
    fewer are returned), then a random subset of nnz is kept in random order."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    cdfs, labels = [], []
    for d, s in zip(dims, exponents):
        d = int(d)
        if s is None:
            cdfs.append(None)
            labels.append(None)
            continue
        ranks = torch.arange(1, d + 1, device=device, dtype=torch.float64)
        cdf = torch.cumsum(ranks.pow(-float(s)), 0)
        cdf /= cdf[-1].clone()
        cdfs.append(cdf)
        labels.append(torch.randperm(d, generator=g, device=device))
        del ranks

    def draw_cols(n):
        cols = []
        for d, cdf, lab in zip(dims, cdfs, labels):
            if cdf is None:
                cols.append(torch.randint(0, int(d), (n,), generator=g, device=device, dtype=torch.int64))
            else:
                u = torch.rand(n, generator=g, device=device, dtype=torch.float64)
                r = torch.searchsorted(cdf, u, right=True).clamp_(max=int(d) - 1)
                del u
                cols.append(lab[r])
                del r
        return cols

    # De-duplicate on a packed key.  When the index bits exceed 63, the lowest
    # `excess` bits of mode 0 select a group and are left out of the key, so
    # each group is de-duplicated on its own 63-bit key.  Power laws collide
    # often, so draws repeat (in batches) until enough distinct coordinates
    # exist.
    bits = [max(1, int(d - 1).bit_length()) for d in dims]
    excess = max(0, sum(bits) - 63)
    gmask = (1 << excess) - 1
    uniq = [torch.empty(0, dtype=torch.int64, device=device) for _ in range(1 << excess)]
    total = 0
    batch = int(nnz * 1.1) + 1024
    for _round in range(64):
        cols = draw_cols(batch)
        for grp in range(1 << excess):
            sel = ((cols[0] & gmask) == grp) if excess else None
            key = None
            sh = 0
            for mi, (c, b) in enumerate(zip(cols, bits)):
                cc = c if sel is None else c[sel]
                if mi == 0 and excess:
                    cc = cc >> excess
                    b -= excess
                key = cc << sh if key is None else key | (cc << sh)
                sh += b
            uniq[grp] = torch.unique(torch.cat([uniq[grp], key]))
            del key, sel
        del cols
        prev, total = total, sum(int(u.numel()) for u in uniq)
        if total >= nnz:
            break
        gained = max(total - prev, 1)
        batch = int(min(max((nnz - total) * batch / gained * 1.1, 1 << 20), 4 * nnz))
    keys = list(enumerate(uniq))
    del cdfs, labels, uniq
    out = [[] for _ in dims]
    for grp, key in keys:
        sh = 0
        for mi, b in enumerate(bits):
            bb = b - excess if (mi == 0 and excess) else b
            v = (key >> sh) & ((1 << bb) - 1)
            if mi == 0 and excess:
                v = (v << excess) | grp
            out[mi].append(v)
            sh += bb
    del keys
    cidx = torch.stack([torch.cat(o) for o in out])
    del out
    perm = torch.randperm(cidx.shape[1], generator=g, device=device)[:nnz]
    cidx = cidx[:, perm].contiguous()
    del perm
    n = cidx.shape[1]
    if values == "lognormal":
        v = torch.randn(n, generator=g, device=device, dtype=torch.float32).exp_()
    else:
        v = torch.rand(n, generator=g, device=device, dtype=torch.float32)
    return cidx, v


def serving_streams(nstreams, slices_per_stream, seed=0, dim_range=(1e3, 1e6), nnz_range=(1e4, 1e6),
                    nnz_median=5e4, ranks=(8, 16, 32)):
    """Independent CP-stream tensors for the serving workload.

    Per stream: three spatial modes with lengths log-uniform in dim_range, a
    rank drawn from `ranks`, a constraint (0 unconstrained, 1 non-negative)
    drawn with equal odds, and slices_per_stream slices of one time step each
    whose nonzero counts are log-normal (median nnz_median, sigma 1) clipped
    to nnz_range; coordinates are uniform over the stream's dims (unique),
    values uniform(0, 1).  Every slice carries the stream's full dims (the
    time mode has extent 1), so the model takes its final size with the
    first slice.  Returns a list of dicts {dims, rank, constraint, slices}."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log10(dim_range[0]), np.log10(dim_range[1])
    out = []
    for k in range(nstreams):
        d = [int(round(10 ** rng.uniform(lo, hi))) for _ in range(3)]
        rank = int(rng.choice(ranks))
        con = int(rng.integers(0, 2))
        bits = [max(1, (x - 1).bit_length()) for x in d]
        slices = []
        for _ in range(slices_per_stream):
            n = int(np.clip(rng.lognormal(np.log(nnz_median), 1.0), nnz_range[0], nnz_range[1]))
            draw = int(n * 1.05) + 64
            cols = [rng.integers(0, x, draw, dtype=np.uint64) for x in d]
            key = cols[0] | (cols[1] << np.uint64(bits[0])) | (cols[2] << np.uint64(bits[0] + bits[1]))
            _, first = np.unique(key, return_index=True)
            keep = np.sort(first)[:n]
            cidx = np.zeros((4, len(keep)), np.uint64)
            for m in range(3):
                cidx[m + 1] = cols[m][keep]
            slices.append(dict(dims=np.array([1] + d, np.uint64), cidx=cidx, vals=rng.random(len(keep))))
        out.append(dict(dims=[1] + d, rank=rank, constraint=con, slices=slices))
    return out
