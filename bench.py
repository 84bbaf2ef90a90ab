#!/usr/bin/env python
"""All-mode ALTO MTTKRP throughput on one or more B200s.

Workload: the 3-mode power-law tensor with dims 4,800,000 x 1,800,000 x
1,800,000 (65 index bits, so 128-bit ALTO keys) and 140,000,000 distinct
nonzeros: per-mode Zipf(1.2) coordinates with randomly permuted labels,
log-normal(0, 1) values, generated on the device from a seed.  One step is
the MTTKRP of every mode at rank 32 with float32 factors and float32
accumulation.  Metric: nonzeros x rank processed per second (nnz*R/s) over
the whole job.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): the one tensor is sharded by output
rows -- per mode, contiguous row blocks of equal nonzero count, each rank
encoding only its block's nonzeros -- and after each mode's MTTKRP the ranks'
row blocks are all-gathered (NCCL broadcasts); strong scaling, the whole
job's nnz*R over the slowest rank's time.  --independent gives every rank a
tensor of its own instead (weak scaling, no collective).

The JSON line carries: value (device-timed, inputs resident in HBM; the
tensor is larger than L2, so no flush is needed), e2e (the same metric
through the host-buffer C-ABI entry point alto_mttkrp_host, float64 host
factors in pinned memory, copies inside the timed region), roofline of the
MTTKRP kernel (algorithmic bytes / CUDA-event time vs the measured HBM copy
bandwidth), cpu_baseline (the reference implementation, compiled from its
sources into oracle/_ref, timed on this host's cores on a bounded sample of
the same distribution), clocks sampled during the timed region, and the
number of this library's kernel launches in the timed region.

`--impl reference` times the reference's own OpenMP MTTKRP (oracle/_ref) on
the host cores instead, on the bounded sample, and prints the same line
with "impl": "reference".

Two more workloads print their own line:

  --workload cpstream   CP-stream over a 4-mode stream: 200 time slices of
                        100,000 x 100,000 x 10,000, per-slice nonzero draws
                        log-normal (median 2e5, sigma 1) clipped to
                        [5e4, 2e6], Zipf(1.1) coordinates, Poisson(3) values
                        (zero draws dropped), rank 16, non-negative ADMM,
                        forgetting 0.95, at most 50 inner iterations, epsilon
                        1e-5.  A step is one slice update through the session
                        API (host COO in); metric slices/s, with p50/p99
                        slice latency.
  --workload serve      64 independent streams (spatial dims log-uniform in
                        [1e3, 1e6], rank 8/16/32, non-negative or
                        unconstrained), slices of log-normal size in
                        [1e4, 1e6] arriving as a Poisson process at 2,000
                        slices/s, served under an 80 GB HBM budget; metric
                        slices/s with p50/p99 latency, against the plain path
                        (one slice at a time, each stream's session in turn).
                        Under torchrun the streams are sharded round robin
                        over the GPUs, one server each, with no collective
                        on the data path (strong scaling: 64 streams in all).
  --workload slice      the stream slicer (StreamingSparseTensor) over the
                        CP-stream workload's shape as one 4-mode tensor:
                        200 time steps with log-normal nonzero counts
                        (median 2e5, sigma 1, clipped to [5e4, 2e6]),
                        100,000 x 100,000 x 10,000 Zipf(1.1) coordinates,
                        int64 indices and float64 values in HBM.  A step is
                        the sort, the first-seen relabel and all 200
                        single-step batches (alto_slicer_cut_all: the cuts
                        of repeated next_dynamic_batch calls, one kernel for
                        the batch-local times); metric nonzeros/s.
  --workload tns        reading the MTTKRP workload's tensor (140M nonzeros,
                        3 modes) from a .tns text file (written once with
                        the library's writer, "%g" values) into device
                        memory; metric nonzeros/s: `value` the device parse
                        with the file's bytes in HBM, `e2e` the whole
                        alto_read_tensor call from a file in the page cache.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "alto-stream_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

DIMS = [4800000, 1800000, 1800000]
NNZ = 140_000_000
ZIPF = [1.2, 1.2, 1.2]
RANK = 32
# bounded CPU sample: 24M nonzeros keep nnz/dims above 4 in every mode (5,
# 13, 13), so the reference runs the same variant (da_mem_pull,
# include/alto.hpp:1544-1634) as on the whole tensor
CPU_SAMPLE_NNZ = 24_000_000
METRIC = "MTTKRP nnz*R/s (all-mode, rank 32)"
WORKLOAD = "powerlaw3d-4.8Mx1.8Mx1.8M-140Mnnz-zipf1.2-R32-allmode"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--workload", choices=["mttkrp", "cpstream", "serve", "slice", "tns", "cpals3d", "cpals5d"],
                    default="mttkrp")
    ap.add_argument("--no-configs", action="store_true",
                    help="mttkrp: leave out the other configurations' sub-objects of the default line")
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (mttkrp: all-mode MTTKRPs, default 10; cpstream: slices, default 197; "
                         "serve: slices per stream, default 7)")
    ap.add_argument("--warmup", type=int, default=None,
                    help="untimed steps before (mttkrp 3; cpstream 3 slices; serve 1 slice per stream)")
    ap.add_argument("--workers", type=int, default=16, help="serve: server worker threads")
    ap.add_argument("--kernel-share", action="store_true",
                    help="cpstream/serve: also record every device activity of the timed region with the CUDA "
                         "profiling interface (torch.profiler) and report kernel time against wall time; the "
                         "line's throughput is then taken under the profiler and is not a bench number")
    ap.add_argument("--no-graph", action="store_true",
                    help="cpstream: launch every inner iteration directly (no CUDA graph; for per-kernel profiles)")
    ap.add_argument("--model", choices=["cpstream", "spcpstream"], default="cpstream",
                    help="cpstream/serve: the streaming model (spcpstream: row-sparse updates, no constraint)")
    ap.add_argument("--streams", type=int, default=64, help="serve: independent streams")
    ap.add_argument("--rate", type=float, default=2000.0, help="serve: aggregate Poisson arrival rate (slices/s)")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nnz", type=int, default=NNZ)
    ap.add_argument("--rank", type=int, default=RANK)
    ap.add_argument("--cpu-sample", type=int, default=CPU_SAMPLE_NNZ)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--factor-dtype", choices=["f32", "bf16"], default="f32",
                    help="factor storage (bf16 halves gather bytes; accumulation stays f32)")
    ap.add_argument("--independent", action="store_true",
                    help="mttkrp under torchrun: an independent tensor per rank (weak scaling, no collective) "
                         "instead of the one tensor sharded by output-row blocks")
    ap.add_argument("--tns-path", default=None, help="tns: where the text file is written (default: a temp dir)")
    ap.add_argument("--profile-small", action="store_true",
                    help="small case for ncu captures (mttkrp: 20M nonzeros; slice: a quarter of the tensor), 1 step")
    args = ap.parse_args()
    defaults = {"mttkrp": (10, 3), "cpstream": (197, 3), "serve": (7, 1), "slice": (20, 3), "tns": (3, 1),
                "cpals3d": (20, 1), "cpals5d": (5, 1)}[args.workload]
    if args.steps is None:
        args.steps = defaults[0]
    if args.warmup is None:
        args.warmup = defaults[1]
    return args


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def line_bytes_per_nnz(alto_bits):
    """Algorithmic line bytes per nonzero: the reference's key (8 bytes for a
    64-bit ALTO mask, 16 for a 128-bit one) plus a float32 value."""
    key = 8 if alto_bits <= 64 else 16
    return key + 4


def mttkrp_bytes(dims, nnz, rank, mode, alto_bits, fbytes=4):
    """Algorithmic bytes of one mode-`mode` MTTKRP: the line once (key + float32
    value per nonzero), each input factor row once, the output once."""
    others = sum(d for m, d in enumerate(dims) if m != mode)
    return nnz * line_bytes_per_nnz(alto_bits) + rank * fbytes * others + rank * 4 * dims[mode]


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None
            return
        # nvidia-smi's start-up (driver and NVML initialisation) stays out of
        # the timed region: wait for its first sample, 10 s at most
        deadline = time.time() + 10
        while not self.rows and self.proc.poll() is None and time.time() < deadline:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm = []
        reasons = set()
        smax = None
        for p in self.rows:
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for name, col in (("hw_slowdown", 5), ("hw_thermal_slowdown", 6), ("sw_thermal_slowdown", 7),
                              ("sw_power_cap", 8)):
                if p[col].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def recorded_traffic():
    """DRAM bytes per MTTKRP launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "mttkrp_powerlaw3d_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return None


def host_tensor(n, seed):
    """n nonzeros of the workload's distribution as host arrays (uint64
    indices [3, n], float64 values): drawn on cuda:0 by the same generator as
    the timed tensor (seed 1234 gives exactly rank 0's timed tensor), else on
    the host with numpy when no GPU is visible."""
    import numpy as np

    from alto_b200 import synth

    try:
        import torch

        if torch.cuda.is_available():
            c, v = synth.zipf_coo_device(DIMS, n, ZIPF, seed=seed, values="lognormal", device="cuda:0")
            cidx = c.cpu().numpy().astype(np.uint64)
            vals = v.double().cpu().numpy()
            del c, v
            torch.cuda.empty_cache()
            return cidx, vals
    except ImportError:
        pass
    return synth.powerlaw_coo(DIMS, n, ZIPF, seed=seed, values="lognormal")


def host_mem_available():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def reference_threads(nnz, rank, threads):
    """Threads (= the reference's partitions) whose per-thread da_mem buffers
    fit the host: each holds a whole-mode output block (the power-law
    intervals span nearly every row), max(dims) x rank float64, beside about
    120 bytes per nonzero of COO, ALTO and sort buffers and the factors."""
    avail = host_mem_available()
    base = nnz * 120 + sum(DIMS) * rank * 8 * 2
    per = max(DIMS) * rank * 8
    fit = int((avail * 0.85 - base) // per) if avail else threads
    return max(0, min(threads, fit)), avail


def time_reference_cpu(n, rank, reps, seed=2024):
    """Seconds per all-mode step of the reference's mttkrp_alto_par (OpenMP)
    on n nonzeros of the workload distribution; returns (sec, threads, nnz,
    host bytes available).  Threads: all host threads, fewer if the
    reference's per-thread buffers would not fit host memory."""
    import numpy as np

    import oracle as O

    L = O.ref_lib(128)
    threads, avail = reference_threads(n, rank, os.cpu_count() or 1)
    if threads < 1:
        raise MemoryError(f"{n} nonzeros need more than the {avail / 2**30:.0f} GiB of host memory available")
    L.ref_set_threads(threads)
    cidx, vals = host_tensor(n, seed)
    rng = np.random.default_rng(seed + 1)
    F = [rng.uniform(-1.0, 1.0, (d, rank)) for d in DIMS]
    with stdout_to_stderr():
        t = O.RefTensor(DIMS, cidx, vals, threads, bits=128)
        del cidx, vals
        sec = t.mttkrp_time(-1, F, rank, reps)
    nnz = t.nnz
    t.close()
    return sec, threads, nnz, avail


def reference_variants(nnz):
    """The variant the reference's dispatcher picks per mode
    (include/alto.hpp:835-846): atomic when dims > 512 and nnz/dims <= 4,
    else da_mem_pull."""
    return ["atomic" if d > 512 and nnz // d <= 4 else "da_mem_pull" for d in DIMS]


def reference_arm(args):
    """The reference's own OpenMP MTTKRP (oracle/_ref, mttkrp_alto_par) on the
    whole workload tensor -- the very tensor rank 0 of the GPU arm times
    (same generator and seed) -- when its buffers fit host memory, else on
    the 24M-nonzero sample that keeps the same variant; steps = repetitions
    of the all-mode MTTKRP after one untimed one."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    n, seed, same = args.nnz, 1234, True
    threads, avail = reference_threads(n, args.rank, os.cpu_count() or 1)
    if threads < max(1, (os.cpu_count() or 1) // 4):
        n, seed, same = args.cpu_sample, 2024, False
    try:
        sec, threads, nnz, avail = time_reference_cpu(n, args.rank, max(args.steps, 1), seed=seed)
    except Exception as e:  # the compiled reference (oracle/_ref) is missing or failed to load
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref could not run: {e}"}))
        return 0
    units = nnz * args.rank * len(DIMS)
    value = units / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "nnz*R/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": 1, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "nnz": nnz, "dims": DIMS, "rank": args.rank, "same_config": same,
                   "threads": threads, "host_mem_available_gib": round(avail / 2**30, 1),
                   "variants": reference_variants(nnz),
                   "note": ("the whole tensor the GPU arm times (same generator and seed)" if same else
                            "24M-nonzero sample of the same distribution: the whole tensor's per-thread "
                            "buffers do not fit this host's memory")},
        "cpu_baseline": {"value": value, "unit": "nnz*R/s", "cores": threads, "kind": "reference",
                         "sample": f"{nnz} nonzeros, all-mode MTTKRP, {max(args.steps, 1)} reps"},
        "e2e": {"value": value, "unit": "nnz*R/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def sampled_rows_error(cidx, vals, factors, outs, R, nrows=4096, seed=5):
    """Max relative (normwise) error of each mode's MTTKRP output against
    float64 sums recomputed on the host from the COO: 4096 rows drawn
    uniformly among the rows that hold nonzeros, plus the heaviest row.
    cidx/vals: the generated COO on the device; factors: the float32 inputs
    (their values widened exactly); outs: the device outputs."""
    import numpy as np
    import torch

    rng = np.random.default_rng(seed)
    F64 = [f.double().cpu() for f in factors]
    errs, picked = [], []
    for m in range(cidx.shape[0]):
        present = torch.unique(cidx[m])
        take = torch.from_numpy(rng.choice(present.numel(), min(nrows, present.numel()), replace=False))
        heavy = torch.bincount(cidx[m]).argmax().view(1)
        rows = torch.unique(torch.cat([present[take.to(present.device)], heavy]))
        sel = torch.isin(cidx[m], rows)
        idx = cidx[:, sel].cpu()
        v = vals[sel].double().cpu()
        prod = v[:, None].expand(-1, R).clone()
        for o in range(cidx.shape[0]):
            if o != m:
                prod *= F64[o].index_select(0, idx[o])
        rows_h = rows.cpu()
        pos = torch.searchsorted(rows_h, idx[m])
        ref = torch.zeros((rows_h.numel(), R), dtype=torch.float64).index_add_(0, pos, prod)
        got = outs[m].index_select(0, rows).double().cpu()
        errs.append(float((got - ref).abs().max() / ref.abs().max().clamp_min(1e-300)))
        picked.append(int(sel.sum()))
    return errs, picked


def ours(args):
    import numpy as np
    import torch

    import alto_b200 as A
    from alto_b200 import synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    nnz = args.nnz
    steps, warmup = args.steps, args.warmup
    if args.profile_small:
        nnz, steps, warmup = 20_000_000, 1, 1
    R = args.rank
    N = len(DIMS)

    # Under torchrun: the one tensor sharded by output-row blocks (strong
    # scaling; every rank draws the same tensor and encodes, per mode, only
    # the nonzeros of its block of that mode's rows), or with --independent
    # a tensor of its own per rank (weak scaling, no collective).
    from alto_b200 import shard

    sharded = world > 1 and not args.independent
    encode = None
    seed = 1234 if (sharded or world == 1) else 1234 + rank
    cidx, vals = synth.zipf_coo_device(DIMS, nnz, ZIPF, seed=seed, values="lognormal", device=dev)
    total_nnz = int(cidx.shape[1])
    bounds = None
    if sharded:
        tens, bounds = [], []
        for m in range(N):
            b = shard.row_blocks(torch.bincount(cidx[m], minlength=DIMS[m]), world)
            c_r, v_r = shard.select_block(cidx, vals, m, b[rank], b[rank + 1])
            tens.append(A.AltoTensor(DIMS, c_r, v_r, nprtn=1))
            bounds.append(b)
            del c_r, v_r
        del cidx, vals
        t = tens[0]
    else:
        # the ALTO encode of the whole tensor (device COO in, line out), timed
        # after a 1M-nonzero encode has loaded the encoder's kernels
        A.AltoTensor(DIMS, cidx[:, :1_000_000].contiguous(), vals[:1_000_000].contiguous(), nprtn=1).close()
        torch.cuda.synchronize()
        te0 = time.perf_counter()
        t = A.AltoTensor(DIMS, cidx, vals, nprtn=1)
        torch.cuda.synchronize()
        encode_s = time.perf_counter() - te0
        # algorithmic bytes: the COO read once (int64 coordinates, float32
        # values), the line written once (key words + value)
        encode_bytes = total_nnz * (8 * N + 4 + line_bytes_per_nnz(t.alto_bits))
        encode = {"ms": round(encode_s * 1e3, 2), "nnz_per_s": total_nnz / encode_s,
                  "algorithmic_gbs": encode_bytes / encode_s / 1e9,
                  "timing": "host clock around the call with device syncs; includes its allocations"}
        tens = [t] * N
    nnz = t.nnz
    torch.cuda.empty_cache()
    g = torch.Generator(device=dev)
    g.manual_seed(99 + rank)
    fdt = torch.bfloat16 if args.factor_dtype == "bf16" else torch.float32
    factors = [(torch.rand((d, R), generator=g, device=dev) * 2 - 1).to(fdt).contiguous() for d in DIMS]
    outs = [torch.empty((d, R), device=dev, dtype=torch.float32) for d in DIMS]
    stream = torch.cuda.current_stream()

    def timed(fn, reps=1):  # ms per call of fn, CUDA events on the stream
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    # the row-sorted copies (built on first use): build time = first call - a later call
    bytes0 = sum(x.device_bytes() for x in set(tens))
    sorted_build_ms = []
    for m in range(N):
        first = timed(lambda: tens[m].mttkrp(m, factors, R, out=outs[m], variant=A.SORTED, stream=stream))
        again = timed(lambda: tens[m].mttkrp(m, factors, R, out=outs[m], variant=A.SORTED, stream=stream))
        sorted_build_ms.append(round(first - again, 2))
    sorted_bytes = sum(x.device_bytes() for x in set(tens)) - bytes0
    # project autotuner: fastest kernel variant per mode (of each mode's tensor)
    tuned = {id(x): x.autotune(factors, R) for x in set(tens)}
    variants = [tuned[id(tens[m])][m] for m in range(N)]
    vnames = {A.ATOMIC: "atomic", A.STAGED: "staged", A.STREAM: "stream", A.SORTED: "sorted"}

    def step(ev=None):
        for m in range(N):
            outs[m].zero_()
            if ev is not None:
                ev[m][0].record(stream)
            tens[m].mttkrp(m, factors, R, out=outs[m], accumulate=True, stream=stream)
            if ev is not None:
                ev[m][1].record(stream)
            if sharded:
                shard.allgather_rows(outs[m], bounds[m])

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    events = [[[torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)] for _ in range(N)]
              for _ in range(steps)]
    launches0 = A.kernel_launches()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed launches
    t0.record(stream)
    for k in range(steps):
        step(events[k])
    t1.record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    launches = A.kernel_launches() - launches0
    if world > 1:
        torch.distributed.barrier()
    clocks = sampler.stop()
    elapsed = t0.elapsed_time(t1) / 1e3
    if world > 1:
        x = torch.tensor([elapsed], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(x, op=torch.distributed.ReduceOp.MAX)
        elapsed = float(x.item())
    units = (total_nnz if sharded else nnz * world) * R * N * steps
    value = units / elapsed

    # roofline of the MTTKRP kernel (per-mode launches, CUDA events on its stream)
    alto_bits = t.alto_bits
    per_mode = []
    for m in range(N):
        dt = statistics.mean(events[k][m][0].elapsed_time(events[k][m][1]) / 1e3 for k in range(steps))
        b = mttkrp_bytes(DIMS, tens[m].nnz, R, m, alto_bits, fbytes=2 if args.factor_dtype == "bf16" else 4)
        per_mode.append((m, dt, b))
    bytes_launch = sum(b for _, _, b in per_mode) / N
    dt_launch = sum(dt for _, dt, _ in per_mode) / N
    achieved = bytes_launch / dt_launch / 1e9
    peak, peak_kind = measured_peaks()
    traffic = recorded_traffic()

    # the ALTO line itself (vector atomics, no row-sorted copy), per mode
    line_ms = [round(timed(lambda: tens[m].mttkrp(m, factors, R, out=outs[m], variant=A.ATOMIC, stream=stream), 3),
                     4) for m in range(N)]
    # the row-sorted walks the autotuner chooses among, per mode (3-mode tensors)
    feed_ms = None
    if N == 3:
        feed_ms = {name: [round(timed(lambda: tens[m].mttkrp(m, factors, R, out=outs[m], variant=A.SORTED | f,
                                                               stream=stream), 3), 4) for m in range(N)]
                   for name, f in (("four_blocks", 0), ("five_blocks", A.FEED_DENSE),
                                   ("five_blocks_fixed_target", A.FEED_FIXED_TARGET))}
    # error against float64 sums from the generated COO, on the last timed step's outputs
    err = None
    if not sharded:
        for m in range(N):
            outs[m].zero_()
            t.mttkrp(m, factors, R, out=outs[m], accumulate=True, stream=stream)
        torch.cuda.synchronize()
        errs, picked = sampled_rows_error(cidx, vals, factors, outs, R)
        err = {"max_rel_err": max(errs), "per_mode": errs, "bound": 1e-5,
               "method": "normwise max |gpu - fp64| / max |fp64| over 4096 uniformly drawn rows with "
                         "nonzeros plus the heaviest row of each mode; float64 sums on the host from the "
                         "generated COO and the float32 factor values",
               "nonzeros_checked": picked}
        del cidx, vals
        torch.cuda.empty_cache()

    # end to end through the host-buffer C-ABI entry point
    e2e = None
    if sharded:
        e2e = {"value": None, "unit": "nnz*R/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
               "note": "not measured when sharded (the host-buffer entry point covers one rank's tensors)"}
    elif not args.no_e2e:
        hostF = [torch.empty((d, R), dtype=torch.float64, pin_memory=True) for d in DIMS]
        for h, f in zip(hostF, factors):
            h.copy_(f.float().double().cpu())
        hostN = [h.numpy() for h in hostF]
        # a CP-ALS caller: after each mode's MTTKRP it rewrites that factor
        # (its solve), so each call declares the previous mode's factor
        # changed and only that one crosses PCIe again
        t.mttkrp_host(N - 1, hostN, R)  # warm (every factor copied)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        prev = N - 1
        ts = time.perf_counter()
        for _ in range(args.e2e_steps):
            for m in range(N):
                t.mttkrp_host(m, hostN, R, changed=[prev])
                prev = m
        te = time.perf_counter() - ts
        if world > 1:
            x = torch.tensor([te], device=dev, dtype=torch.float64)
            torch.distributed.all_reduce(x, op=torch.distributed.ReduceOp.MAX)
            te = float(x.item())
        h2d = sum(d * R * 8 for d in DIMS)
        d2h = sum(d * R * 8 for d in DIMS)
        e2e = {"value": nnz * R * N * args.e2e_steps * world / te, "unit": "nnz*R/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": te / args.e2e_steps * 1e3,
               "api": "alto_mttkrp_host_changed (float64 host factors, pinned; per call the factor the "
                      "previous call returned is declared changed, as a CP-ALS loop rewrites it, and crosses "
                      "PCIe again; the output factor comes back)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.profile_small:
        try:
            sec, threads, snnz, _ = time_reference_cpu(args.cpu_sample, R, 3)
            cpu = {"value": snnz * R * N / sec, "unit": "nnz*R/s", "cores": threads, "kind": "reference",
                   "sample": f"{snnz} nonzeros of the same distribution, all-mode MTTKRP, 3 reps; the "
                             f"reference's variants per mode: {reference_variants(snnz)} (as on the whole "
                             f"tensor: {reference_variants(nnz)})"}
        except Exception as e:
            cpu = {"value": None, "unit": "nnz*R/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "nnz*R/s", "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": elapsed / steps * 1e3, "higher_is_better": True,
            "scaling": "strong" if sharded else "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "dims": DIMS, "nnz": total_nnz if sharded else nnz, "rank": R,
                       "zipf": 1.2,
                       "values": "lognormal(0,1)", "key_bits": t.key_bits, "alto_bits": alto_bits,
                       "factor_dtype": args.factor_dtype,
                       "parallelism": (f"one tensor; per mode, equal-nnz output-row blocks on {world} GPUs, each "
                                       f"encoding its own nonzeros, + a row all-gather (NCCL broadcast per block) "
                                       f"per mode" if sharded else
                                       (f"independent tensor per GPU x{world}" if world > 1 else "one GPU")),
                       "l2": "inputs larger than L2 (line + factors > 3 GB); no flush",
                       "line_bytes_per_nnz": line_bytes_per_nnz(alto_bits),
                       "variants": [vnames.get(v, str(v)) for v in variants],
                       "row_sorted_copies": {
                           "bytes": sorted_bytes, "build_ms_per_mode": sorted_build_ms,
                           "order": "per mode: output row, ALTO order kept among equal rows (stable LSD "
                                    "sort on the row); built once, outside the timed region"},
                       "alto_line_atomic_ms_per_mode": line_ms,
                       "row_sorted_walks_ms_per_mode": feed_ms,
                       "alto_encode": encode,
                       "device_bytes": sum(x.device_bytes() for x in set(tens))},
            "error_vs_fp64": err,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic.get("bytes_per_launch") if traffic else None,
                         "traffic_captured_on": traffic.get("kernel") if traffic else None,
                         "per_mode_ms": [round(dt * 1e3, 4) for _, dt, _ in per_mode],
                         "algorithmic_bytes_per_mode": [b for _, _, b in per_mode]},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clocks,
            "gpu_launches": launches,
        }
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    for x in set(tens):
        x.close()
    return line if rank == 0 else None


# ----------------------------------------------------------------- CP-stream

C4_SPACE = [100000, 100000, 10000]
C4_RANK = 16
C4_SEED = 7
CPSTREAM_METRIC = "CP-stream slices/s (rank 16, non-negative ADMM)"
CPSTREAM_WORKLOAD = "cpstream4d-200slices-100Kx100Kx10K-zipf1.1-poisson3-R16-nonneg-f0.95-m50-e1e-5"


def c4_batches(n):
    """The first n slices of the CP-stream workload (host COO)."""
    import numpy as np

    from alto_b200 import synth

    return synth.stream_batches(
        C4_SPACE, n, lambda rng, s: int(np.clip(rng.lognormal(np.log(2e5), 1.0), 5e4, 2e6)),
        [1.1, 1.1, 1.1], seed=C4_SEED, values="poisson3")


def stream_need(batches, R):
    """Initial values consumed per batch (new rows x rank, mode order)."""
    import numpy as np

    prev = np.zeros(len(batches[0]["dims"]), np.int64)
    out = []
    for b in batches:
        d = b["dims"].astype(np.int64)
        out.append(int(np.sum(np.maximum(d - prev, 0))) * R)
        prev = np.maximum(prev, d)
    return out


def cpstream_bytes(b, R, inner):
    """Algorithmic HBM bytes of one slice update: per inner iteration the
    line once per mode (key + value) and, per non-stream mode, the factor,
    previous factor and solve buffer read plus buffer and factor written."""
    N = len(b["dims"])
    nnz = len(b["vals"])
    return inner * (N * nnz * 12 + sum(int(d) * R * 4 * 5 for m, d in enumerate(b["dims"]) if m != 0))


class stdout_to_stderr:
    """Sends what native code prints to file descriptor 1 (the reference's
    per-slice tables) to stderr, so stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *exc):
        sys.stdout.flush()
        import ctypes

        ctypes.CDLL(None).fflush(None)  # C stdio buffers still hold the native prints
        os.dup2(self.saved, 1)
        os.close(self.saved)


def ref_cpstream_rate(batches, R, iv, model="cpstream"):
    """Slices/s of the reference's cpstream or spcpstream (oracle/_ref, all
    host threads)."""
    import oracle as O

    L = O.ref_lib(64)
    threads = os.cpu_count() or 1
    L.ref_set_threads(threads)
    with stdout_to_stderr():
        if model == "spcpstream":
            _, _, secs = O.ref_spcpstream(batches, 0, R, 50, 1e-5, iv, bits=64)
        else:
            _, _, secs = O.ref_cpstream(batches, 0, R, 50, 1e-5, 1, iv, bits=64)
    return len(batches) / float(secs.sum()), threads, [round(float(x) * 1e3, 1) for x in secs]


class DeviceActivity:
    """Device activity of a region (kernels, copies, memsets) recorded by
    torch.profiler (CUPTI), which sees this library's kernels and the kernel
    nodes of its CUDA graphs as well as torch's own."""

    def __init__(self, enabled):
        self.prof = None
        if enabled:
            from torch.profiler import ProfilerActivity, profile

            self.prof = profile(activities=[ProfilerActivity.CUDA])

    def start(self):
        if self.prof is not None:
            self.prof.__enter__()

    def stop(self, wall_s):
        if self.prof is None:
            return None
        import torch

        torch.cuda.synchronize()
        self.prof.__exit__(None, None, None)
        try:
            per = {}
            busy = []
            for e in self.prof.events():
                if e.device_type != torch.autograd.DeviceType.CUDA:
                    continue
                t0, t1 = e.time_range.start, e.time_range.end
                busy.append((t0, t1))
                k = per.setdefault(e.name, [0.0, 0])
                k[0] += (t1 - t0) / 1e3
                k[1] += 1
            busy.sort()
            covered, end = 0.0, None  # union of the activity intervals (us)
            for t0, t1 in busy:
                if end is None or t0 > end:
                    covered += t1 - t0
                    end = t1
                elif t1 > end:
                    covered += t1 - end
                    end = t1
            top = sorted(per.items(), key=lambda kv: -kv[1][0])[:15]
            total = sum(v[0] for v in per.values())
            return {"device_busy_ms": covered / 1e3, "wall_ms": wall_s * 1e3,
                    "busy_share": covered / 1e3 / (wall_s * 1e3), "activity_ms_sum": total,
                    "activities": sum(v[1] for v in per.values()),
                    "top": [{"name": n[:90], "ms": round(v[0], 3), "count": v[1]} for n, v in top],
                    "note": "recorded with torch.profiler (CUPTI); the throughput of this run is not a bench number"}
        except Exception as e:  # the profiler's event model differs between torch versions
            return {"error": f"{type(e).__name__}: {e}"}


def ours_cpstream(args):
    import numpy as np
    import torch

    import alto_b200 as A
    from alto_b200 import synth

    torch.cuda.set_device(0)
    W, K = args.warmup, args.steps
    batches = c4_batches(W + K)
    R = C4_RANK
    need = stream_need(batches, R)
    iv = synth.init_values(sum(need) + 64, seed=1)
    s = A.CPStream(4, 0, R, constraint=A.NONNEG, forgetting=0.95, max_inner=50, epsilon=1e-5)
    if args.model == "spcpstream":
        s.set_model(A.SPCPSTREAM)
    s.set_graph(not args.no_graph)
    used = 0
    lat, inner, dev_ms, nbytes, h2d = [], [], [], 0, 0
    stream = torch.cuda.current_stream()
    sampler = None
    launches0 = 0
    activity = DeviceActivity(args.kernel_share)
    for k, b in enumerate(batches):
        if k == W:
            torch.cuda.synchronize()
            sampler = ClockSampler(0)
            sampler.start()
            time.sleep(0.3)
            launches0 = A.kernel_launches()
            activity.start()
            t_start = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ts = time.perf_counter()
        it = s.push(b["dims"], b["cidx"], b["vals"], iv[used:used + need[k]])
        te = time.perf_counter() - ts
        e1.record(stream)
        used += need[k]
        if k >= W:
            e1.synchronize()
            lat.append(te * 1e3)
            dev_ms.append(e0.elapsed_time(e1))
            inner.append(it)
            nbytes += cpstream_bytes(b, R, it)
            h2d += b["cidx"].nbytes + b["vals"].nbytes + need[k] * 8
    t_total = time.perf_counter() - t_start
    share = activity.stop(t_total)
    launches = A.kernel_launches() - launches0
    clocks = sampler.stop()
    phases = s.stats()
    s.close()
    dev_total = sum(dev_ms) / 1e3
    peak, peak_kind = measured_peaks()
    cpu = None
    if not args.no_cpu_baseline:
        try:
            nb = 6
            rate, threads, secs = ref_cpstream_rate(batches[:nb], R, iv, args.model)
            cpu = {"value": rate, "unit": "slices/s", "cores": threads, "kind": "reference",
                   "sample": f"first {nb} slices of the same stream through the reference's cpstream "
                             f"(its forgetting factor is fixed at 0.99); per-slice ms {secs}"}
        except Exception as e:
            cpu = {"value": None, "unit": "slices/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}
    line = {
        "metric": CPSTREAM_METRIC + (" [spCP-stream model]" if args.model == "spcpstream" else ""),
        "value": K / dev_total, "unit": "slices/s", "n_gpus": 1, "steps": K,
        "warmup": W, "ms_per_step": dev_total / K * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": CPSTREAM_WORKLOAD, "model": args.model, "space_dims": C4_SPACE, "rank": R,
                   "constraint": "nonneg" if args.model == "cpstream" else "none (spCP-stream does not constrain)",
                   "forgetting": 0.95, "max_inner": 50, "epsilon": 1e-5,
                   "slice_nnz_mean": float(np.mean([len(b["vals"]) for b in batches[W:]])),
                   "inner_iters_mean": float(np.mean(inner)), "inner_iters_max": int(np.max(inner)),
                   "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                   "latency_ms": [round(x, 2) for x in lat],
                   "inner_iters": [int(x) for x in inner],
                   "launch": ("every inner iteration launched directly" if args.no_graph
                              else "one captured graph per session, relaunched for every slice (a device-side "
                                   "loop over the inner iterations)"),
                   "l2": "per-slice work streams the slice and the factors (> L2 in total over a slice); no flush"},
        "roofline": {"bound": "hbm", "achieved": nbytes / dev_total / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": nbytes / dev_total / 1e9 / peak, "peak_kind": peak_kind, "traffic": None,
                     "note": "algorithmic bytes per inner iteration: N*nnz*12 + sum_j I_j*R*4*5"},
        "cpu_baseline": cpu,
        "e2e": {"value": K / t_total, "unit": "slices/s", "h2d_bytes_per_step": h2d // K,
                "d2h_bytes_per_step": R * 8, "api": "alto_stream_push (host COO batch in, time row out)"},
        "clocks": clocks,
        "gpu_launches": launches,
    }
    # the session's own account of every push (warm-up included): host ms
    # per phase and the device ms of the inner-iteration launches
    line["config"]["session_phases"] = {k: round(v, 2) if isinstance(v, float) else v for k, v in phases.items()}
    if share is not None:
        line["kernel_share"] = share
    return line


# ------------------------------------------------------------------- serving

SERVE_METRIC = "CP-stream serving slices/s (64 streams, Poisson 2000 slices/s)"
SERVE_WORKLOAD = "serve-64streams-dims1e3..1e6-R8/16/32-nnz1e4..1e6-poisson2000-budget80GB"
SERVE_SEED = 11


def serve_setup(args):
    import numpy as np

    from alto_b200 import synth

    # (each stream's slices: warm-up, the saturated phase, the sustained phase)
    streams = synth.serving_streams(args.streams, args.warmup + 2 * args.steps, seed=SERVE_SEED)
    rng = np.random.default_rng(SERVE_SEED + 1)
    need = [sum(st["dims"][1:]) * st["rank"] for st in streams]
    pool = rng.uniform(0.0, 3.0, max(need) + 1024) * np.where(rng.random(max(need) + 1024) < 0.5, -1.0, 1.0)
    offs = [int(rng.integers(0, len(pool) - n)) for n in need]
    # arrival order of the timed slices: a random interleaving that keeps each
    # stream's slices in order, at exponential gaps
    order = np.repeat(np.arange(len(streams)), args.steps)
    rng.shuffle(order)
    gaps = rng.exponential(1.0 / args.rate, len(order))
    return streams, pool, offs, need, order, np.cumsum(gaps)


def ours_serve(args):
    import numpy as np
    import torch

    import alto_b200 as A

    from alto_b200 import shard

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:  # streams sharded over the GPUs, one server each; no data crosses GPUs
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    streams, pool, offs, need, order, arrive = serve_setup(args)
    mine = shard.streams_for_rank(len(streams), rank, world)
    keep = np.isin(order, mine)
    order, arrive = order[keep], arrive[keep]
    W, K = args.warmup, args.steps
    cons = {0: A.UNCONSTRAINED, 1: A.NONNEG}

    def across_ranks(x, op):  # max / sum / min of a host number over the ranks
        if world == 1:
            return x
        import torch.distributed as dist

        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op={"max": dist.ReduceOp.MAX, "sum": dist.ReduceOp.SUM, "min": dist.ReduceOp.MIN}[op])
        return t.item()

    def init_for(k, j):  # initial values with the first slice only
        return pool[offs[k]:offs[k] + need[k]] if j == 0 else None

    # plain path: one session per stream, one slice at a time, arrival order
    model = A.SPCPSTREAM if args.model == "spcpstream" else A.CPSTREAM
    sess = {k: A.CPStream(4, 0, streams[k]["rank"], constraint=cons[streams[k]["constraint"]], forgetting=0.99,
                          max_inner=10, epsilon=1e-5) for k in mine}
    for x in sess.values():
        x.set_model(model)
    for j in range(W):
        for k in mine:
            b = streams[k]["slices"][j]
            sess[k].push(b["dims"], b["cidx"], b["vals"], init_for(k, j))
    torch.cuda.synchronize()
    nxt = [W] * len(streams)
    iso = []
    t0 = time.perf_counter()
    for k in order:
        b = streams[k]["slices"][nxt[k]]
        ts = time.perf_counter()
        sess[k].push(b["dims"], b["cidx"], b["vals"])
        iso.append((time.perf_counter() - ts) * 1e3)
        nxt[k] += 1
    plain_s = time.perf_counter() - t0
    check = mine[:8]
    plain_out = {k: [sess[k].factor(m, int(streams[k]["dims"][m]) + 1) for m in (1, 2, 3)] for k in check}
    for x in sess.values():
        x.close()
    del sess
    torch.cuda.synchronize()

    # server: warm-up slices, then the timed slices at their arrival times
    srv = A.Server(80 << 30, workers=args.workers)
    sids = {k: srv.open(4, 0, streams[k]["rank"], streams[k]["dims"], max(len(b["vals"]) for b in streams[k]["slices"]),
                        constraint=cons[streams[k]["constraint"]], forgetting=0.99, max_inner=10, epsilon=1e-5,
                        model=model) for k in mine}
    for j in range(W):
        for k in mine:
            b = streams[k]["slices"][j]
            srv.submit(sids[k], b["dims"], b["cidx"], b["vals"], init_for(k, j))
    srv.drain()
    st0 = srv.stats()
    if world > 1:
        torch.distributed.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    launches0 = A.kernel_launches()
    nxt = [W] * len(streams)
    tickets = []
    h2d = 0
    activity = DeviceActivity(args.kernel_share)
    activity.start()
    t0 = time.perf_counter()
    for k, ta in zip(order, arrive):
        while time.perf_counter() - t0 < ta:
            pass
        b = streams[k]["slices"][nxt[k]]
        tickets.append(srv.submit(sids[k], b["dims"], b["cidx"], b["vals"]))
        h2d += b["cidx"].nbytes + b["vals"].nbytes
        nxt[k] += 1
    srv.drain()
    served_s = time.perf_counter() - t0
    share = activity.stop(served_s)
    launches = A.kernel_launches() - launches0
    clocks = sampler.stop()
    lat = [srv.wait(t)[1] for t in tickets]
    st1 = srv.stats()
    same = all(np.array_equal(srv.factor(sids[k], m), plain_out[k][i]) for k in check
               for i, m in enumerate((1, 2, 3)))
    # sustained phase: the next slices of every stream at 60% of the rate the
    # saturated phase sustained (each rank at its share), so latency is the
    # update's own and not a queue's
    rate2 = 0.6 * len(order) / served_s
    rng2 = np.random.default_rng(SERVE_SEED + 2)
    order2 = np.repeat(np.asarray(mine), K)
    rng2.shuffle(order2)
    arrive2 = np.cumsum(rng2.exponential(1.0 / rate2, len(order2)))
    tickets2 = []
    t0 = time.perf_counter()
    for k, ta in zip(order2, arrive2):
        while time.perf_counter() - t0 < ta:
            pass
        b = streams[k]["slices"][nxt[k]]
        tickets2.append(srv.submit(sids[k], b["dims"], b["cidx"], b["vals"]))
        nxt[k] += 1
    srv.drain()
    sustained_s = time.perf_counter() - t0
    lat2 = [srv.wait(t)[1] for t in tickets2]
    srv.destroy()

    # whole job: every rank's slices over the slowest rank's time
    n_local = len(order)
    n = int(across_ranks(n_local, "sum"))
    served_s = across_ranks(served_s, "max")
    plain_s = across_ranks(plain_s, "max")
    same = bool(across_ranks(1 if same else 0, "min"))
    launches = int(across_ranks(launches, "sum"))
    h2d = int(across_ranks(h2d, "sum"))
    if world > 1:
        import torch.distributed as dist

        parts = [None] * world
        dist.all_gather_object(parts, (lat, iso, lat2, rate2, len(order2), sustained_s))
        lat = [x for p in parts for x in p[0]]
        iso = [x for p in parts for x in p[1]]
        lat2 = [x for p in parts for x in p[2]]
        rate2 = sum(p[3] for p in parts)
        sustained_rate = sum(p[4] for p in parts) / max(p[5] for p in parts)
        dist.barrier()
        dist.destroy_process_group()
        if rank != 0:
            return None
    value = n / served_s
    plain_rate = n / plain_s
    p99_iso = float(np.percentile(iso, 99))
    if world == 1:
        sustained_rate = len(order2) / sustained_s
    line = {
        "metric": SERVE_METRIC + (" [spCP-stream model]" if args.model == "spcpstream" else ""),
        "value": value, "unit": "slices/s", "n_gpus": world, "steps": n, "warmup": W * len(streams),
        "ms_per_step": served_s / n * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": SERVE_WORKLOAD, "model": args.model, "streams": len(streams), "slices_per_stream": W + K,
                   "parallelism": ("streams sharded round robin over %d GPUs, one server each, no collective" % world
                                   if world > 1 else "one GPU"),
                   "workers": args.workers, "arrival_rate": args.rate, "hbm_budget_bytes": 80 << 30,
                   "max_inner": 10, "epsilon": 1e-5,
                   "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                   "plain_slices_per_s": plain_rate, "speedup_vs_plain": value / plain_rate,
                   "isolated_p50_ms": float(np.percentile(iso, 50)), "isolated_p99_ms": p99_iso,
                   "p99_vs_isolated_p99": float(np.percentile(lat, 99)) / p99_iso,
                   "sustained": {"arrival_rate": rate2, "slices_per_s": sustained_rate,
                                 "speedup_vs_plain": sustained_rate / plain_rate,
                                 "p50_ms": float(np.percentile(lat2, 50)), "p99_ms": float(np.percentile(lat2, 99)),
                                 "p99_vs_isolated_p99": float(np.percentile(lat2, 99)) / p99_iso,
                                 "note": "the next slices of every stream arriving at 60% of the saturated "
                                         "phase's throughput (Poisson)"},
                   "results_identical_to_plain": bool(same), "checked_streams": len(check) * world,
                   "reserved_bytes": st1["reserved_bytes"], "admitted_streams": st1["admitted_streams"],
                   "warmup_completed": st0["completed"],
                   "server_time_ms": {k: round(st1[k] - st0[k], 1) for k in ("prepare_ms", "step_ms", "finish_ms")},
                   "group_steps": st1["steps"] - st0["steps"],
                   "mean_slices_per_step": ((st1["step_slices"] - st0["step_slices"]) /
                                            max(st1["steps"] - st0["steps"], 1)),
                   "timing": "host clock from the first timed arrival to the drained server",
                   "l2": "per-slice data and factors exceed L2 across streams; no flush"},
        "roofline": None,
        "cpu_baseline": None,
        "e2e": {"value": value, "unit": "slices/s", "h2d_bytes_per_step": h2d // n, "d2h_bytes_per_step": 0,
                "api": "alto_server_submit / alto_server_drain (host COO batches)"},
        "clocks": clocks,
        "gpu_launches": launches,
    }
    if share is not None:
        line["kernel_share"] = share
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = serve_reference_sample(streams, pool, offs, need, model=args.model)
    return line


def serve_reference_sample(streams, pool, offs, need, nstreams=6, nslices=3, model="cpstream"):
    """The reference's cpstream run stream after stream (its plain path) on a
    bounded sample: the first nslices slices of the first nstreams streams."""
    import oracle as O

    try:
        L = O.ref_lib(64)
        threads = os.cpu_count() or 1
        L.ref_set_threads(threads)
        total, count = 0.0, 0
        for k in range(min(nstreams, len(streams))):
            st = streams[k]
            iv = pool[offs[k]:offs[k] + need[k]]
            with stdout_to_stderr():
                if model == "spcpstream":
                    _, _, secs = O.ref_spcpstream(st["slices"][:nslices], 0, st["rank"], 10, 1e-5, iv, bits=64)
                else:
                    _, _, secs = O.ref_cpstream(st["slices"][:nslices], 0, st["rank"], 10, 1e-5, st["constraint"],
                                                iv, bits=64)
            total += float(secs.sum())
            count += nslices
        return {"value": count / total, "unit": "slices/s", "cores": threads, "kind": "reference",
                "sample": f"first {nslices} slices of the first {nstreams} streams, one stream after another"}
    except Exception as e:
        return {"value": None, "unit": "slices/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}


def reference_stream_arm(args):
    """--impl reference for the cpstream and serve workloads."""
    rank, _, _ = dist_env()
    if rank != 0:
        return 0
    try:
        if args.workload == "cpstream":
            from alto_b200 import synth

            nb = 6
            batches = c4_batches(nb)
            iv = synth.init_values(sum(stream_need(batches, C4_RANK)) + 64, seed=1)
            rate, threads, secs = ref_cpstream_rate(batches, C4_RANK, iv, args.model)
            metric, unit, workload = CPSTREAM_METRIC, "slices/s", CPSTREAM_WORKLOAD
            sample = f"first {nb} slices; per-slice ms {secs}"
        else:
            steps = args.steps
            args.steps = 2  # only the sample's slices are generated
            streams, pool, offs, need, _, _ = serve_setup(args)
            args.steps = steps
            cb = serve_reference_sample(streams, pool, offs, need, model=args.model)
            if cb["value"] is None:
                raise RuntimeError(cb["sample"])
            rate, threads, sample = cb["value"], cb["cores"], cb["sample"]
            metric, unit, workload = SERVE_METRIC, "slices/s", SERVE_WORKLOAD
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref could not run: {e}"}))
        return 0
    print(json.dumps({
        "impl": "reference", "metric": metric, "value": rate, "unit": unit, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": 0, "ms_per_step": 1e3 / rate, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": {"workload": workload},
        "cpu_baseline": {"value": rate, "unit": unit, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": rate, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


SLICE_METRIC = "stream slicer nnz/s (sort by time, first-seen relabel, every single-step batch)"
SLICE_WORKLOAD = "c4-shape-one-tensor-200x100kx100kx10k-lognormal-steps-zipf1.1"
SLICE_DIMS = [200, 100000, 100000, 10000]
SLICE_SEED = 77
SLICE_CPU_SAMPLE = 6_000_000


def slice_counts():
    import numpy as np

    rng = np.random.default_rng(SLICE_SEED)
    return np.clip(rng.lognormal(np.log(2e5), 1.0, SLICE_DIMS[0]), 5e4, 2e6).astype(np.int64)


def slice_tensor(dev, scale=1.0):
    """The slicer workload on the device: int64 index columns, float64 values
    (scale < 1 shrinks every time step's count, for profiler captures)."""
    import torch

    from alto_b200 import synth

    counts = (slice_counts() * scale).astype("int64")
    n = int(counts.sum())
    sp, v = synth.zipf_coo_device(SLICE_DIMS[1:], n, [1.1, 1.1, 1.1], seed=SLICE_SEED, device=dev)
    n = sp.shape[1]
    g = torch.Generator(device=dev)
    g.manual_seed(SLICE_SEED + 1)
    time_col = torch.repeat_interleave(torch.arange(SLICE_DIMS[0], device=dev),
                                       torch.as_tensor(counts, device=dev))[:n]
    time_col = time_col[torch.randperm(n, generator=g, device=dev)].contiguous()
    cols = [time_col] + [sp[m].contiguous() for m in range(3)]
    return cols, v.double()


def ref_slice_rate(cols, vals, n):
    """The reference's StreamingSparseTensor (oracle/_ref: tt_sort, relabel,
    next_dynamic_batch per time step, batches copied out) on the first n
    nonzeros (a uniform sample: the order is random); (nnz/s, threads, n)."""
    import numpy as np

    import oracle as O

    L = O.ref_lib(64)
    threads = os.cpu_count() or 1
    L.ref_set_threads(threads)
    c = np.stack([x[:n].cpu().numpy().astype(np.uint64) for x in cols])
    v = vals[:n].cpu().numpy()
    t0 = time.perf_counter()
    with stdout_to_stderr():
        O.ref_slice_stream(np.array(SLICE_DIMS, np.uint64), c, v, 0, 1, 1)
    sec = time.perf_counter() - t0
    return c.shape[1] / sec, threads, c.shape[1]


def ours_slice(args):
    import numpy as np
    import torch

    import alto_b200 as A

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    if args.profile_small:  # a quarter of the tensor, one warm-up and one timed step
        args.steps, args.warmup, args.no_e2e, args.no_cpu_baseline = 1, 1, True, True
    cols, vals = slice_tensor(dev, 0.25 if args.profile_small else 1.0)
    nnz = cols[0].numel()
    N = len(SLICE_DIMS)
    stream = torch.cuda.current_stream()

    def one(cidx, v):  # construction, then every single-step batch in one call
        sl = A.Slicer(SLICE_DIMS, cidx, v, 0)
        nb = sl.cut_all(1, 1)
        return sl, (sl.batch(0) if nb else None), nb

    for _ in range(args.warmup):
        one(cols, vals)[0].close()
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    launches0 = A.kernel_launches()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    nbs = []
    torch.cuda.synchronize()
    for k in range(args.steps):
        ev[k][0].record(stream)
        sl, _, nb = one(cols, vals)
        ev[k][1].record(stream)
        nbs.append(nb)
        sl.close()
    torch.cuda.synchronize()
    launches = A.kernel_launches() - launches0
    clocks = sampler.stop()
    ms = [a.elapsed_time(b) for a, b in ev]
    step_ms = sum(ms) / len(ms)
    value = nnz / (step_ms * 1e-3)

    # end to end through the C ABI: host COO (the reference's uint64 indices
    # and float64 values, pinned) in, every batch's indices and values back
    # into pinned host memory
    h_idx = torch.empty((N, nnz), dtype=torch.int64, pin_memory=True)
    for m in range(N):
        h_idx[m].copy_(cols[m])
    h_val = torch.empty(nnz, dtype=torch.float64, pin_memory=True)
    h_val.copy_(vals)
    hc = h_idx.numpy().view(np.uint64)  # one pinned [N, nnz] block: passed without a host copy
    hv = h_val.numpy()
    o_idx = [torch.empty(nnz, dtype=torch.int32, pin_memory=True) for _ in range(N)]
    o_val = torch.empty(nnz, dtype=torch.float64, pin_memory=True)
    e2e_ms = []
    for _ in range(0 if args.no_e2e else max(args.e2e_steps, 1) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sl, first, _ = one(hc, hv)
        # the batches are consecutive ranges of the slicer's arrays: one copy per array
        for m in range(N):
            o_idx[m].copy_(torch.as_tensor(A._DeviceArray(first.coo.cidx[m], nnz, "<i4"), device="cuda"),
                           non_blocking=True)
        o_val.copy_(torch.as_tensor(A._DeviceArray(first.coo.vals, nnz, "<f8"), device="cuda"), non_blocking=True)
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        sl.close()
    e2e_ms = e2e_ms[1:]
    e2e_val = nnz / (statistics.median(e2e_ms) * 1e-3) if e2e_ms else None

    peak, peak_kind = measured_peaks()
    algo = nnz * (N * 8 + 8) + nnz * (N * 4 + 8)
    achieved = algo / (step_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "slicer_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            t = json.load(f)
        traffic = t["bytes_per_nnz"] * nnz
    line = {
        "metric": SLICE_METRIC, "value": value, "unit": "nnz/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32+u64", "data": "synthetic",
        "config": {"workload": SLICE_WORKLOAD, "nnz": nnz, "dims": SLICE_DIMS, "stream_mode": 0,
                   "nnz_threshold": 1, "timeslice_limit": 1, "batches": nbs[0],
                   "step_ms_min": min(ms), "step_ms_max": max(ms), "step_ms_median": statistics.median(ms),
                   "step_ms": [round(x, 2) for x in ms],
                   "l2": "input (%.1f GB) exceeds L2; no flush" % (nnz * 40 / 1e9)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "kernel": "the whole slicing (all kernels of a step)",
                     "algorithmic_bytes": "per nonzero: 4 int64 indices + a float64 value read once, "
                                          "4 uint32 indices + a float64 value written once (64 B)",
                     "peak_kind": peak_kind},
        "cpu_baseline": None,
        "e2e": {"value": e2e_val, "unit": "nnz/s", "h2d_bytes_per_step": nnz * (N * 8 + 8),
                "d2h_bytes_per_step": nnz * (N * 4 + 8),
                "api": "alto_slicer_create (host COO) + alto_slicer_cut_all + batch contents to host"},
        "clocks": clocks,
        "gpu_launches": launches,
    }
    if not args.no_cpu_baseline:
        try:
            rate, threads, n = ref_slice_rate(cols, vals, args.cpu_sample if args.cpu_sample != CPU_SAMPLE_NNZ
                                              else SLICE_CPU_SAMPLE)
            line["cpu_baseline"] = {"value": rate, "unit": "nnz/s", "cores": threads, "kind": "reference",
                                    "sample": f"first {n} nonzeros (uniform sample), all single-step batches"}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": "nnz/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    print(json.dumps(line))
    return 0


def reference_slice_arm(args):
    rank, _, _ = dist_env()
    if rank != 0:
        return 0
    try:
        import torch

        cols, vals = slice_tensor(torch.device("cuda", 0)) if torch.cuda.is_available() else (None, None)
        if cols is None:
            raise RuntimeError("the workload generator needs a GPU")
        rate, threads, n = ref_slice_rate(cols, vals, SLICE_CPU_SAMPLE)
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref could not run: {e}"}))
        return 0
    print(json.dumps({
        "impl": "reference", "metric": SLICE_METRIC, "value": rate, "unit": "nnz/s", "n_gpus": args.gpus,
        "steps": 1, "warmup": 0, "ms_per_step": n / rate * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": {"workload": SLICE_WORKLOAD},
        "cpu_baseline": {"value": rate, "unit": "nnz/s", "cores": threads, "kind": "reference",
                         "sample": f"first {n} nonzeros (uniform sample), all single-step batches"},
        "e2e": {"value": rate, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


TNS_METRIC = "tensor file import nnz/s (.tns text into device memory)"
TNS_WORKLOAD = "tns-" + WORKLOAD.split("-R32")[0]
TNS_CPU_SAMPLE = 4_000_000


def tns_file(args, dev):
    """Write the MTTKRP workload's tensor as a .tns text file (once)."""
    import tempfile

    import torch

    import alto_b200 as A
    from alto_b200 import synth

    nnz = 20_000_000 if args.profile_small else args.nnz
    path = args.tns_path or os.path.join(tempfile.gettempdir(), f"alto_bench_{nnz}.tns")
    cidx, vals = synth.zipf_coo_device(DIMS, nnz, ZIPF, seed=1234, values="lognormal", device=dev)
    n = cidx.shape[1]
    A.write_tensor(path, DIMS, [cidx[m] for m in range(3)], vals.double())
    del cidx, vals
    torch.cuda.empty_cache()
    return path, n


def ref_import_rate(path, n_sample):
    """The reference's ImportSparseTensor (oracle/_ref, one host thread: the
    reader is serial) on the file's first n_sample lines."""
    import tempfile

    import oracle as O

    sample = os.path.join(tempfile.gettempdir(), "alto_bench_sample.tns")
    with open(path, "rb") as f, open(sample, "wb") as g:
        for _ in range(n_sample):
            line = f.readline()
            if not line:
                break
            g.write(line)
    L = O.ref_lib(64)
    import ctypes

    nm, nnz = ctypes.c_uint64(), ctypes.c_uint64()
    import numpy as np

    dims = np.zeros(16, np.uint64)
    t0 = time.perf_counter()
    L.ref_import_info(sample.encode(), 0, ctypes.c_uint64(0), ctypes.byref(nm),
                      dims.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nnz))
    sec = time.perf_counter() - t0
    size = os.path.getsize(sample)
    os.remove(sample)
    return nnz.value / sec, nnz.value, size


def ours_tns(args):
    import torch

    import alto_b200 as A

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    if args.profile_small:
        args.steps, args.warmup, args.no_cpu_baseline = 1, 1, True
    path, nnz = tns_file(args, dev)
    size = os.path.getsize(path)
    for _ in range(args.warmup):
        A.read_tensor(path).close()
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    launches0 = A.kernel_launches()
    walls, parses, reads, hostv = [], [], [], []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        t = A.read_tensor(path)
        walls.append((time.perf_counter() - t0) * 1e3)
        st = t.stats()
        parses.append(st["parse_ms"])
        reads.append(st["read_ms"])
        hostv.append(st["host_values"])
        n_read, dims = t.nnz, [int(x) for x in t.dims]
        t.close()
    launches = A.kernel_launches() - launches0
    clocks = sampler.stop()
    parse_ms = statistics.median(parses)
    wall_ms = statistics.median(walls)
    peak, peak_kind = measured_peaks()
    algo = size + n_read * 4 * 8
    achieved = algo / (parse_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "tns_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f)["bytes_per_line"] * n_read
    line = {
        "metric": TNS_METRIC, "value": n_read / (parse_ms * 1e-3), "unit": "nnz/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": parse_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": TNS_WORKLOAD, "nnz": n_read, "file_bytes": size, "dims": dims,
                   "wall_ms": wall_ms, "host_read_ms": statistics.median(reads),
                   "values_left_to_host_strtod": hostv[0],
                   "l2": "file (%.1f GB) exceeds L2; no flush" % (size / 1e9),
                   "timing": "value: CUDA events around the device parse (file bytes in HBM); "
                             "e2e: host clock around alto_read_tensor, file in the page cache"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "the device parse (all kernels after the file is in HBM)",
                     "algorithmic_bytes": "the file once, plus 3 uint64 indices and a float64 value per nonzero",
                     "peak_kind": peak_kind},
        "cpu_baseline": None,
        "e2e": {"value": n_read / (wall_ms * 1e-3), "unit": "nnz/s", "h2d_bytes_per_step": size,
                "d2h_bytes_per_step": 8 * len(dims), "api": "alto_read_tensor (text file -> device COO)"},
        "clocks": clocks,
        "gpu_launches": launches,
    }
    if not args.no_cpu_baseline:
        try:
            rate, n, sbytes = ref_import_rate(path, TNS_CPU_SAMPLE)
            line["cpu_baseline"] = {"value": rate, "unit": "nnz/s", "cores": 1, "kind": "reference",
                                    "sample": f"first {n} lines ({sbytes} bytes) of the same file"}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": "nnz/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    if not args.tns_path:
        os.remove(path)
    print(json.dumps(line))
    return 0


def reference_tns_arm(args):
    rank, _, _ = dist_env()
    if rank != 0:
        return 0
    try:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("the workload generator needs a GPU")
        args.nnz = min(args.nnz, 10_000_000)  # only the sample is read
        path, _ = tns_file(args, torch.device("cuda", 0))
        rate, n, sbytes = ref_import_rate(path, TNS_CPU_SAMPLE)
        os.remove(path)
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref could not run: {e}"}))
        return 0
    print(json.dumps({
        "impl": "reference", "metric": TNS_METRIC, "value": rate, "unit": "nnz/s", "n_gpus": args.gpus,
        "steps": 1, "warmup": 0, "ms_per_step": n / rate * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic", "config": {"workload": TNS_WORKLOAD},
        "cpu_baseline": {"value": rate, "unit": "nnz/s", "cores": 1, "kind": "reference",
                         "sample": f"first {n} lines ({sbytes} bytes) of the workload's file"},
        "e2e": {"value": rate, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


# ------------------------------------------------------------------ CP-ALS

CPALS3_DIMS = [1000, 1000, 1000]
CPALS3_NNZ = 1_000_000
CPALS5_DIMS = [100000, 100000, 10000, 1000, 100]
CPALS5_NNZ = 50_000_000
CPALS5_ZIPF = [1.1, 1.1, None, None, None]


def init_model(dims, R, seed):
    """Initial factors in [-3, 3] with random sign (the reference's rand_val range)."""
    from alto_b200 import synth

    init = synth.init_values(int(sum(dims)) * R, seed=seed)
    U0, off = [], 0
    for d in dims:
        U0.append(init[off:off + int(d) * R].reshape(int(d), R).copy())
        off += int(d) * R
    return U0


def flush_l2(buf):
    buf.add_(1.0)  # writes 256 MB, twice the L2


def ours_cpals3d(args):
    """CP-ALS on 1000^3 with 1,000,000 uniform distinct nonzeros (values
    U(0,1)), rank 16, a 64-bit ALTO mask, 20 iterations, plus 100 standalone
    mode-0 MTTKRPs; fits, factors and the MTTKRP checked against the FP64
    oracle (single-threaded restatement, fed the original float64 values and
    initial model).  The tensor is L2-resident (12 MB), so L2 is flushed
    before every timed MTTKRP."""
    import numpy as np
    import torch

    import alto_b200 as A
    import oracle as O
    from alto_b200 import synth

    torch.cuda.set_device(0)
    R, iters = 16, 20
    dims = np.array(CPALS3_DIMS, np.uint64)
    cidx, vals = synth.uniform_coo(dims, CPALS3_NNZ, seed=55)
    nnz = cidx.shape[1]
    t = A.create_alto(dims, cidx, vals)
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(5)
    F = [rng.uniform(-1, 1, (int(d), R)).astype(np.float32) for d in dims]
    Fd = [torch.tensor(f, device="cuda") for f in F]
    out = torch.empty((int(dims[0]), R), device="cuda", dtype=torch.float32)
    junk = torch.empty(64 << 20, device="cuda", dtype=torch.float32)
    for _ in range(3):
        t.mttkrp(0, Fd, R, out=out, stream=stream)
    launches0 = A.kernel_launches()
    ms = []
    for _ in range(100):
        flush_l2(junk)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t.mttkrp(0, Fd, R, out=out, stream=stream)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    launches = A.kernel_launches() - launches0
    mt_ms = float(np.mean(ms))
    enc = O.build(dims, cidx, vals)
    fo64 = [f.astype(np.float64) for f in F]
    fo64[0][:] = 0
    ref = O.mttkrp(enc, 0, fo64, R)[0]
    got = out.cpu().numpy()
    mt_err = float(np.abs(got - ref).max() / np.abs(ref).max())
    U0 = init_model(dims, R, 55)
    A.cpd_alto(t, U0, np.ones(R), R, 1, 1e-12)  # warm
    ts = time.perf_counter()
    U, lam, fits, it = A.cpd_alto(t, U0, np.ones(R), R, iters, 1e-12)
    cpd_s = time.perf_counter() - ts
    Uo, lo, fo, ito = O.cpd_als(enc, U0, np.ones(R), R, iters, 1e-12)
    fit_err = float(np.max(np.abs(np.asarray(fits) - fo) / np.abs(fo)))
    fac_err = max(float(np.abs(a - b).max() / np.abs(b).max()) for a, b in zip(U, Uo))
    t_bits = t.alto_bits
    t.close()
    cpu = None
    if not args.no_cpu_baseline:
        try:
            L = O.ref_lib(64)
            threads = os.cpu_count() or 1
            L.ref_set_threads(threads)
            rt = O.RefTensor(dims, cidx, vals, threads, bits=64)
            Fr = [f.astype(np.float64) for f in F]
            sec = rt.mttkrp_time(0, Fr, R, 100)
            with stdout_to_stderr():
                ts = time.perf_counter()
                rt.cpd_als(U0, np.ones(R), R, iters, 1e-12)
                ref_cpd = time.perf_counter() - ts
            rt.close()
            cpu = {"value": nnz * R / sec, "unit": "nnz*R/s", "cores": threads, "kind": "reference",
                   "sample": "the whole tensor: 100 mode-0 mttkrp_alto_par calls",
                   "cpals_ms_per_iter": ref_cpd / iters * 1e3}
        except Exception as e:
            cpu = {"value": None, "unit": "nnz*R/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}
    peak, peak_kind = measured_peaks()
    b = mttkrp_bytes(CPALS3_DIMS, nnz, R, 0, t_bits)
    return {
        "metric": "CP-ALS ms/iteration; mode-0 MTTKRP nnz*R/s (rank 16)", "value": nnz * R / (mt_ms / 1e3),
        "unit": "nnz*R/s", "n_gpus": 1, "steps": 100, "warmup": 3, "ms_per_step": mt_ms, "higher_is_better": True,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "cpals3d-1000^3-1Mnnz-uniform-R16-it20", "dims": CPALS3_DIMS, "nnz": nnz, "rank": R,
                   "alto_bits": t_bits, "l2": "L2 flushed (256 MB write) before every timed MTTKRP"},
        "cpals": {"ms_per_iter": cpd_s / iters * 1e3, "iters": it, "final_fit": float(fits[-1]),
                  "api": "alto_cpd_als (float64 host model in and out)"},
        "error_vs_fp64": {"fit_max_rel_err": fit_err, "fit_bound": 1e-5, "factor_max_rel_err": fac_err,
                          "mttkrp_max_rel_err": mt_err, "mttkrp_bound": 1e-5,
                          "method": "the oracle's CP-ALS (float64) from the original values and initial model; "
                                    "MTTKRP against the oracle's with the same float32 factor values"},
        "roofline": {"bound": "hbm", "achieved": b / (mt_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": b / (mt_ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind, "traffic": None},
        "cpu_baseline": cpu,
        "gpu_launches": launches,
    }


def ours_cpals5d(args):
    """Rank-64 CP-ALS on the 5-mode tensor 100k x 100k x 10k x 1k x 100 with
    50,000,000 distinct nonzeros (modes 0-1 Zipf(1.1) with permuted labels,
    modes 2-4 uniform, values U(0,1)), generated on the device; once with
    float32 and once with bfloat16 factor storage (float32 accumulation,
    float64 Grams and Cholesky).  Per-mode MTTKRP GB/s for both storages,
    their error against float64 sums of sampled rows (bfloat16 against the
    float32 factor values before rounding), fits and time per iteration."""
    import numpy as np
    import torch

    import alto_b200 as A
    from alto_b200 import synth

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    R, iters = 64, args.steps if args.workload == "cpals5d" else 5
    N = len(CPALS5_DIMS)
    cidx, vals = synth.zipf_coo_device(CPALS5_DIMS, CPALS5_NNZ, CPALS5_ZIPF, seed=9, values="uniform", device=dev)
    t = A.AltoTensor(CPALS5_DIMS, cidx, vals, nprtn=1)
    nnz = t.nnz
    stream = torch.cuda.current_stream()
    g = torch.Generator(device=dev)
    g.manual_seed(17)
    F32 = [(torch.rand((d, R), generator=g, device=dev) * 2 - 1).contiguous() for d in CPALS5_DIMS]
    FB = [f.to(torch.bfloat16).contiguous() for f in F32]
    outs = [torch.empty((d, R), device=dev, dtype=torch.float32) for d in CPALS5_DIMS]
    peak, peak_kind = measured_peaks()
    launches0 = A.kernel_launches()
    res = {}
    for name, F, fb in (("f32", F32, 4), ("bf16", FB, 2)):
        t.autotune(F, R)
        per = []
        for m in range(N):
            for _ in range(2):
                t.mttkrp(m, F, R, out=outs[m], stream=stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(3):
                t.mttkrp(m, F, R, out=outs[m], stream=stream)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / 3
            b = mttkrp_bytes(CPALS5_DIMS, nnz, R, m, t.alto_bits, fbytes=fb)
            per.append({"ms": round(ms, 4), "gbs": round(b / (ms / 1e3) / 1e9, 1),
                        "frac": round(b / (ms / 1e3) / 1e9 / peak, 4),
                        "variant": {A.ATOMIC: "atomic", A.STAGED: "staged", A.SORTED: "sorted"}.get(
                            t.choose_variant(m, R, A.BF16 if fb == 2 else A.F32), "other")})
        torch.cuda.synchronize()
        errs, _ = sampled_rows_error(cidx, vals, F32, outs, R, nrows=2048)
        res[name] = {"per_mode": per, "mttkrp_max_rel_err": max(errs), "mttkrp_err_per_mode": errs}
    launches = A.kernel_launches() - launches0
    del cidx, vals, F32, FB, outs
    torch.cuda.empty_cache()
    U0 = init_model(CPALS5_DIMS, R, 3)
    for name, storage in (("f32", A.F32), ("bf16", A.BF16)):
        A.cpd_alto(t, U0, np.ones(R), R, 1, 1e-12, storage=storage)  # warm
        ts = time.perf_counter()
        _, _, fits, it = A.cpd_alto(t, U0, np.ones(R), R, iters, 1e-12, storage=storage)
        res[name]["cpals_ms_per_iter"] = (time.perf_counter() - ts) / iters * 1e3
        res[name]["fits"] = [float(x) for x in fits]
    t.close()
    flops = nnz * R * N
    ms_all = sum(p["ms"] for p in res["f32"]["per_mode"])
    b_all = sum(mttkrp_bytes(CPALS5_DIMS, nnz, R, m, 65) for m in range(N))
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12  # TFLOP/s of FP32 FMA on CUDA cores at max clock
    return {
        "metric": "CP-ALS rank 64, per-mode MTTKRP GB/s (float32 and bfloat16 factor storage)",
        "value": b_all / (ms_all / 1e3) / 1e9, "unit": "GB/s", "n_gpus": 1, "steps": iters, "warmup": 1,
        "ms_per_step": res["f32"]["cpals_ms_per_iter"], "higher_is_better": True, "dtype": "f32/bf16+f64",
        "data": "synthetic",
        "config": {"workload": "cpals5d-100kx100kx10kx1kx100-50Mnnz-zipf1.1-R64", "dims": CPALS5_DIMS, "nnz": nnz,
                   "rank": R, "alto_bits": t.alto_bits, "iters": iters,
                   "l2": "line (1 GB) and factors exceed L2; no flush"},
        "storage": res,
        "error_vs_fp64": {"mttkrp_max_rel_err_f32": res["f32"]["mttkrp_max_rel_err"],
                          "mttkrp_max_rel_err_bf16": res["bf16"]["mttkrp_max_rel_err"],
                          "fit_rel_diff_bf16_vs_f32": abs(res["bf16"]["fits"][-1] - res["f32"]["fits"][-1])
                          / abs(res["f32"]["fits"][-1]),
                          "method": "sampled rows (2048 per mode + the heaviest) in float64 from the COO; "
                                    "bfloat16 against the float32 factor values before rounding. The CP-ALS "
                                    "fit against the FP64 oracle is tested at 2M nonzeros (tests/test_gpu_configs.py)"},
        "roofline": {"bound": "hbm", "achieved": b_all / (ms_all / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": b_all / (ms_all / 1e3) / 1e9 / peak, "peak_kind": peak_kind, "traffic": None,
                     "fp32_fma": {"achieved_tflops": flops * N / (ms_all / 1e3) / 1e12,
                                  "peak_tflops_nominal": fp32_peak}},
        "cpu_baseline": None,
        "gpu_launches": launches,
    }


def reference_cpals_arm(args):
    """--impl reference for cpals3d: the reference's CP-ALS (oracle/_ref,
    all host threads) on the same tensor; cpals5d: not run (its per-thread
    buffers at rank 64 and 50M nonzeros are outside a bounded run)."""
    import numpy as np

    import oracle as O
    from alto_b200 import synth

    rank, _, _ = dist_env()
    if rank != 0:
        return 0
    if args.workload == "cpals5d":
        print(json.dumps({"impl": "reference", "unavailable": "cpals5d is not timed on the reference (bounded runs only)"}))
        return 0
    try:
        dims = np.array(CPALS3_DIMS, np.uint64)
        cidx, vals = synth.uniform_coo(dims, CPALS3_NNZ, seed=55)
        R = 16
        L = O.ref_lib(64)
        threads = os.cpu_count() or 1
        L.ref_set_threads(threads)
        rt = O.RefTensor(dims, cidx, vals, threads, bits=64)
        rng = np.random.default_rng(5)
        F = [rng.uniform(-1, 1, (int(d), R)) for d in dims]
        sec = rt.mttkrp_time(0, F, R, max(args.steps, 1) * 5)
        rt.close()
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref could not run: {e}"}))
        return 0
    value = cidx.shape[1] * R / sec
    print(json.dumps({
        "impl": "reference", "metric": "CP-ALS ms/iteration; mode-0 MTTKRP nnz*R/s (rank 16)", "value": value,
        "unit": "nnz*R/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": 1, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "cpals3d-1000^3-1Mnnz-uniform-R16-it20"},
        "cpu_baseline": {"value": value, "unit": "nnz*R/s", "cores": threads, "kind": "reference",
                         "sample": "the whole tensor, mode-0 mttkrp_alto_par"},
        "e2e": {"value": value, "unit": "nnz*R/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


def config_lines(args):
    """The other workload configurations, one sub-object each, for the
    default one-GPU line: CP-ALS on 1000^3 (1M nonzeros, rank 16, 20
    iterations), rank-64 CP-ALS on the 5-mode tensor (50M nonzeros, float32
    and bfloat16 factor storage), CP-stream (the first 40 slices) and serving
    (64 streams)."""
    out = {}
    for name, fn, steps, warmup in (("cpals_1000cubed_1M_r16", ours_cpals3d, None, None),
                                    ("cpals_5mode_50M_r64", ours_cpals5d, None, None),
                                    ("cpstream", ours_cpstream, 37, 3),
                                    ("serve", ours_serve, 4, 1)):
        sub = argparse.Namespace(**vars(args))
        sub.workload = name
        if steps is not None:
            sub.steps, sub.warmup = steps, warmup
        try:
            out[name] = fn(sub)
        except Exception as e:  # one configuration failing must not hide the others
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        import torch

        torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    if args.workload == "tns":
        return reference_tns_arm(args) if args.impl == "reference" else ours_tns(args)
    if args.workload == "slice":
        return reference_slice_arm(args) if args.impl == "reference" else ours_slice(args)
    if args.workload in ("cpals3d", "cpals5d"):
        if args.impl == "reference":
            return reference_cpals_arm(args)
        line = ours_cpals3d(args) if args.workload == "cpals3d" else ours_cpals5d(args)
        print(json.dumps(line))
        return 0
    if args.workload != "mttkrp":
        if args.impl == "reference":
            return reference_stream_arm(args)
        line = ours_cpstream(args) if args.workload == "cpstream" else ours_serve(args)
        if line is not None:
            print(json.dumps(line))
        return 0
    if args.impl == "reference":
        return reference_arm(args)
    line = ours(args)
    if line is not None:
        if line["n_gpus"] == 1 and not (args.profile_small or args.no_configs):
            line["configs"] = config_lines(args)
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
