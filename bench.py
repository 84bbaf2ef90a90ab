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

Multi-GPU (torchrun, one rank per GPU): every rank owns its own tensor of the
same size (independent tensors, weak scaling); no data-path collective.

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
# bounded CPU sample: every mode keeps nnz/dims <= 4, so the reference runs
# its atomic variant (no per-thread da_mem buffers of whole-mode size)
CPU_SAMPLE_NNZ = 7_000_000
METRIC = "MTTKRP nnz*R/s (all-mode, rank 32)"
WORKLOAD = "powerlaw3d-4.8Mx1.8Mx1.8M-140Mnnz-zipf1.2-R32-allmode"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nnz", type=int, default=NNZ)
    ap.add_argument("--rank", type=int, default=RANK)
    ap.add_argument("--cpu-sample", type=int, default=CPU_SAMPLE_NNZ)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--factor-dtype", choices=["f32", "bf16"], default="f32",
                    help="factor storage (bf16 halves gather bytes; accumulation stays f32)")
    ap.add_argument("--profile-small", action="store_true",
                    help="small tensor (for ncu captures): 20M nonzeros, 1 step")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def line_bytes_per_nnz(alto_bits):
    key = 8 if alto_bits <= 64 else (12 if alto_bits <= 96 else 16)
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


def cpu_sample(n, rank, seed=2024):
    """The bounded host sample of the workload's distribution."""
    import numpy as np

    from alto_b200 import synth

    cidx, vals = synth.powerlaw_coo(DIMS, n, ZIPF, seed=seed, values="lognormal")
    rng = np.random.default_rng(seed + 1)
    F = [rng.uniform(-1.0, 1.0, (d, rank)) for d in DIMS]
    return cidx, vals, F


def time_reference_cpu(n, rank, reps):
    """Seconds per all-mode step of the reference's mttkrp_alto_par (OpenMP,
    all host threads) on an n-nonzero sample; returns (sec, threads, nnz)."""
    import numpy as np  # noqa: F401

    import oracle as O

    L = O.ref_lib(128)
    threads = os.cpu_count() or 1
    L.ref_set_threads(threads)
    cidx, vals, F = cpu_sample(n, rank)
    t = O.RefTensor(DIMS, cidx, vals, threads, bits=128)
    sec = t.mttkrp_time(-1, F, rank, reps)
    nnz = t.nnz
    t.close()
    return sec, threads, nnz


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    try:
        sec, threads, nnz = time_reference_cpu(args.cpu_sample, args.rank, max(args.steps, 1))
    except Exception as e:  # the checker library is missing or failed to load
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref could not run: {e}"}))
        return 0
    units = nnz * args.rank * len(DIMS)
    value = units / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "nnz*R/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": 1, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_nnz": nnz, "dims": DIMS, "rank": args.rank,
                   "note": "bounded sample of the same distribution (full tensor does not fit the "
                           "reference's per-thread buffers on this host)"},
        "cpu_baseline": {"value": value, "unit": "nnz*R/s", "cores": threads, "kind": "reference",
                         "sample": f"{nnz} nonzeros of the workload distribution, all-mode MTTKRP"},
        "e2e": {"value": value, "unit": "nnz*R/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


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

    cidx, vals = synth.zipf_coo_device(DIMS, nnz, ZIPF, seed=1234 + rank, values="lognormal", device=dev)
    t = A.AltoTensor(DIMS, cidx, vals, nprtn=1)
    nnz = t.nnz
    del cidx, vals
    torch.cuda.empty_cache()
    g = torch.Generator(device=dev)
    g.manual_seed(99 + rank)
    fdt = torch.bfloat16 if args.factor_dtype == "bf16" else torch.float32
    factors = [(torch.rand((d, R), generator=g, device=dev) * 2 - 1).to(fdt).contiguous() for d in DIMS]
    outs = [torch.empty((d, R), device=dev, dtype=torch.float32) for d in DIMS]
    stream = torch.cuda.current_stream()
    variants = t.autotune(factors, R)  # project autotuner: fastest kernel variant per mode
    vnames = {A.ATOMIC: "atomic", A.STAGED: "staged", A.STREAM: "stream", A.SORTED: "sorted"}

    def step(ev=None):
        for m in range(N):
            outs[m].zero_()
            if ev is not None:
                ev[m][0].record(stream)
            t.mttkrp(m, factors, R, out=outs[m], accumulate=True, stream=stream)
            if ev is not None:
                ev[m][1].record(stream)

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
    t0.record(stream)
    for k in range(steps):
        step(events[k])
    t1.record(stream)
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
    units = nnz * R * N * steps * world
    value = units / elapsed

    # roofline of the MTTKRP kernel (per-mode launches, CUDA events on its stream)
    alto_bits = t.alto_bits
    per_mode = []
    for m in range(N):
        dt = statistics.mean(events[k][m][0].elapsed_time(events[k][m][1]) / 1e3 for k in range(steps))
        b = mttkrp_bytes(DIMS, nnz, R, m, alto_bits, fbytes=2 if args.factor_dtype == "bf16" else 4)
        per_mode.append((m, dt, b))
    bytes_launch = sum(b for _, _, b in per_mode) / N
    dt_launch = sum(dt for _, dt, _ in per_mode) / N
    achieved = bytes_launch / dt_launch / 1e9
    peak, peak_kind = measured_peaks()
    traffic = recorded_traffic()

    # end to end through the host-buffer C-ABI entry point
    e2e = None
    if not args.no_e2e:
        hostF = [torch.empty((d, R), dtype=torch.float64, pin_memory=True) for d in DIMS]
        for h, f in zip(hostF, factors):
            h.copy_(f.float().double().cpu())
        hostN = [h.numpy() for h in hostF]
        t.mttkrp_host(0, hostN, R)  # warm
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ts = time.perf_counter()
        for _ in range(args.e2e_steps):
            for m in range(N):
                t.mttkrp_host(m, hostN, R)
        te = time.perf_counter() - ts
        if world > 1:
            x = torch.tensor([te], device=dev, dtype=torch.float64)
            torch.distributed.all_reduce(x, op=torch.distributed.ReduceOp.MAX)
            te = float(x.item())
        h2d = sum(N * d * R * 8 for d in DIMS)
        d2h = sum(d * R * 8 for d in DIMS)
        e2e = {"value": nnz * R * N * args.e2e_steps * world / te, "unit": "nnz*R/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": te / args.e2e_steps * 1e3,
               "api": "alto_mttkrp_host (float64 host factors, pinned)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.profile_small:
        try:
            sec, threads, snnz = time_reference_cpu(args.cpu_sample, R, 3)
            cpu = {"value": snnz * R * N / sec, "unit": "nnz*R/s", "cores": threads, "kind": "reference",
                   "sample": f"{snnz} nonzeros of the same distribution, all-mode MTTKRP, 3 reps"}
        except Exception as e:
            cpu = {"value": None, "unit": "nnz*R/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "nnz*R/s", "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": elapsed / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "dims": DIMS, "nnz": nnz, "rank": R, "zipf": 1.2,
                       "values": "lognormal(0,1)", "key_bits": t.key_bits, "alto_bits": alto_bits,
                       "factor_dtype": args.factor_dtype, "parallelism": f"independent tensor per GPU x{world}",
                       "l2": "inputs larger than L2 (line + factors > 3 GB); no flush",
                       "line_bytes_per_nnz": line_bytes_per_nnz(alto_bits),
                       "variants": [vnames.get(v, str(v)) for v in variants],
                       "device_bytes": t.device_bytes()},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic.get("bytes_per_launch") if traffic else None,
                         "per_mode_ms": [round(dt * 1e3, 4) for _, dt, _ in per_mode],
                         "algorithmic_bytes_per_mode": [b for _, _, b in per_mode]},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clocks,
            "gpu_launches": launches,
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    t.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
