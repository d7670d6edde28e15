#!/usr/bin/env python
"""Benchmark of the B200 ring-arithmetic hot path.

Default workload (one "step"): the batched twisted negacyclic pipeline
out = INTT(NTT(a) (.) b) over 2^22 polynomials of degree d = 64, uint32
Montgomery words mod q = 4294966657, inputs resident in HBM (3 GiB per step,
larger than the 126 MB L2, so no explicit flush is needed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ntt64|ntt256]

Under torchrun (N > 1) every rank runs an independent replica (the path has no
exchange step); the step time is the max over ranks. `--impl reference` times
the CPU restatement of the reference algorithm (the oracle port) on this host's
cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

Q64 = 4294966657     # largest prime < 2^32 with q = 1 mod 128
Q256 = 4294962689    # largest prime < 2^32 with q = 1 mod 512 (d = 256 needs a 512th root)
METRIC = "ring products/s (batched twisted NTT -> Montgomery pointwise -> INTT)"

WORKLOADS = {
    # name: (q, d, npolys)
    "ntt64": (Q64, 64, 1 << 22),
    "ntt256": (Q256, 256, 1 << 20),
}


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic(kernel_key):
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as fh:
            return json.load(fh).get(kernel_key)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]
        return False

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


def run_reference(args, rank, world):
    """CPU restatement of the reference path on this host's cores."""
    if rank != 0:
        return
    from oracle import oracle as O
    q, d, n_full = WORKLOADS[args.workload]
    threads = os.cpu_count() or 1
    sample = 1 << 15
    P = O.Plan(q, d)
    rng = np.random.default_rng(1)
    a = rng.integers(0, q, (sample, d), dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, q, (sample, d), dtype=np.uint64).astype(np.uint32)
    for _ in range(max(1, args.warmup)):
        P.ntt_mul_inverse(a[:1024], b[:1024], threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        P.ntt_mul_inverse(a, b, threads=threads)
        times.append(time.perf_counter() - t0)
    per_step = sum(times) / len(times)
    value = sample / per_step
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "polys/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded uniform mod q)",
        "config": {"workload": f"{args.workload}: q={q}, d={d}, {n_full} polys (sampled)",
                   "sample_polys": sample},
        "cpu_baseline": {"value": value, "unit": "polys/s", "cores": threads, "kind": "port",
                         "sample": f"{sample} polys of the {n_full}-poly workload per step"},
        "e2e": {"value": value, "unit": "polys/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(q, d, n_full):
    """Single-thread oracle port on a bounded sample (the reference CPU path is single-threaded)."""
    from oracle import oracle as O
    P = O.Plan(q, d)
    rng = np.random.default_rng(2)
    sample = 1 << 14
    a = rng.integers(0, q, (sample, d), dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, q, (sample, d), dtype=np.uint64).astype(np.uint32)
    P.ntt_mul_inverse(a[:256], b[:256])
    reps, elapsed = 0, 0.0
    while elapsed < 10.0 and reps < 64:
        t0 = time.perf_counter()
        P.ntt_mul_inverse(a, b)
        elapsed += time.perf_counter() - t0
        reps += 1
    return {"value": sample * reps / elapsed, "unit": "polys/s", "cores": 1, "kind": "port",
            "sample": f"{reps} x {sample} polys of the {n_full}-poly workload, 1 thread"}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from lattica_b200 import TwistedNttPlan, _lib

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    q, d, n = WORKLOADS[args.workload]
    if args.polys:
        n = args.polys
    plan = TwistedNttPlan(q, d)
    lib = _lib.load()

    g = torch.Generator(device=dev).manual_seed(1234 + rank)
    a = torch.randint(0, q, (n, d), dtype=torch.int64, device=dev, generator=g).to(torch.int32)
    b = torch.randint(0, q, (n, d), dtype=torch.int64, device=dev, generator=g).to(torch.int32)
    out = torch.empty_like(a)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    def step():
        st = lib.grid_gpu_ntt_mul_inverse_dev(plan.handle, a.data_ptr(), b.data_ptr(),
                                              out.data_ptr(), n, sptr)
        if st:
            raise RuntimeError(f"kernel launch failed: {st}")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local_rank)
    with sampler:
        time.sleep(0.3)
        t_begin = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_begin.record(stream)
        for i in range(args.steps):
            starts[i].record(stream)
            step()
            ends[i].record(stream)
        t_end.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    plan.check_device()
    elapsed_ms = t_begin.elapsed_time(t_end)
    kernel_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / args.steps
    if world > 1:
        t = torch.tensor([elapsed_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    ms_per_step = elapsed_ms / args.steps
    value = world * n / (ms_per_step / 1e3)

    # End-to-end through the host-buffer C-ABI call: pinned host inputs copied
    # in, computed, result copied out, every step.
    ha = a.cpu().pin_memory()
    hb = b.cpu().pin_memory()
    hout = torch.empty_like(ha).pin_memory()
    e2e_steps = max(3, min(10, args.steps))

    def e2e_step():
        st = lib.grid_gpu_ntt_mul_inverse(plan.handle, ha.data_ptr(), hb.data_ptr(),
                                          hout.data_ptr(), n)
        if st:
            raise RuntimeError(f"host-buffer call failed: {st}")

    e2e_step()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    assert torch.equal(hout, out.cpu()), "host-buffer path disagrees with the device path"

    if rank != 0:
        return
    peak, peak_kind = _peaks()
    bytes_per_launch = 3 * 4 * d * n
    achieved = bytes_per_launch / (kernel_ms / 1e3) / 1e9
    traffic = _traffic(f"{args.workload}_mulinv")
    if args.polys:
        traffic = None
    line = {
        "metric": METRIC, "value": value, "unit": "polys/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded uniform mod q, generated on device)",
        "config": {"workload": f"{args.workload}: out = INTT(NTT(a) * b), q={q}, d={d}, "
                               f"{n} polys per GPU",
                   "polys_per_gpu": n, "q": q, "d": d, "l2": "inputs 3 GiB > L2, no flush",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                     "algorithmic_bytes_per_launch": bytes_per_launch,
                     "kernel_ms": kernel_ms},
        "e2e": {"value": world * n / e2e_s, "unit": "polys/s",
                "h2d_bytes_per_step": 2 * 4 * d * n, "d2h_bytes_per_step": 4 * d * n},
        "gpu_launches": args.steps,
        "clocks": sampler.summary(),
    }
    if world == 1:
        line["cpu_baseline"] = cpu_baseline(q, d, WORKLOADS[args.workload][2])
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="ntt64")
    ap.add_argument("--polys", type=int, default=0,
                    help="override the polynomial count (smaller cases for profiling)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
