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
import platform
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


def max_over_ranks(x: float, world: int, device) -> float:
    """The largest x over the job's ranks (for times: the slowest rank sets the
    job's time); x itself on one rank."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank: int, world: int, seconds_max: float) -> float:
    """Whole-job units per second when every rank processes units_per_rank in
    at most seconds_max (the max over ranks)."""
    return world * units_per_rank / seconds_max


def run_reference(args, rank, world):
    """CPU restatement of the reference path (the AVX2 port of its x86 NTT
    kernels, oracle/oracle_avx2.c) on this host's cores."""
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
        P.ntt_mul_inverse(a[:1024], b[:1024], threads=threads, avx2=True)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        P.ntt_mul_inverse(a, b, threads=threads, avx2=True)
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
                         "sample": f"{sample} polys of the {n_full}-poly workload per step "
                                   "(AVX2 restatement of the reference's x86 path)",
                         "host": host_cpu()},
        "e2e": {"value": value, "unit": "polys/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def host_cpu():
    """This host's CPU model and logical core count, recorded beside CPU timings."""
    model = platform.processor() or "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count() or 1}


def cpu_baseline(q, d, n_full):
    """Single-thread AVX2 port of the reference's x86 path on a bounded sample
    (the reference CPU path is single-threaded)."""
    from oracle import oracle as O
    P = O.Plan(q, d)
    rng = np.random.default_rng(2)
    sample = 1 << 14
    a = rng.integers(0, q, (sample, d), dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, q, (sample, d), dtype=np.uint64).astype(np.uint32)
    P.ntt_mul_inverse(a[:256], b[:256], avx2=True)
    reps, elapsed = 0, 0.0
    while elapsed < 10.0 and reps < 64:
        t0 = time.perf_counter()
        P.ntt_mul_inverse(a, b, avx2=True)
        elapsed += time.perf_counter() - t0
        reps += 1
    return {"value": sample * reps / elapsed, "unit": "polys/s", "cores": 1, "kind": "port",
            "sample": f"{reps} x {sample} polys of the {n_full}-poly workload, 1 thread "
                      "(AVX2 restatement of the reference's x86 path)",
            "host": host_cpu()}


def _mont_words(q, values):
    """Signed integers -> PrimeField<q, u32> Montgomery words (host numpy)."""
    v = np.asarray(values, dtype=np.int64) % q
    return ((v.astype(object) << 32) % q).astype(np.uint64).astype(np.uint32)


def _events_ms(fn, n, stream):
    import torch
    times = []
    for _ in range(n):
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        fn()
        s1.record(stream)
        s1.synchronize()
        times.append(s0.elapsed_time(s1))
    return times


def _pct(xs, p):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(round(p / 100.0 * (len(xs) - 1))))]


def measure_commit_plain(dev, reps=50):
    """Plain Ajtai commit: A = 8 x 64 ring matrix (d = 64, q = 4294966657)
    expanded from a ChaCha20 seed (ChaCha20Rng, the reference's
    sample_uniform_mat rule), 64 witnesses of 64 ternary polys; t = A s per
    witness."""
    import ctypes as C
    import torch
    from lattica_b200 import TwistedNttPlan, _lib
    from lattica_b200.commit import PreparedMatrix
    from lattica_b200.labrador import sample_uniform_polys
    q, d, rows, cols, batch = Q64, 64, 8, 64, 64
    lib = _lib.load()
    plan = TwistedNttPlan(q, d)
    rng = np.random.default_rng(11)
    A = sample_uniform_polys(plan, bytes(range(100, 132)), rows * cols).reshape(rows, cols, d)
    s_host = _mont_words(q, rng.integers(-1, 2, (batch, cols, d))).reshape(batch, cols, d)
    M = PreparedMatrix(plan, A, rows, cols)
    s = torch.from_numpy(s_host.view(np.int32)).to(dev)
    t = torch.empty((batch, rows, d), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    ws_b = M.workspace_bytes(batch)
    ws = torch.empty(max(16, ws_b), dtype=torch.uint8, device=dev)
    ws1 = torch.empty(max(16, M.workspace_bytes(1)), dtype=torch.uint8, device=dev)

    def batched():
        st = lib.grid_gpu_commit_dev(M.handle, s.data_ptr(), batch, t.data_ptr(), ws.data_ptr(),
                                     ws.numel(), stream.cuda_stream)
        assert st == 0

    def per_call():  # one C-ABI call per commitment
        for i in range(batch):
            st = lib.grid_gpu_commit_dev(M.handle, s[i].data_ptr(), 1, t[i].data_ptr(),
                                         ws1.data_ptr(), ws1.numel(), stream.cuda_stream)
            assert st == 0

    for _ in range(5):
        batched()
        per_call()
    tb = _events_ms(batched, reps, stream)
    tp = _events_ms(per_call, max(5, reps // 5), stream)
    # steady state: batches back to back between two events, so the GPU does
    # not idle while the host prepares each call (the per-call times above
    # include that launch latency)
    steady_n = 200
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(steady_n):
        batched()
    s1.record(stream)
    s1.synchronize()
    steady_ms = s0.elapsed_time(s1) / steady_n
    # device throughput: 50 batches captured once in a CUDA graph and replayed,
    # so the host's per-call cost is out of the timed region
    graph_ms = None
    try:
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            cap = torch.cuda.current_stream(dev).cuda_stream
            for _ in range(50):
                assert lib.grid_gpu_commit_dev(M.handle, s.data_ptr(), batch, t.data_ptr(),
                                               ws.data_ptr(), ws.numel(), cap) == 0
        graph.replay()
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(4):
            graph.replay()
        g1.record(stream)
        g1.synchronize()
        graph_ms = g0.elapsed_time(g1) / 200
        del graph
    except Exception as exc:  # a capture failure leaves the other figures intact
        print(f"config 0 graph timing skipped: {exc}", file=sys.stderr)
    hs = torch.from_numpy(s_host.view(np.int32).copy()).pin_memory()
    ht = torch.empty((batch, rows, d), dtype=torch.int32).pin_memory()
    e2e = []
    for i in range(reps + 3):
        t0 = time.perf_counter()
        st = lib.grid_gpu_commit(M.handle, hs.data_ptr(), batch, ht.data_ptr())
        assert st == 0
        if i >= 3:
            e2e.append((time.perf_counter() - t0) * 1e3)
    med_b, med_p, med_e = statistics.median(tb), statistics.median(tp), statistics.median(e2e)
    # CPU beside it: the prepared commit path with A_hat cached (linear.rs:717-742),
    # through the AVX2 restatement of the reference's x86 kernels, on the same
    # inputs, one thread and all host cores
    from oracle import oracle as O
    P = O.Plan(q, d)
    a_hat = P.forward(np.ascontiguousarray(A).reshape(rows * cols, d)).reshape(-1)
    cpu = {}
    for label, threads in (("1t", 1), ("all", os.cpu_count() or 1)):
        want = P.matvec(a_hat, rows, cols, s_host, batch, a_is_eval=True, threads=threads,
                        avx2=True)  # warm
        t0 = time.perf_counter()
        for _ in range(3):
            P.matvec(a_hat, rows, cols, s_host, batch, a_is_eval=True, threads=threads,
                     avx2=True)
        cpu[label] = batch * 3 / (time.perf_counter() - t0)
    assert np.array_equal(t.cpu().numpy().view(np.uint32).reshape(-1), want), "GPU != oracle"
    return {"workload": "plain Ajtai commit: A 8x64 from a ChaCha20 seed, d=64, 64 ternary "
                        "witnesses per batch",
            "cpu_oracle_commits_per_s": {"threads_1": cpu["1t"], "threads_all": cpu["all"],
                                         "cores": os.cpu_count() or 1,
                                         "kind": "AVX2 port, A_hat cached"},
            "commits_per_s": batch / (med_b / 1e3), "batch_ms_p50": med_b,
            "commits_per_s_steady": batch / (steady_ms / 1e3), "batch_ms_steady": steady_ms,
            "commits_per_s_graph": batch / (graph_ms / 1e3) if graph_ms else None,
            "batch_ms_graph": graph_ms,
            "per_call_commits_per_s": batch / (med_p / 1e3),
            "e2e_commits_per_s": batch / (med_e / 1e3), "e2e_batch_ms_p50": med_e,
            "e2e_h2d_bytes": s_host.nbytes, "e2e_d2h_bytes": batch * rows * d * 4}


def measure_round(dev, reps=50):
    """LaBRADOR prover round on one instance: r = 64 witness vectors of
    n = 2048 polys (d = 64, coefficients in [-2^11, 2^11]); inner commitments by
    a 16 x 2048 matrix + base-2^8 balanced limbs (4), the r x r Gram (upper
    triangle) + limbs, the 256-row JL projection."""
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import CommitKey, prover_round_dev
    q, d, r, n, kappa = Q64, 64, 64, 2048, 16
    plan = TwistedNttPlan(q, d)
    g = torch.Generator(device=dev).manual_seed(5)
    A = torch.randint(0, q, (kappa, n, d), dtype=torch.int64, device=dev, generator=g).to(torch.int32)
    key = CommitKey(plan, A, kappa, n)
    coeffs = torch.randint(-2048, 2049, (r, n, d), dtype=torch.int64, device=dev, generator=g) % q
    wit = ((coeffs * ((1 << 32) % q)) % q).to(torch.int32)  # Montgomery words x * 2^32 mod q
    del coeffs
    seed = bytes(range(32))
    stream = torch.cuda.current_stream(dev)
    ws = None
    for _ in range(3):
        out = prover_round_dev(key, wit, 256, 4, 256, 4, seed, 256)
    torch.cuda.synchronize()
    times = _events_ms(lambda: prover_round_dev(key, wit, 256, 4, 256, 4, seed, 256), reps, stream)
    times_x = _events_ms(lambda: prover_round_dev(key, wit, 256, 4, 256, 4, seed, 256, extract=True),
                         max(5, reps // 5), stream)
    # the round plus the 256 conjugated JL evaluations prove_step aggregates
    # later; p is read from their coefficient 0 (one keystream pass)
    prover_round_dev(key, wit, 256, 4, 256, 4, seed, 256, jl_evals=True)
    times_ev_round = _events_ms(
        lambda: prover_round_dev(key, wit, 256, 4, 256, 4, seed, 256, jl_evals=True),
        max(5, reps // 5), stream)
    # end to end: witness from pinned host memory, outputs back to the host
    hw = wit.cpu().pin_memory()
    outs_host = None
    e2e = []
    for i in range(reps + 2):
        t0 = time.perf_counter()
        dw = hw.to(dev, non_blocking=True)
        o = prover_round_dev(key, dw, 256, 4, 256, 4, seed, 256)
        outs_host = [x.to("cpu", non_blocking=True) for x in (o.t_limbs, o.g, o.g_limbs, o.p)]
        torch.cuda.synchronize()
        if i >= 2:
            e2e.append((time.perf_counter() - t0) * 1e3)
    d2h = sum(x.numel() * x.element_size() for x in outs_host)
    # CPU beside it: the oracle's round pieces (inner commitments, Gram, JL
    # projection) at n = 128 polys per witness part, scaled by n / 128 (each
    # piece is linear in n), on one thread and on all host cores
    from oracle import oracle as O
    P = O.Plan(q, d)
    ns = 128
    A_h = A[:, :ns].contiguous().cpu().numpy().view(np.uint32)
    S_h = wit[:, :ns].contiguous().cpu().numpy().view(np.uint32)
    cpu_round = {}
    for label, threads in (("threads_1", 1), ("threads_all", os.cpu_count() or 1)):
        t0 = time.perf_counter()
        P.matvec(A_h, kappa, ns, S_h, r, threads=threads)
        P.gram(S_h, r, ns, threads=threads)
        O.jl_project(P.field, seed, 256, S_h.reshape(r, ns * d), r, ns * d, d, want_flat=False,
                     threads=threads)
        cpu_round[label] = (time.perf_counter() - t0) * 1e3 * (n / ns)
    cpu_round["cores"] = os.cpu_count() or 1
    cpu_round["sample"] = f"n = {ns} of {n} polys per part, scaled x{n // ns}"
    # the round's neighbours at the same size: garbage h (aggregated phis of
    # the witness shape) and the amortized witness z = sum_i c_i s_i
    from lattica_b200.labrador import amortize_witness, compute_garbage_h
    phis = torch.randint(0, q, (r, n, d), dtype=torch.int64, device=dev, generator=g).to(torch.int32)
    chal = torch.randint(0, q, (r, d), dtype=torch.int64, device=dev, generator=g).to(torch.int32)
    for _ in range(3):
        compute_garbage_h(plan, wit, phis)
        amortize_witness(plan, wit, chal)
    torch.cuda.synchronize()
    times_h = _events_ms(lambda: compute_garbage_h(plan, wit, phis), max(5, reps // 5), stream)
    times_z = _events_ms(lambda: amortize_witness(plan, wit, chal), max(5, reps // 5), stream)
    del phis
    # outer commitments of the round's limbs (kappa1 = kappa2 = 16): u1 = B t + C g
    # over t (r * 4 * kappa = 4096 polys) and g (4 * 2080 = 8320), u2 = D h (8320)
    from lattica_b200.commit import BdlopCommitmentKey
    from lattica_b200.labrador import OuterCommitKey
    k1, t_len, g_len = 16, r * 4 * kappa, 4 * (r * (r + 1) // 2)
    rnd = lambda *shape: torch.randint(0, q, shape, dtype=torch.int64, device=dev,
                                       generator=g).to(torch.int32)
    outer = OuterCommitKey(plan, rnd(k1, t_len, d), rnd(k1, g_len, d), rnd(k1, g_len, d), k1, k1,
                           t_len, g_len, g_len)
    tv, gv = rnd(t_len, d), rnd(g_len, d)
    times_u1 = _events_ms(lambda: outer.outer_commit_u1_slice(tv, gv), max(5, reps // 5), stream)
    times_u2 = _events_ms(lambda: outer.outer_commit_u2_slice(gv), max(5, reps // 5), stream)
    del outer
    # BDLOP parts at the plain-commit shape: 8 x 64 matrices, a batch of 64
    bd = BdlopCommitmentKey(plan, rnd(8, 64, d), rnd(8, 64, d), rnd(8, 64, d), 8, 64, 64)
    bm, br = rnd(64, 64, d), rnd(64, 64, d)
    times_bd = _events_ms(lambda: bd.recompute_parts(bm, br), max(5, reps // 5), stream)
    # aggregation-side JL evaluations of the round's witness, from the keystream
    from lattica_b200.labrador import JLMatrix
    jlm = JLMatrix(seed, 256, n * d)
    wflat = wit.reshape(r, n * d)
    jlm.conjugated_evals(plan, wflat, r, d)
    times_ev = _events_ms(lambda: jlm.conjugated_evals(plan, wflat, r, d), max(5, reps // 5), stream)
    # the round's commitment key expanded from a seed on the device (A, B, C, D:
    # kappa = kappa1 = kappa2 = 16, t1 = t2 = 4; 364544 polys)
    from lattica_b200.labrador import sample_uniform_polys
    crs_polys = kappa * n + 16 * (r * 4 * kappa) + 2 * 16 * (4 * (r * (r + 1) // 2))
    sample_uniform_polys(plan, seed, crs_polys, device=dev)
    times_crs = _events_ms(lambda: sample_uniform_polys(plan, seed, crs_polys, device=dev),
                           max(5, reps // 5), stream)
    parity = check_round_parity(key, A, wit, seed, plan)
    return {"workload": "LaBRADOR round: r=64, n=2048, d=64, kappa=16, JL 256 rows, base 2^8 x4 limbs",
            "round_ms_p50": _pct(times, 50), "round_ms_p99": _pct(times, 99),
            "parity": parity,
            "cpu_oracle_round_ms": cpu_round,
            "garbage_h_ms_p50": _pct(times_h, 50), "amortize_ms_p50": _pct(times_z, 50),
            "outer_u1_ms_p50": _pct(times_u1, 50), "outer_u2_ms_p50": _pct(times_u2, 50),
            "bdlop_batch64_ms_p50": _pct(times_bd, 50),
            "jl_evals_ms_p50": _pct(times_ev, 50),
            "crs_expand_ms_p50": _pct(times_crs, 50),
            "round_with_jl_extraction_ms_p50": _pct(times_x, 50),
            "round_with_jl_evals_ms_p50": _pct(times_ev_round, 50),
            "e2e_round_ms_p50": _pct(e2e, 50), "e2e_round_ms_p99": _pct(e2e, 99),
            "e2e_h2d_bytes": hw.numel() * 4, "e2e_d2h_bytes": d2h, "rounds": reps}


def check_round_parity(key, A, wit, seed, plan):
    """One round on the timed inputs, every output word compared with the
    oracle at the round's own size (r = 64, n = 2048, kappa = 16): t limbs,
    g, g limbs and the JL projection p. Raises on any difference."""
    import torch
    from lattica_b200.labrador import prover_round_dev
    from oracle import oracle as O
    r, n, d = (int(x) for x in wit.shape)
    kappa = int(A.shape[0])
    o = prover_round_dev(key, wit, 256, 4, 256, 4, seed, 256)
    torch.cuda.synchronize()
    got = {k: getattr(o, k).cpu().numpy().view(np.uint32).reshape(-1)
           for k in ("t_limbs", "g", "g_limbs", "p")}
    P = O.Plan(plan.q, d)
    F = P.field
    S = wit.cpu().numpy().view(np.uint32)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    t = P.matvec(A.cpu().numpy().view(np.uint32), kappa, n, S, r, threads=threads)
    g = P.gram(S, r, n, threads=threads)
    p, _ = O.jl_project(F, seed, 256, S.reshape(r, n * d), r, n * d, d, want_flat=False,
                        threads=threads)
    want = {"t_limbs": O.decompose_polys(F, d, t, 256, 4), "g": g,
            "g_limbs": O.decompose_polys(F, d, g, 256, 4), "p": p}
    for k, w in want.items():
        if not np.array_equal(got[k], w.reshape(-1)):
            raise AssertionError(f"round {k}: {int(np.count_nonzero(got[k] != w.reshape(-1)))} "
                                 "words differ from the oracle")
    return {"checked": "every word of t_limbs, g, g_limbs, p vs the oracle",
            "words": int(sum(v.size for v in got.values())),
            "oracle_s": round(time.perf_counter() - t0, 2)}


def measure_batch(dev, reps=10):
    """Uneven batched commits: 4096 instances, n log-uniform in [64, 8192],
    rank m uniform in {8, 16, 32}, d = 64, ternary witnesses; one m x 8192
    matrix per rank shared by its instances (instance uses the first n
    columns). Batched (one CUDA-graph replay) vs one commit call per instance."""
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.batch import UnevenCommitBatch, per_call_commit, sample_uneven_instances
    from lattica_b200.commit import PreparedMatrix
    q, d, ranks = Q64, 64, (8, 16, 32)
    plan = TwistedNttPlan(q, d)
    g = torch.Generator(device=dev).manual_seed(3)
    mats, mats_host = [], []
    for m in ranks:
        A = torch.randint(0, q, (m, 8192, d), dtype=torch.int64, device=dev, generator=g).to(torch.int32)
        mats.append(PreparedMatrix(plan, A, m, 8192))
        mats_host.append(A.cpu().numpy().view(np.uint32))
        del A
    items, s_polys, t_polys = sample_uneven_instances(4096, 7)
    r1 = (1 << 32) % q
    tern = torch.randint(-1, 2, (s_polys, d), dtype=torch.int64, device=dev, generator=g) % q
    s = ((tern * r1) % q).to(torch.int32)
    del tern
    t = torch.zeros((t_polys, d), dtype=torch.int32, device=dev)
    batch = UnevenCommitBatch(plan, mats, items)
    tune = batch.autotune(s, t)
    side = torch.cuda.Stream(dev)
    with torch.cuda.stream(side):
        batch.commit_dev(s, t, graph=True, stream=side)
        side.synchronize()
        tb = _events_ms(lambda: batch.commit_dev(s, t, graph=True, stream=side), reps, side)
    t2 = torch.zeros_like(t)
    per_call_commit(plan, mats, items, s, t2)
    stream = torch.cuda.current_stream(dev)
    tp = _events_ms(lambda: per_call_commit(plan, mats, items, s, t2), 3, stream)
    same = bool(torch.equal(t, t2))
    if not same:
        raise AssertionError("batched commits differ from the per-call path")
    # 32 instances (the longest, the shortest and 30 spread over the batch)
    # against the oracle
    from oracle import oracle as O
    P = O.Plan(q, d)
    order = sorted(range(len(items)), key=lambda i: items[i][2])
    pick = sorted(set([order[-1], order[0]] + order[:: max(1, len(order) // 30)][:30]))
    for i in pick:
        so, to, nn, m = items[i]
        rows = ranks[m]
        A_i = np.ascontiguousarray(mats_host[m][:, :nn, :])
        sw = s[so:so + nn].cpu().numpy().view(np.uint32)
        want = P.matvec(A_i, rows, nn, sw, 1).reshape(rows, d)
        if not np.array_equal(t[to:to + rows].cpu().numpy().view(np.uint32), want):
            raise AssertionError(f"batched commit of instance {i} (n={nn}, m={rows}) differs "
                                 "from the oracle")
    n = len(items)
    macs = sum(ranks[m] * nn for _, _, nn, m in items) * d
    return {"workload": "uneven batched commits: 4096 instances, n log-uniform [64, 8192], "
                        "m in {8,16,32}, d=64",
            "batched_commits_per_s": n / (statistics.median(tb) / 1e3),
            "batched_ms_p50": statistics.median(tb),
            "per_call_commits_per_s": n / (statistics.median(tp) / 1e3),
            "per_call_ms_p50": statistics.median(tp),
            "speedup_vs_per_call": statistics.median(tp) / statistics.median(tb),
            "outputs_identical": same, "mod_macs": macs,
            "parity": f"all outputs equal the per-call path; {len(pick)} instances "
                      "(longest and shortest included) equal the oracle",
            "autotune": {k: v for k, v in tune.items()
                         if k in ("schedule", "engine", "tile_instances", "k_split", "cached",
                                  "ms")},
            "schedule": batch.config()}


def measure_serve(dev, rates=(1000, 2000, 5000, 10000, 20000, 50000), seconds=0.4):
    """Served mixed stream, open-loop Poisson arrivals: 70% commits (n
    log-uniform [64, 4096], m in {8, 16, 32}), 25% Gram + JL steps (r in
    {8, 16, 32, 64}, n = 1024), 5% LaBRADOR rounds (r = 64, n = 2048,
    kappa = 16); d = 64. Continuous batching over 4 streams vs the plain
    per-call path (one request at a time), at each offered rate; latency from
    scheduled arrival to the result on the host."""
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.commit import PreparedMatrix
    from lattica_b200.labrador import CommitKey
    from lattica_b200.serve import RingServer, sample_requests, run_load
    q, d = Q64, 64
    plan = TwistedNttPlan(q, d)
    g = torch.Generator(device=dev).manual_seed(9)
    mats = {}
    for m in (8, 16, 32):
        A = torch.randint(0, q, (m, 4096, d), dtype=torch.int64, device=dev, generator=g)
        mats[m] = PreparedMatrix(plan, A.to(torch.int32), m, 4096)
        del A
    A = torch.randint(0, q, (16, 2048, d), dtype=torch.int64, device=dev, generator=g)
    key = CommitKey(plan, A.to(torch.int32), 16, 2048)
    del A
    arena, pool_polys = 1 << 18, 1 << 19
    coeffs = torch.randint(-2048, 2049, (pool_polys, d), dtype=torch.int64, device=dev, generator=g)
    pool = (((coeffs % q) * ((1 << 32) % q)) % q).to(torch.int32)
    del coeffs
    torch.cuda.synchronize()

    def schedule(seed, count, rate):
        out = sample_requests(seed, count, rate, commit_arena=arena, pool_polys=pool_polys)
        for _, r in out:
            r.keep = False
        return out

    out = {"workload": "served stream: 70% commits n~logU[64,4096] m in {8,16,32}; 25% Gram+JL "
                       "r in {8,16,32,64} n=1024; 5% LaBRADOR rounds r=64 n=2048; d=64; "
                       f"Poisson arrivals, {seconds} s of arrivals per rate",
           "rates": {}}
    for mode in ("continuous", "plain"):
        with RingServer(plan, mats, key, pool, mode=mode) as srv:
            # warm-up at a sparse and a dense rate: the first sparse-traffic
            # requests of a process pay a one-time host-side cost (tens of ms)
            # that dense traffic does not trigger
            run_load(srv, schedule(2, 200, 1000.0))
            run_load(srv, schedule(1, 300, 3000.0))
            for lam in rates:
                res = run_load(srv, schedule(100 + lam, max(200, int(lam * seconds)), float(lam)))
                out["rates"].setdefault(str(lam), {})[mode] = res
        # capacity: the whole stream queued at once, so throughput is what the
        # server sustains rather than the offered rate
        with RingServer(plan, mats, key, pool, mode=mode) as srv:
            run_load(srv, schedule(2, 200, 1000.0))
            out.setdefault("saturated", {})[mode] = run_load(srv, schedule(55, 600, 1e9))
    best = {m: max(v[m]["commits_per_s"] for v in out["rates"].values())
            for m in ("continuous", "plain")}
    out["max_commits_per_s"] = best
    out["commits_per_s_ratio"] = best["continuous"] / best["plain"]
    sat = out["saturated"]
    out["saturated_req_per_s_ratio"] = sat["continuous"]["req_per_s"] / sat["plain"]["req_per_s"]
    out["saturated_commits_per_s_ratio"] = (sat["continuous"]["commits_per_s"]
                                            / sat["plain"]["commits_per_s"])
    out["parity"] = check_serve_parity(plan, mats, key, pool, arena, pool_polys)
    return out


def check_serve_parity(plan, mats, key, pool, arena, pool_polys, count=300, rate=20000.0):
    """Every result of a mixed stream served continuously (batched, overlapped)
    equals the same request served alone (the plain per-call path). Raises on
    any difference."""
    from lattica_b200.serve import RingServer, run_load, sample_requests
    results = {}
    for mode in ("continuous", "plain"):
        sched = sample_requests(777, count, rate, commit_arena=arena, pool_polys=pool_polys)
        with RingServer(plan, mats, key, pool, mode=mode) as srv:
            run_load(srv, sched)
        results[mode] = [(r.kind, r.future.result()) for _, r in sched]
    kinds = {}
    for (k, a), (_, b) in zip(results["continuous"], results["plain"]):
        if len(a) != len(b) or not all(np.array_equal(x, y) for x, y in zip(a, b)):
            raise AssertionError(f"a served {k} request differs from the same request alone")
        kinds[k] = kinds.get(k, 0) + 1
    return {"checked": f"{count} requests at {int(rate)} req/s: continuous == alone",
            "by_kind": kinds}


def measure_ring_round(dev, reps=20):
    """The LaBRADOR round at r = 64, n = 2048, kappa = 16 over the reference's own
    LaBRADOR modulus q = 2^32 - 5, which has no 128th root of unity (the
    reference multiplies by the schoolbook rule there): ring plan through three
    auxiliary NTT primes. t limbs, g and p are checked against the oracle's
    schoolbook products."""
    import torch
    from lattica_b200.labrador import CommitKey, prover_round_dev
    from lattica_b200.ntt import RingPlan
    from oracle import oracle as O
    q, d, r, n, kappa = 4294967291, 64, 64, 2048, 16
    plan = RingPlan(q, d)
    g = torch.Generator(device=dev).manual_seed(6)
    A = torch.randint(0, q, (kappa, n, d), dtype=torch.int64, device=dev, generator=g)
    coeffs = torch.randint(-2048, 2049, (r, n, d), dtype=torch.int64, device=dev, generator=g) % q
    wit = ((coeffs * ((1 << 32) % q)) % q).to(torch.int32)
    A = A.to(torch.int32)
    del coeffs
    key = CommitKey(plan, A, kappa, n)
    seed = bytes(range(32))
    stream = torch.cuda.current_stream(dev)
    for _ in range(3):
        o = prover_round_dev(key, wit, 256, 4, 256, 4, seed, 256)
    torch.cuda.synchronize()
    times = _events_ms(lambda: prover_round_dev(key, wit, 256, 4, 256, 4, seed, 256), reps, stream)
    F = O.Field(q)
    S = wit.cpu().numpy().view(np.uint32)
    t0 = time.perf_counter()
    t = F.ring_matvec(d, A.cpu().numpy().view(np.uint32), kappa, n, S, r)
    gram = F.ring_gram(d, S, r, n)
    p, _ = O.jl_project(F, seed, 256, S.reshape(r, n * d), r, n * d, d, want_flat=False)
    oracle_s = time.perf_counter() - t0
    host = lambda x: x.cpu().numpy().view(np.uint32).reshape(-1)
    if not (np.array_equal(host(o.t_limbs), O.decompose_polys(F, d, t, 256, 4))
            and np.array_equal(host(o.g), gram) and np.array_equal(host(o.p), p)):
        raise AssertionError("ring-plan round differs from the oracle's schoolbook products")
    return {"workload": "LaBRADOR round r=64 n=2048 kappa=16 at q=2^32-5 (no NTT: three "
                        "auxiliary primes, exact reconstruction)",
            "round_ms_p50": _pct(times, 50), "round_ms_p99": _pct(times, 99),
            "oracle_schoolbook_s": round(oracle_s, 2), "oracle_cores": os.cpu_count() or 1,
            "parity": "t limbs, g, p bit-exact vs the oracle's schoolbook products"}


def measure_ntt64_transforms(dev, reps=20):
    """The batched transforms alone (config 1's 2^22 polys at d = 64, in place):
    forward and inverse each read and write 256 B per poly, 2 GiB per call
    (inputs > L2). Checked: the inverse returns the input (every word), and 16
    sampled polys of the forward equal the oracle's."""
    import torch
    from lattica_b200 import TwistedNttPlan, _lib
    q, d, n = WORKLOADS["ntt64"]
    plan = TwistedNttPlan(q, d)
    lib = _lib.load()
    g = torch.Generator(device=dev).manual_seed(64)
    x = torch.randint(0, q, (n, d), dtype=torch.int64, device=dev, generator=g).to(torch.int32)
    x0 = x.clone()
    stream = torch.cuda.current_stream(dev)
    fwd = lambda: lib.grid_gpu_ntt_forward_dev(plan.handle, x.data_ptr(), n, stream.cuda_stream)
    inv = lambda: lib.grid_gpu_ntt_inverse_dev(plan.handle, x.data_ptr(), n, stream.cuda_stream)
    # parity: one forward against the oracle on sampled polys, then the round trip
    if fwd() or inv():
        raise RuntimeError("transform launch failed")
    torch.cuda.synchronize()
    if not torch.equal(x, x0):
        raise AssertionError("forward then inverse does not return the input")
    from oracle import oracle as O
    rows = torch.linspace(0, n - 1, 16, dtype=torch.int64, device=dev)
    want = O.Plan(q, d).forward(x0[rows].cpu().numpy().view(np.uint32))
    if fwd():
        raise RuntimeError("transform launch failed")
    torch.cuda.synchronize()
    if not np.array_equal(x[rows].cpu().numpy().view(np.uint32), want.reshape(16, d)):
        raise AssertionError("forward transform differs from the oracle")
    if inv():
        raise RuntimeError("transform launch failed")
    peak, _ = _peaks()
    out = {}
    for name, f in (("forward", fwd), ("inverse", inv)):
        for _ in range(3):
            f()
        ms = statistics.median(_events_ms(f, reps, stream))
        out[name] = {"ms_p50": ms, "polys_per_s": n / (ms / 1e3),
                     "frac": 2 * 4 * d * n / (ms / 1e3) / 1e9 / peak}
    torch.cuda.synchronize()
    return out


def measure_ntt256(dev, reps=20):
    """The d = 256 sweep of the batched products: 2^20 polys at q' = 4294962689."""
    import torch
    from lattica_b200 import TwistedNttPlan, _lib
    q, d, n = WORKLOADS["ntt256"]
    plan = TwistedNttPlan(q, d)
    lib = _lib.load()
    g = torch.Generator(device=dev).manual_seed(256)
    a = torch.randint(0, q, (n, d), dtype=torch.int64, device=dev, generator=g).to(torch.int32)
    b = torch.randint(0, q, (n, d), dtype=torch.int64, device=dev, generator=g).to(torch.int32)
    out = torch.empty_like(a)
    stream = torch.cuda.current_stream(dev)

    def step():
        assert lib.grid_gpu_ntt_mul_inverse_dev(plan.handle, a.data_ptr(), b.data_ptr(),
                                                out.data_ptr(), n, stream.cuda_stream) == 0

    for _ in range(3):
        step()
    ms = statistics.median(_events_ms(step, reps, stream))
    peak, _ = _peaks()
    return {"polys_per_s": n / (ms / 1e3), "ms_p50": ms,
            "frac": 3 * 4 * d * n / (ms / 1e3) / 1e9 / peak}


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
    elapsed_ms = max_over_ranks(elapsed_ms, world, dev)
    ms_per_step = elapsed_ms / args.steps
    value = replica_throughput(n, world, ms_per_step / 1e3)

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
    e2e_s = max_over_ranks(e2e_s, world, dev)
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
        "e2e": {"value": replica_throughput(n, world, e2e_s), "unit": "polys/s",
                "h2d_bytes_per_step": 2 * 4 * d * n, "d2h_bytes_per_step": 4 * d * n},
        "gpu_launches": args.steps,
        "clocks": sampler.summary(),
    }
    if world == 1:
        line["cpu_baseline"] = cpu_baseline(q, d, WORKLOADS[args.workload][2])
    if args.secondary:
        detail = {"commit": measure_commit_plain(dev), "round": measure_round(dev),
                  "batch": measure_batch(dev), "ntt256": measure_ntt256(dev),
                  "ntt64_transforms": measure_ntt64_transforms(dev),
                  "ring_round": measure_ring_round(dev)}
        if args.serve:
            detail["serve"] = measure_serve(dev)
        line["secondary"] = secondary_summary(detail)
        path = os.environ.get("BENCH_DETAIL", os.path.join(ROOT, "gpurun_out",
                                                           "bench_detail.json"))
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as fh:
                json.dump(detail, fh, indent=1)
            line["secondary"]["detail_file"] = os.path.relpath(path, ROOT)
        except OSError as exc:
            print(f"bench detail not written: {exc}", file=sys.stderr)
    print(json.dumps(line), flush=True)


def secondary_summary(detail):
    """The figures BASELINE's metric names, flat and short (the JSON line stays
    a few KB): config 0 commits/s, the round's p50/p99, config 3 batched
    commits/s, the served ratios, the d = 256 sweep; each checked in the run."""
    def r(x, nd=3):
        return None if x is None else round(float(x), nd)
    c, rd, b, n2 = detail["commit"], detail["round"], detail["batch"], detail["ntt256"]
    out = {
        "round_ms_p50": r(rd["round_ms_p50"], 4), "round_ms_p99": r(rd["round_ms_p99"], 4),
        "round_e2e_ms_p50": r(rd["e2e_round_ms_p50"]),
        "round_parity": "bit-exact, every word at r=64 n=2048 kappa=16",
        "round_cpu_oracle_ms_1t": r(rd["cpu_oracle_round_ms"]["threads_1"], 1),
        "round_cpu_oracle_ms_all": r(rd["cpu_oracle_round_ms"]["threads_all"], 1),
        "config0_commits_per_s": r(c["commits_per_s"], 0),
        "config0_commits_per_s_graph": r(c["commits_per_s_graph"], 0),
        "config0_per_call_commits_per_s": r(c["per_call_commits_per_s"], 0),
        "config0_e2e_commits_per_s": r(c["e2e_commits_per_s"], 0),
        "config0_cpu_commits_per_s_1t": r(c["cpu_oracle_commits_per_s"]["threads_1"], 0),
        "config0_parity": "bit-exact vs oracle",
        "config3_commits_per_s": r(b["batched_commits_per_s"], 0),
        "config3_per_call_commits_per_s": r(b["per_call_commits_per_s"], 0),
        "config3_ms_p50": r(b["batched_ms_p50"]),
        "config3_parity": "all == per-call; 32 sampled == oracle",
        "ntt256_polys_per_s": r(n2["polys_per_s"], 0), "ntt256_frac": r(n2["frac"]),
        "ntt64_forward_frac": r(detail["ntt64_transforms"]["forward"]["frac"]),
        "ntt64_inverse_frac": r(detail["ntt64_transforms"]["inverse"]["frac"]),
        "round_q_2e32m5_ms_p50": r(detail["ring_round"]["round_ms_p50"], 4),
        "host_cores": os.cpu_count() or 1,
    }
    sv = detail.get("serve")
    if sv:
        sat = sv["saturated"]
        out.update({
            "served_commits_per_s_ratio": r(sv["commits_per_s_ratio"]),
            "served_req_per_s_ratio": r(sv["saturated_req_per_s_ratio"]),
            "served_saturated_req_per_s": {m: sat[m]["req_per_s"] for m in sat},
            "served_saturated_p99_ms": {m: sat[m]["p99_ms"] for m in sat},
            "served_p99_ms_at_5k": {m: sv["rates"]["5000"][m]["p99_ms"]
                                    for m in ("continuous", "plain")},
            "served_parity": "continuous == alone, 300 mixed requests",
        })
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="ntt64")
    ap.add_argument("--no-secondary", dest="secondary", action="store_false",
                    help="skip the plain-commit and prover-round measurements")
    ap.add_argument("--no-serve", dest="serve", action="store_false",
                    help="skip the served-stream measurement")
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
