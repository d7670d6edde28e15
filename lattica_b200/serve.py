"""Continuous-batching request server for the ring-arithmetic hot path.

Requests: single Ajtai commitments (t = A_m[:, :n] s, rank m, length n), Gram
+ JL prover steps (the r x r Gram of a witness and its 256-row JL projection)
and full LaBRADOR prover rounds (commitments + limbs, Gram + limbs, JL). The
public matrices are expanded once and stay resident on the device; witnesses
are per-request device state, slices of a resident witness pool, as for a
prover whose previous level ran on the GPU. Commit witnesses come from an
arena that hands out consecutive slices in arrival order (wrapping at its
end), so a run of queued commitments reads one contiguous span.

Continuous mode: a scheduler thread admits waiting requests whenever a stream
slot and device-memory budget are free. All waiting commitments (up to
`max_batch`, within the budget) are packed into one batched launch sequence
(grid_gpu_batch_commit_oneshot_dev); all waiting Gram + JL requests (up to
`max_gram_batch`) share one batched Gram launch sequence
(grid_gpu_batch_gram_dev) and then run their JL projections on the same slot;
round requests each take a slot of their own. Slots are separate CUDA streams, so work admitted while
other work is on the GPU overlaps with it. Plain mode is the per-call
baseline: one request at a time, in arrival order, through the
one-call-per-request C-ABI entry points, waiting for each to finish.

Results come back to the host through pinned buffers as numpy uint32 arrays;
each request's result is identical whether it runs alone or in a mix.
"""
from __future__ import annotations

import collections
import ctypes as C
import math
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .ntt import raise_status

JL_ROWS = 256
KINDS = ("commit", "gramjl", "round")


@dataclass
class Request:
    kind: str                 # "commit" | "gramjl" | "round"
    offset: int               # witness start, in polys of the pool
    shape: tuple              # commit: (m, n); gramjl / round: (r, n)
    t_arrival: float = 0.0
    t_done: float = 0.0
    keep: bool = True         # False: the result is copied to the host, then released
    future: Future = field(default_factory=Future)


@dataclass
class _Job:
    requests: list
    event: object
    outputs: list             # per request: list of pinned host tensors
    footprint: int
    keepalive: list           # device tensors referenced by in-flight work


class RingServer:
    """commit_mats: {rank m: PreparedMatrix (m x n_max)}; round_key: a
    labrador.CommitKey whose shape fixes the round requests' n; pool: CUDA
    int32 tensor (polys, d) of witness words."""

    def __init__(self, plan, commit_mats: dict, round_key, pool, mode: str = "continuous",
                 streams: int = 4, commit_slots: int = 2, hbm_budget: int = 8 << 30,
                 k_split: int = 0, max_batch: int = 4096, max_gram_batch: int = 32,
                 jl_seed: bytes = bytes(range(32)), round_limbs=(256, 4, 256, 4)):
        import torch
        if mode not in ("continuous", "plain"):
            raise ValueError("mode must be 'continuous' or 'plain'")
        self._torch = torch
        self._lib = _lib.load()
        self.plan = plan
        self.d = plan.d
        self.mode = mode
        self.commit_mats = dict(commit_mats)
        ranks = sorted(self.commit_mats)
        self._mat_index = {m: i for i, m in enumerate(ranks)}
        self._mat_handles = (C.c_void_p * len(ranks))(
            *[self.commit_mats[m].handle.value for m in ranks])
        self.round_key = round_key
        self.pool = pool
        self.device = pool.device
        self.k_split = k_split
        self.max_batch = max_batch
        self.max_gram_batch = max_gram_batch
        self.jl_seed = bytes(jl_seed)
        self._seed_c = (C.c_uint8 * 32).from_buffer_copy(self.jl_seed)
        self.round_limbs = round_limbs
        # Slots [0, nc) carry commit batches on high-priority streams, so their
        # blocks are scheduled ahead of a long Gram / JL / round launch's
        # remaining blocks; the other slots carry one heavy request each.
        if mode == "plain":
            self._streams = [torch.cuda.Stream(self.device)]
            self._slot_class = ["any"]
        else:
            nslots = max(2, streams)
            nc = max(1, min(commit_slots, nslots - 1))
            self._streams = ([torch.cuda.Stream(self.device, priority=-1) for _ in range(nc)] +
                             [torch.cuda.Stream(self.device) for _ in range(nslots - nc)])
            self._slot_class = ["commit"] * nc + ["heavy"] * (nslots - nc)
        self._free = {c: [i for i, k in enumerate(self._slot_class) if k == c]
                      for c in set(self._slot_class)}
        self._inflight = {}                           # slot -> _Job (scheduler thread only)
        self._budget_left = hbm_budget
        self._queues = {k: collections.deque() for k in KINDS}
        self._cv = threading.Condition()
        self._stop = False
        self._views = {}                              # (m, n) -> matrix view (plain commits)
        self._error = None
        self.batches = 0                              # commit launch sequences issued
        self._thread = threading.Thread(target=self._loop, name="ring-server", daemon=True)

    # ---------------------------------------------------------------- public
    def start(self, prime: bool = True):
        if prime:
            self.prime()
        self._thread.start()
        return self

    def prime(self, gram_r: int = 64, gram_n: int = 1024, round_r: int = 64):
        """Runs one request of each kind, at its largest shape, on every stream
        that can carry it, and waits. Each stream's memory pool then holds the
        blocks its requests need, and every kernel is loaded. Without this, the
        first round or Gram on a stream grows the pool in the middle of the
        traffic, and a device-synchronising allocation stalls the work already
        in flight on the other streams."""
        torch = self._torch
        polys = self.pool.shape[0]
        m = max(self.commit_mats)
        shapes = {"commit": (m, min(self.commit_mats[m].cols, polys)),
                  "gramjl": (gram_r, gram_n),
                  "round": (round_r, self.round_key.n)}
        for slot, cls in enumerate(self._slot_class):
            kinds = {"commit": ("commit",), "heavy": ("gramjl", "round")}.get(cls, KINDS)
            jobs = []
            for kind in kinds:
                a, b = shapes[kind]
                if kind != "commit":
                    a = min(a, polys // b)  # r witness vectors of n polys from the pool
                if a < 1 or b > polys:
                    continue
                req = Request(kind, 0, (a, b), keep=False)
                jobs.append(self._run(kind, [req], self._streams[slot], 0))
            for job in jobs:
                job.event.synchronize()
        torch.cuda.synchronize(self.device)

    def stop(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        self._thread.join()
        for h in self._views.values():
            self._lib.grid_gpu_matrix_destroy(h)
        self._views.clear()
        if self._error is not None:
            raise self._error

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.stop()

    def submit(self, req: Request) -> Future:
        if req.kind not in self._queues:
            raise ValueError(f"unknown request kind {req.kind!r}")
        if req.t_arrival == 0.0:
            req.t_arrival = time.perf_counter()
        with self._cv:
            if self._stop:
                raise RuntimeError("server is stopped")
            self._queues[req.kind].append(req)
            self._cv.notify()
        return req.future

    # ------------------------------------------------------------ scheduling
    def _loop(self):
        self._torch.cuda.set_device(self.device)
        picks = []
        try:
            while True:
                self._retire()
                with self._cv:
                    if self._stop and not self._inflight and not any(self._queues.values()):
                        return
                    picks = self._pick()
                    if not picks:
                        self._cv.wait(timeout=0.00005 if self._inflight else 0.001)
                        continue
                while picks:
                    slot, kind, reqs, fp = picks[0]
                    job = self._run(kind, reqs, self._streams[slot], fp)
                    picks.pop(0)
                    self._inflight[slot] = job
                    if self.mode == "plain":
                        job.event.synchronize()
        except BaseException as exc:  # hand scheduler failures to every waiter
            self._error = exc
            with self._cv:
                self._stop = True
                pending = [r for q in self._queues.values() for r in q]
                for q in self._queues.values():
                    q.clear()
            pending += [r for job in self._inflight.values() for r in job.requests]
            pending += [r for pick in picks for r in pick[2]]
            for r in pending:
                if not r.future.done():
                    r.future.set_exception(exc)

    def _retire(self):
        for slot in [s for s, job in self._inflight.items() if job.event.query()]:
            job = self._inflight.pop(slot)
            now = time.perf_counter()
            for req, outs in zip(job.requests, job.outputs):
                req.t_done = now
                res = [o.numpy().view(np.uint32) for o in outs]
                req.future.set_result(res if req.keep else None)
            self._free[self._slot_class[slot]].append(slot)
            self._budget_left += job.footprint

    def _pick(self):
        """With the queue lock held: choose (slot, kind, requests, bytes) to launch."""
        picks = []
        if self.mode == "plain":
            heads = [q[0] for q in self._queues.values() if q]
            if self._free["any"] and heads:
                head = min(heads, key=lambda r: r.t_arrival)
                self._queues[head.kind].popleft()
                picks.append((self._free["any"].pop(), head.kind, [head], 0))
            return picks
        for kind in KINDS:
            q = self._queues[kind]
            free = self._free["commit" if kind == "commit" else "heavy"]
            limit = {"commit": self.max_batch, "gramjl": self.max_gram_batch}.get(kind, 1)
            while q and free:
                reqs, fp = [], 0
                while q and len(reqs) < limit:
                    f = self._footprint(q[0])
                    if fp + f > self._budget_left and (reqs or self._inflight or picks):
                        break                   # admit only what fits the budget
                    reqs.append(q.popleft())
                    fp += f
                if not reqs:
                    break
                self._budget_left -= fp
                picks.append((free.pop(), kind, reqs, fp))
        return picks

    def _footprint(self, req: Request) -> int:
        """Device bytes a request holds while in flight (workspace + outputs)."""
        d = self.d
        if req.kind == "commit":
            m, n = req.shape
            return n * d * 4 + m * d * 12 + 256
        r, n = req.shape
        g = r * (r + 1) // 2 * d * 4
        base = r * n * d * 4 + g * 2 + 4 * JL_ROWS * 8 + 65536
        if req.kind == "gramjl":
            return base
        kappa = self.round_key.kappa
        b1, t1, b2, t2 = self.round_limbs
        return base + r * kappa * d * 4 * (2 + t1) + g * t2

    # ---------------------------------------------------------------- jobs
    def _run(self, kind, reqs, stream, fp):
        torch = self._torch
        with torch.cuda.stream(stream):
            if kind == "commit":
                if self.mode == "continuous":
                    return self._commit_batch(reqs, stream, fp)
                return self._commit_one(reqs[0], stream)
            if kind == "gramjl":
                if self.mode == "continuous":
                    return self._gramjl_batch(reqs, stream, fp)
                return self._gramjl(reqs[0], stream, fp)
            return self._round(reqs[0], stream, fp)

    def _pin(self, dev_tensor):
        host = self._torch.empty(dev_tensor.shape, dtype=dev_tensor.dtype, pin_memory=True)
        host.copy_(dev_tensor, non_blocking=True)
        return host

    def _finish(self, reqs, outputs, footprint, keepalive, stream):
        ev = self._torch.cuda.Event()
        ev.record(stream)
        return _Job(reqs, ev, outputs, footprint, keepalive)

    @staticmethod
    def _runs(reqs, gap: int = 1024):
        """Split requests into runs of nearby witness offsets (indices into reqs)."""
        order = sorted(range(len(reqs)), key=lambda i: reqs[i].offset)
        runs, cur, end = [], [], None
        for i in order:
            r = reqs[i]
            if cur and r.offset > end + gap:
                runs.append(cur)
                cur, end = [], None
            cur.append(i)
            e = r.offset + r.shape[1]
            end = e if end is None else max(end, e)
        if cur:
            runs.append(cur)
        return runs

    def _commit_batch(self, reqs, stream, fp):
        torch = self._torch
        lib = self._lib
        d = self.d
        t_offsets, t_total = [], 0
        for r in reqs:
            t_offsets.append(t_total)
            t_total += r.shape[0]
        t = torch.empty((t_total, d), dtype=torch.int32, device=self.device)
        calls, ws_need = [], 0
        for run in self._runs(reqs):
            lo = min(reqs[i].offset for i in run)
            items = (_lib.BatchItem * len(run))()
            for j, i in enumerate(run):
                m, n = reqs[i].shape
                items[j] = _lib.BatchItem(reqs[i].offset - lo, t_offsets[i], n,
                                          self._mat_index[m])
            nb = C.c_size_t()
            raise_status(lib.grid_gpu_batch_oneshot_workspace(
                self.plan.handle, self._mat_handles, len(self._mat_index), items, len(run),
                self.k_split, C.byref(nb)), "grid_gpu_batch_oneshot_workspace")
            ws_need = max(ws_need, nb.value)
            calls.append((lo, items, len(run)))
        ws = torch.empty(max(256, ws_need), dtype=torch.uint8, device=self.device)
        for lo, items, count in calls:
            raise_status(lib.grid_gpu_batch_commit_oneshot_dev(
                self.plan.handle, self._mat_handles, len(self._mat_index), items, count,
                self.k_split, self.pool.data_ptr() + lo * d * 4, t.data_ptr(), ws.data_ptr(),
                ws.numel(), stream.cuda_stream), "grid_gpu_batch_commit_oneshot_dev")
            self.batches += 1
        host = self._pin(t)
        outs = [[host[o:o + r.shape[0]]] for o, r in zip(t_offsets, reqs)]
        return self._finish(reqs, outs, fp, [ws, t], stream)

    def _view(self, m, n):
        key = (m, n)
        if key not in self._views:
            h = C.c_void_p()
            raise_status(self._lib.grid_gpu_matrix_view(self.commit_mats[m].handle, n,
                                                        C.byref(h)), "grid_gpu_matrix_view")
            self._views[key] = h
        return self._views[key]

    def _commit_one(self, req, stream):
        torch = self._torch
        m, n = req.shape
        view = self._view(m, n)
        nb = C.c_size_t()
        raise_status(self._lib.grid_gpu_commit_workspace(view, 1, C.byref(nb)),
                     "grid_gpu_commit_workspace")
        ws = torch.empty(max(256, nb.value), dtype=torch.uint8, device=self.device)
        t = torch.empty((m, self.d), dtype=torch.int32, device=self.device)
        s_ptr = self.pool.data_ptr() + req.offset * self.d * 4
        raise_status(self._lib.grid_gpu_commit_dev(view, s_ptr, 1, t.data_ptr(), ws.data_ptr(),
                                                   ws.numel(), stream.cuda_stream),
                     "grid_gpu_commit_dev")
        self.batches += 1
        return self._finish([req], [[self._pin(t)]], 0, [ws, t], stream)

    def _gramjl(self, req, stream, fp):
        torch = self._torch
        lib = self._lib
        r, n = req.shape
        d = self.d
        gw, jw = C.c_size_t(), C.c_size_t()
        raise_status(lib.grid_gpu_gram_workspace(self.plan.handle, r, n, C.byref(gw)),
                     "grid_gpu_gram_workspace")
        raise_status(lib.grid_gpu_jl_workspace(JL_ROWS, C.byref(jw)), "grid_gpu_jl_workspace")
        ws = torch.empty(max(256, gw.value), dtype=torch.uint8, device=self.device)
        jws = torch.empty(max(256, jw.value), dtype=torch.uint8, device=self.device)
        g = torch.empty((r * (r + 1) // 2, d), dtype=torch.int32, device=self.device)
        p = torch.empty(JL_ROWS, dtype=torch.int32, device=self.device)
        s_ptr = self.pool.data_ptr() + req.offset * d * 4
        raise_status(lib.grid_gpu_gram_dev(self.plan.handle, s_ptr, r, n, g.data_ptr(),
                                           ws.data_ptr(), ws.numel(), stream.cuda_stream),
                     "grid_gpu_gram_dev")
        raise_status(lib.grid_gpu_jl_project_dev(
            self.plan.handle, self._seed_c, JL_ROWS, s_ptr, r, n * d, d, p.data_ptr(), None,
            jws.data_ptr(), jws.numel(), stream.cuda_stream), "grid_gpu_jl_project_dev")
        return self._finish([req], [[self._pin(g), self._pin(p)]], fp, [ws, jws, g, p], stream)

    def _gramjl_batch(self, reqs, stream, fp):
        """All queued Gram + JL requests in one job: their Gram matrices in one
        batched launch sequence (grid_gpu_batch_gram_dev), then one JL
        projection per request on the same stream."""
        from .labrador import compute_garbage_g_batch, garbage_count
        torch = self._torch
        lib = self._lib
        d = self.d
        items = [(r.offset, r.shape[0], r.shape[1]) for r in reqs]
        G = compute_garbage_g_batch(self.plan, self.pool, items)
        jw = C.c_size_t()
        raise_status(lib.grid_gpu_jl_workspace(JL_ROWS, C.byref(jw)), "grid_gpu_jl_workspace")
        jws = torch.empty(max(256, jw.value), dtype=torch.uint8, device=self.device)
        p = torch.empty((len(reqs), JL_ROWS), dtype=torch.int32, device=self.device)
        for i, req in enumerate(reqs):
            r, n = req.shape
            s_ptr = self.pool.data_ptr() + req.offset * d * 4
            raise_status(lib.grid_gpu_jl_project_dev(
                self.plan.handle, self._seed_c, JL_ROWS, s_ptr, r, n * d, d, p[i].data_ptr(), None,
                jws.data_ptr(), jws.numel(), stream.cuda_stream), "grid_gpu_jl_project_dev")
        g_host, p_host = self._pin(G), self._pin(p)
        outs, g0 = [], 0
        for i, req in enumerate(reqs):
            cnt = garbage_count(req.shape[0])
            outs.append([g_host[g0:g0 + cnt], p_host[i]])
            g0 += cnt
        return self._finish(reqs, outs, fp, [G, jws, p], stream)

    def _round(self, req, stream, fp):
        from .labrador import prover_round_dev
        r, n = req.shape
        if n != self.round_key.n:
            raise ValueError("round request length does not match the commitment key")
        b1, t1, b2, t2 = self.round_limbs
        wit = self.pool[req.offset:req.offset + r * n].view(r, n, self.d)
        o = prover_round_dev(self.round_key, wit, b1, t1, b2, t2, self.jl_seed, JL_ROWS)
        hosts = [self._pin(x) for x in (o.t_limbs, o.g, o.g_limbs, o.p)]
        return self._finish([req], [hosts], fp, [o], stream)


# -------------------------------------------------------------------- load
def sample_requests(seed: int, count: int, rate: float, mix=(0.70, 0.25, 0.05),
                    commit_n=(64, 4096), ranks=(8, 16, 32), gram_r=(8, 16, 32, 64),
                    gram_n=1024, round_shape=(64, 2048), commit_arena=1 << 18,
                    pool_polys=1 << 19):
    """Open-loop Poisson arrivals at `rate` req/s of the mixed stream: commits
    (n log-uniform over commit_n, rank uniform over ranks), Gram + JL steps (r
    uniform over gram_r, n = gram_n) and full prover rounds (round_shape).
    Commit witnesses are consecutive slices of the arena [0, commit_arena);
    the others are random slices of [commit_arena, pool_polys).
    Returns [(arrival offset in seconds, Request)]."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, count)
    arrivals = np.cumsum(gaps) - gaps[0]
    kinds = rng.choice(3, count, p=list(mix))
    out, cursor = [], 0
    big = max(gram_n * max(gram_r), round_shape[0] * round_shape[1])
    if pool_polys - commit_arena < big or commit_arena < commit_n[1]:
        raise ValueError("pool too small for the request witnesses")
    for a, k in zip(arrivals.tolist(), kinds.tolist()):
        if k == 0:
            n = int(math.exp(rng.uniform(math.log(commit_n[0]), math.log(commit_n[1]))))
            n = min(max(n, commit_n[0]), commit_n[1])
            m = int(rng.choice(ranks))
            if cursor + n > commit_arena:
                cursor = 0
            req = Request("commit", cursor, (m, n))
            cursor += n
        elif k == 1:
            r = int(rng.choice(gram_r))
            off = int(rng.integers(commit_arena, pool_polys - r * gram_n + 1))
            req = Request("gramjl", off, (r, gram_n))
        else:
            r, n = round_shape
            off = int(rng.integers(commit_arena, pool_polys - r * n + 1))
            req = Request("round", off, (r, n))
        out.append((a, req))
    return out


def run_load(server: RingServer, schedule, timeout: float = 300.0) -> dict:
    """Replay `schedule` (from sample_requests) open loop against a started
    server; latency runs from each request's scheduled arrival to the moment
    its result is on the host."""
    reqs = []
    t0 = time.perf_counter()
    for offset, req in schedule:
        target = t0 + offset
        wait = target - time.perf_counter()
        if wait > 0:
            time.sleep(wait)          # sleeping (not spinning) leaves the GIL to the scheduler
        req.t_arrival = target
        server.submit(req)
        reqs.append(req)
    for r in reqs:
        r.future.result(timeout=timeout)
    span = max(r.t_done for r in reqs) - t0
    lat = np.array([(r.t_done - r.t_arrival) * 1e3 for r in reqs])
    by_kind = {}
    for kind in KINDS:
        sel = [r for r in reqs if r.kind == kind]
        if sel:
            ks = np.array([(r.t_done - r.t_arrival) * 1e3 for r in sel])
            kspan = max(r.t_done for r in sel) - t0
            by_kind[kind] = {"count": len(sel), "per_s": round(len(sel) / kspan, 1),
                             "p50_ms": round(float(np.percentile(ks, 50)), 3),
                             "p99_ms": round(float(np.percentile(ks, 99)), 3)}
    return {"requests": len(reqs), "seconds": round(span, 4),
            "req_per_s": round(len(reqs) / span, 1),
            "commits_per_s": by_kind.get("commit", {}).get("per_s", 0.0),
            "p50_ms": round(float(np.percentile(lat, 50)), 3),
            "p99_ms": round(float(np.percentile(lat, 99)), 3), "by_kind": by_kind}
