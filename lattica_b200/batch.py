"""Uneven batched commitments and their autotuner.

`UnevenCommitBatch` runs many Ajtai commitments t_i = A_{m_i}[:, :n_i] s_i of
different lengths n_i and matrices in one launch sequence (one NTT of all
witnesses, the persistent grouped evaluation-domain product on the tensor
cores, one INTT), optionally captured once into a CUDA graph and replayed. Its
schedule — the engine (tensor cores or CUDA cores), the instances per tile (the
tile shape: 32, 64 or 128 rows of the product) and the K range of a work item —
is picked by `autotune`, which times the candidates on the actual batch with
CUDA events and persists the winner in a JSON file keyed by the batch's shape
signature.

The per-call path (`per_call_commit`) issues one C-ABI commit per instance
through column views of the same prepared matrices; it is the plain GPU path
the batched form is compared against and must match word for word.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import math
import os

import numpy as np

from . import _lib
from .commit import PreparedMatrix
from .ntt import TwistedNttPlan, _stream_ptr, raise_status

K_SPLIT_CANDIDATES = (1024, 2048, 4096, 8192)
TILE_CANDIDATES = (0, 64, 32)  # instances per tile (0: the engine's largest, 128)
ENGINE_NAMES = {_lib.ENGINE_AUTO: "auto", _lib.ENGINE_TENSOR: "tensor",
                _lib.ENGINE_CUDA_CORE: "cuda_core", _lib.ENGINE_POINT_MAJOR: "point_major"}


def default_cache_path() -> str:
    return os.environ.get("GRID_GPU_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "lattica_b200",
                                       "autotune.json"))


class UnevenCommitBatch:
    """items: sequence of (s_offset, t_offset, n, matrix_index)."""

    def __init__(self, plan: TwistedNttPlan, matrices, items):
        self._lib = _lib.load()
        self.plan = plan
        self.matrices = list(matrices)
        arr = (_lib.BatchItem * len(items))()
        for i, (so, to, n, m) in enumerate(items):
            arr[i] = _lib.BatchItem(int(so), int(to), int(n), int(m))
        mats = (C.c_void_p * len(self.matrices))(*[m.handle.value for m in self.matrices])
        h = C.c_void_p()
        st = self._lib.grid_gpu_batch_create(plan.handle, mats, len(self.matrices), arr,
                                             len(items), C.byref(h))
        raise_status(st, "grid_gpu_batch_create")
        self._h = h
        self.items = [tuple(int(x) for x in it) for it in items]
        sp, tp = C.c_uint64(), C.c_uint64()
        raise_status(self._lib.grid_gpu_batch_shape(h, C.byref(sp), C.byref(tp)), "batch_shape")
        self.s_polys, self.t_polys = sp.value, tp.value
        nb = C.c_size_t()
        raise_status(self._lib.grid_gpu_batch_workspace(h, C.byref(nb)), "batch_workspace")
        self.workspace_bytes = nb.value
        self._ws = None

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.grid_gpu_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- schedule
    def config(self) -> dict:
        c = _lib.BatchConfig()
        raise_status(self._lib.grid_gpu_batch_get_config(self._h, C.byref(c)), "get_config")
        return {"k_split": c.k_split, "work_items": c.work_items, "tiles": c.tiles,
                "tile_instances": c.tile_instances, "engine": ENGINE_NAMES[c.engine],
                "tensor_cores": bool(c.tensor_cores)}

    def set_config(self, k_split: int, tile_instances: int = 0,
                   engine: int = _lib.ENGINE_AUTO) -> None:
        c = _lib.BatchConfig(int(k_split), 0, 0, int(tile_instances), int(engine), 0)
        raise_status(self._lib.grid_gpu_batch_set_config(self._h, C.byref(c)), "set_config")

    def set_k_split(self, k_split: int) -> None:
        cur = _lib.BatchConfig()
        raise_status(self._lib.grid_gpu_batch_get_config(self._h, C.byref(cur)), "get_config")
        self.set_config(k_split, cur.tile_instances, cur.engine)

    def signature(self) -> str:
        """Shape signature: matrix shapes plus a log2 histogram of lengths per matrix."""
        hist = {}
        for _, _, n, m in self.items:
            key = (m, int(math.log2(max(1, n))))
            hist[key] = hist.get(key, 0) + 1
        shapes = [(mm.rows, mm.cols) for mm in self.matrices]
        text = json.dumps({"d": self.plan.d, "mats": shapes,
                           "hist": sorted([list(k) + [v] for k, v in hist.items()])})
        return hashlib.sha256(text.encode()).hexdigest()[:24]

    # -- execution
    def _workspace(self, device):
        import torch
        if self._ws is None or self._ws.device != device:
            self._ws = torch.empty(max(16, self.workspace_bytes), dtype=torch.uint8, device=device)
        return self._ws

    def commit_dev(self, s, t, graph: bool = False, stream=None):
        """s: CUDA int32 tensor of >= s_polys * d words; t: >= t_polys * d words."""
        import torch
        ws = self._workspace(s.device)
        sp = stream.cuda_stream if stream is not None else _stream_ptr(s)
        fn = self._lib.grid_gpu_batch_commit_graph if graph else self._lib.grid_gpu_batch_commit_dev
        st = fn(self._h, s.data_ptr(), t.data_ptr(), ws.data_ptr(), ws.numel(), sp)
        raise_status(st, "grid_gpu_batch_commit")
        return t

    def schedules(self, k_splits=K_SPLIT_CANDIDATES):
        """Candidate schedules (k_split, tile_instances, engine): tile shapes on
        the tensor cores, and the CUDA-core kernel with its own tiles."""
        out = [(k, ti, _lib.ENGINE_TENSOR) for ti in TILE_CANDIDATES for k in k_splits]
        out += [(k, 0, _lib.ENGINE_CUDA_CORE) for k in k_splits]
        out += [(k, ti, _lib.ENGINE_POINT_MAJOR) for ti in TILE_CANDIDATES for k in k_splits]
        return out

    def autotune(self, s, t, candidates=None, reps: int = 3,
                 cache_path: str | None = None, use_cache: bool = True) -> dict:
        """Time each schedule candidate on this batch and keep the fastest.
        candidates: schedules (k_split, tile_instances, engine), or plain k_split
        values (the current tiles and engine); default: schedules()."""
        import torch
        path = cache_path or default_cache_path()
        sig = self.signature()
        cache = {}
        if use_cache and os.path.exists(path):
            try:
                with open(path) as fh:
                    cache = json.load(fh)
            except (OSError, ValueError):
                cache = {}
        if use_cache and sig in cache and "schedule" in cache[sig]:
            self.set_config(*cache[sig]["schedule"])
            return dict(cache[sig], cached=True)
        stream = torch.cuda.current_stream(s.device)
        cur = self.config()
        engine_now = {v: k for k, v in ENGINE_NAMES.items()}[cur["engine"]]
        if candidates is None:
            candidates = self.schedules()
        candidates = [tuple(c) if isinstance(c, (tuple, list))
                      else (int(c), cur["tile_instances"], engine_now) for c in candidates]
        results = {}
        for k in candidates:
            try:
                self.set_config(*k)
            except Exception:  # e.g. no tensor-core products on this plan
                continue
            self.commit_dev(s, t)
            times = []
            for _ in range(reps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                self.commit_dev(s, t)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
            results[k] = min(times)
        best = min(results, key=results.get)
        self.set_config(*best)
        entry = {"schedule": list(best), "k_split": best[0], "tile_instances": best[1],
                 "engine": ENGINE_NAMES[best[2]], "ms": results[best],
                 "candidates_ms": {"%d/%d/%s" % (k[0], k[1], ENGINE_NAMES[k[2]]): v
                                   for k, v in results.items()}}
        cache[sig] = entry
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as fh:
                json.dump(cache, fh, indent=1)
        except OSError:
            pass
        return dict(entry, cached=False)


def per_call_commit(plan: TwistedNttPlan, matrices, items, s, t, workspace=None):
    """One grid_gpu_commit_dev call per instance (column views of the matrices)."""
    import torch
    lib = _lib.load()
    d = plan.d
    views = {}
    max_ws = 0
    for _, _, n, m in items:
        if (m, n) not in views:
            h = C.c_void_p()
            raise_status(lib.grid_gpu_matrix_view(matrices[m].handle, n, C.byref(h)), "view")
            views[(m, n)] = h
            nb = C.c_size_t()
            lib.grid_gpu_commit_workspace(h, 1, C.byref(nb))
            max_ws = max(max_ws, nb.value)
    ws = workspace if workspace is not None else torch.empty(max(16, max_ws), dtype=torch.uint8,
                                                            device=s.device)
    sp = _stream_ptr(s)
    try:
        for so, to, n, m in items:
            st = lib.grid_gpu_commit_dev(views[(m, n)], s.data_ptr() + so * d * 4, 1,
                                         t.data_ptr() + to * d * 4, ws.data_ptr(), ws.numel(), sp)
            raise_status(st, "grid_gpu_commit_dev")
    finally:
        torch.cuda.current_stream(s.device).synchronize()
        for h in views.values():
            lib.grid_gpu_matrix_destroy(h)
    return t


def sample_uneven_instances(num: int, seed: int, n_lo: int = 64, n_hi: int = 8192,
                            ranks=(8, 16, 32)):
    """Instance shapes of the uneven-batch workload: n log-uniform in
    [n_lo, n_hi], rank uniform over `ranks`; packed offsets in order."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(n_lo), math.log(n_hi), num)).astype(np.int64)
    ns = np.clip(ns, n_lo, n_hi)
    ms = rng.integers(0, len(ranks), num)
    items, so, to = [], 0, 0
    for n, mi in zip(ns.tolist(), ms.tolist()):
        items.append((so, to, int(n), int(mi)))
        so += int(n)
        to += ranks[mi]
    return items, so, to
