"""Uneven batched commitments: the one-sequence batched path (plain and CUDA
graph), the per-call path and the oracle agree word for word; the autotuner
persists its choice."""
import json

import numpy as np
import pytest

Q = 4294966657

pytestmark = pytest.mark.gpu


def _setup(cuda, oracle, ranks, n_hi, num, seed):
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.batch import sample_uneven_instances
    from lattica_b200.commit import PreparedMatrix
    d = 64
    plan = TwistedNttPlan(Q, d)
    rng = np.random.default_rng(seed)
    mats_host = [rng.integers(0, Q, (m, n_hi, d), dtype=np.uint64).astype(np.uint32) for m in ranks]
    mats = [PreparedMatrix(plan, A, A.shape[0], n_hi) for A in mats_host]
    items, s_polys, t_polys = sample_uneven_instances(num, seed, n_lo=1, n_hi=n_hi, ranks=ranks)
    s_host = rng.integers(0, Q, (s_polys, d), dtype=np.uint64).astype(np.uint32)
    s = torch.from_numpy(s_host.view(np.int32)).to(cuda)
    return plan, mats, mats_host, items, s_host, s, t_polys


def _oracle_expect(oracle, mats_host, items, s_host, t_polys):
    P = oracle.Plan(Q, 64)
    want = np.zeros((t_polys, 64), np.uint32)
    for so, to, n, m in items:
        A = np.ascontiguousarray(mats_host[m][:, :n, :])
        rows = A.shape[0]
        t = P.matvec(A, rows, n, s_host[so:so + n], 1).reshape(rows, 64)
        want[to:to + rows] = t
    return want


def test_batched_uneven_commits_match_oracle_and_per_call(cuda, oracle, tmp_path):
    import torch
    from lattica_b200.batch import UnevenCommitBatch, per_call_commit
    ranks = (3, 8, 32)
    plan, mats, mats_host, items, s_host, s, t_polys = _setup(cuda, oracle, ranks, 300, 70, 4)
    want = _oracle_expect(oracle, mats_host, items, s_host, t_polys)
    batch = UnevenCommitBatch(plan, mats, items)
    assert batch.s_polys == s_host.shape[0] and batch.t_polys == t_polys
    t = torch.zeros((t_polys, 64), dtype=torch.int32, device=cuda)
    for k_split in (16, 64, 256, 4096):
        batch.set_k_split(k_split)
        t.zero_()
        batch.commit_dev(s, t)
        torch.cuda.synchronize()
        assert np.array_equal(t.cpu().numpy().view(np.uint32), want), k_split
    # graph capture on a side stream, replayed twice
    side = torch.cuda.Stream(cuda)
    with torch.cuda.stream(side):
        for _ in range(2):
            t.zero_()
            batch.commit_dev(s, t, graph=True, stream=side)
    side.synchronize()
    assert np.array_equal(t.cpu().numpy().view(np.uint32), want)
    # per-call path
    t2 = torch.zeros_like(t)
    per_call_commit(plan, mats, items, s, t2)
    assert torch.equal(t, t2)
    # one-shot path: tables built into the caller's workspace, no handle
    import ctypes as C
    from lattica_b200 import _lib
    lib = _lib.load()
    arr = (_lib.BatchItem * len(items))(*[_lib.BatchItem(*it) for it in items])
    hs = (C.c_void_p * len(mats))(*[m.handle.value for m in mats])
    for k_split in (0, 32, 1024):      # 0: the library picks the K range
        nb = C.c_size_t()
        assert lib.grid_gpu_batch_oneshot_workspace(plan.handle, hs, len(mats), arr, len(items),
                                                    k_split, C.byref(nb)) == 0
        ws = torch.empty(nb.value, dtype=torch.uint8, device=cuda)
        t3 = torch.zeros_like(t)
        st = lib.grid_gpu_batch_commit_oneshot_dev(
            plan.handle, hs, len(mats), arr, len(items), k_split, s.data_ptr(), t3.data_ptr(),
            ws.data_ptr(), ws.numel(), torch.cuda.current_stream(cuda).cuda_stream)
        assert st == 0
        torch.cuda.synchronize()
        assert torch.equal(t3, t), k_split
        assert lib.grid_gpu_batch_commit_oneshot_dev(
            plan.handle, hs, len(mats), arr, len(items), k_split, s.data_ptr(), t3.data_ptr(),
            ws.data_ptr(), ws.numel() - 256, 0) != 0     # workspace too small
    # autotuner: picks a candidate, persists it, reuses it
    cache = tmp_path / "autotune.json"
    res = batch.autotune(s, t, candidates=(64, 256), reps=2, cache_path=str(cache))
    assert res["k_split"] in (64, 256) and not res["cached"]
    assert json.loads(cache.read_text())[batch.signature()]["k_split"] == res["k_split"]
    res2 = batch.autotune(s, t, candidates=(64, 256), cache_path=str(cache))
    assert res2["cached"] and res2["k_split"] == res["k_split"]
    batch.commit_dev(s, t)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy().view(np.uint32), want)
    plan.check_device()


def test_batch_rejects_bad_items(cuda):
    import ctypes as C
    from lattica_b200 import CommitmentError, TwistedNttPlan
    from lattica_b200.batch import UnevenCommitBatch
    from lattica_b200.commit import PreparedMatrix
    plan = TwistedNttPlan(Q, 64)
    M = PreparedMatrix(plan, np.zeros((4, 10, 64), np.uint32), 4, 10)
    with pytest.raises(CommitmentError):
        UnevenCommitBatch(plan, [M], [(0, 0, 11, 0)])   # n beyond the matrix
    with pytest.raises(CommitmentError):
        UnevenCommitBatch(plan, [M], [(0, 0, 5, 1)])    # no such matrix


@pytest.mark.parametrize("schedule", [(1024, 0, 1), (2048, 64, 1), (8192, 32, 1), (256, 0, 1),
                                      (4096, 0, 2), (1024, 0, 3), (8192, 0, 3), (256, 64, 3),
                                      (32, 32, 3), (96, 0, 3)])
def test_batched_commit_schedules_match_oracle(cuda, oracle, schedule):
    """Every engine and tile shape (tensor cores with 128, 64 or 32 instances per
    tile; CUDA cores; tensor cores over point-major evaluations, down to one
    32-word chunk per K range) gives the oracle's words."""
    import torch
    from lattica_b200.batch import UnevenCommitBatch
    ranks = (8, 16, 32)
    plan, mats, mats_host, items, s_host, s, t_polys = _setup(cuda, oracle, ranks, 700, 150, 11)
    want = _oracle_expect(oracle, mats_host, items, s_host, t_polys)
    batch = UnevenCommitBatch(plan, mats, items)
    batch.set_config(*schedule)
    cfg = batch.config()
    assert cfg["tensor_cores"] == (schedule[2] in (1, 3)) and cfg["k_split"] == schedule[0]
    t = torch.zeros((t_polys, 64), dtype=torch.int32, device=cuda)
    batch.commit_dev(s, t)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy().view(np.uint32), want), schedule
    plan.check_device()


def test_point_major_engine_needs_whole_chunks_and_point_major_matrices(cuda):
    """The point-major engine takes K ranges of whole 32-word chunks, and only
    matrices that hold point-major evaluations (cols a multiple of 4)."""
    from lattica_b200 import CommitmentError, TwistedNttPlan, _lib
    from lattica_b200._lib import GridGpuError
    from lattica_b200.batch import UnevenCommitBatch
    from lattica_b200.commit import PreparedMatrix
    plan = TwistedNttPlan(Q, 64)
    M = PreparedMatrix(plan, np.zeros((4, 40, 64), np.uint32), 4, 40)
    batch = UnevenCommitBatch(plan, [M], [(0, 0, 40, 0), (40, 4, 7, 0)])
    with pytest.raises(CommitmentError):
        batch.set_config(48, 0, _lib.ENGINE_POINT_MAJOR)
    batch.set_config(64, 0, _lib.ENGINE_POINT_MAJOR)
    M2 = PreparedMatrix(plan, np.zeros((4, 41, 64), np.uint32), 4, 41)  # no point-major copy
    batch2 = UnevenCommitBatch(plan, [M2], [(0, 0, 41, 0)])
    with pytest.raises(GridGpuError, match="UnsupportedDegree"):  # this engine cannot run it
        batch2.set_config(64, 0, _lib.ENGINE_POINT_MAJOR)
    plan.check_device()


def test_autotuner_searches_tile_shapes(cuda, oracle, tmp_path):
    import torch
    from lattica_b200.batch import UnevenCommitBatch
    plan, mats, mats_host, items, s_host, s, t_polys = _setup(cuda, oracle, (8, 32), 400, 60, 12)
    want = _oracle_expect(oracle, mats_host, items, s_host, t_polys)
    batch = UnevenCommitBatch(plan, mats, items)
    t = torch.zeros((t_polys, 64), dtype=torch.int32, device=cuda)
    res = batch.autotune(s, t, reps=1, cache_path=str(tmp_path / "a.json"))
    assert len(res["candidates_ms"]) == len(batch.schedules())
    assert res["engine"] in ("tensor", "cuda_core", "point_major") and not res["cached"]
    t.zero_()
    batch.commit_dev(s, t)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy().view(np.uint32), want)
    res2 = batch.autotune(s, t, cache_path=str(tmp_path / "a.json"))
    assert res2["cached"] and res2["schedule"] == res["schedule"]


@pytest.mark.parametrize("k_split", [0, 64, 1024])
def test_batched_gram_of_uneven_rank_matches_oracle(cuda, oracle, k_split):
    """compute_garbage_g for witnesses of r in {1, 5, 8, 16, 17, 33, 64} and
    uneven n, at scattered offsets of one pool, in one launch sequence."""
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import compute_garbage_g, compute_garbage_g_batch
    plan = TwistedNttPlan(Q, 64)
    P = oracle.Plan(Q, 64)
    rng = np.random.default_rng(k_split + 5)
    shapes = [(64, 300), (1, 7), (5, 130), (16, 64), (17, 33), (33, 200), (8, 1), (64, 40),
              (16, 1100)]
    items, off = [], 0
    for r, n in shapes:
        off += int(rng.integers(0, 50))  # gaps: witnesses not packed
        items.append((off, r, n))
        off += r * n
    pool_h = rng.integers(0, Q, (off, 64), dtype=np.uint64).astype(np.uint32)
    pool_h[items[0][0]:items[0][0] + 64 * 300][:, :] = Q - 1  # largest words in one witness
    pool = torch.from_numpy(pool_h.view(np.int32)).to(cuda)
    G = compute_garbage_g_batch(plan, pool, items, k_split=k_split)
    torch.cuda.synchronize()
    got = G.cpu().numpy().view(np.uint32)
    g0 = 0
    for so, r, n in items:
        cnt = r * (r + 1) // 2
        want = P.gram(pool_h[so:so + r * n], r, n, threads=0).reshape(cnt, 64)
        assert np.array_equal(got[g0:g0 + cnt], want), (r, n)
        g0 += cnt
    # packed witnesses (one transform launch) give the same words
    packed, items2, o = [], [], 0
    for so, r, n in items:
        packed.append(pool_h[so:so + r * n])
        items2.append((o, r, n))
        o += r * n
    pool2 = torch.from_numpy(np.concatenate(packed).view(np.int32)).to(cuda)
    G2 = compute_garbage_g_batch(plan, pool2, items2, k_split=k_split)
    assert torch.equal(G2, G)
    # and one compute_garbage_g per item
    so, r, n = items[2]
    assert torch.equal(compute_garbage_g(plan, pool[so:so + r * n].view(r, n, 64)),
                       G[sum(x[1] * (x[1] + 1) // 2 for x in items[:2]):][:r * (r + 1) // 2])
    plan.check_device()


def test_batched_gram_rejects_bad_items(cuda):
    import ctypes as C
    from lattica_b200 import TwistedNttPlan, _lib
    lib = _lib.load()
    plan = TwistedNttPlan(Q, 64)
    nb = C.c_size_t()
    bad = (_lib.GramItem * 1)(_lib.GramItem(0, 65, 10))  # r > 64
    assert lib.grid_gpu_batch_gram_workspace(plan.handle, bad, 1, 0, C.byref(nb)) == 5
    zero = (_lib.GramItem * 1)(_lib.GramItem(0, 3, 0))
    assert lib.grid_gpu_batch_gram_workspace(plan.handle, zero, 1, 0, C.byref(nb)) == 5
    ok = (_lib.GramItem * 1)(_lib.GramItem(0, 3, 10))
    assert lib.grid_gpu_batch_gram_workspace(plan.handle, ok, 1, 100, C.byref(nb)) == 5  # k % 16
