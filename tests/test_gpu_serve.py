"""Served request stream: every request's result is the same word for word
whether it runs alone (plain per-call mode) or inside a continuously batched
mix, and matches the oracle."""
import numpy as np
import pytest

Q = 4294966657
D = 64

pytestmark = pytest.mark.gpu


def _server_parts(cuda, seed=11):
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.commit import PreparedMatrix
    from lattica_b200.labrador import CommitKey
    plan = TwistedNttPlan(Q, D)
    rng = np.random.default_rng(seed)
    n_max = 512
    mats_host = {m: rng.integers(0, Q, (m, n_max, D), dtype=np.uint64).astype(np.uint32)
                 for m in (8, 16)}
    mats = {m: PreparedMatrix(plan, A, m, n_max) for m, A in mats_host.items()}
    kappa, rn = 4, 128
    A_round = rng.integers(0, Q, (kappa, rn, D), dtype=np.uint64).astype(np.uint32)
    key = CommitKey(plan, A_round, kappa, rn)
    pool_host = rng.integers(0, Q, (8192, D), dtype=np.uint64).astype(np.uint32)
    pool = torch.from_numpy(pool_host.view(np.int32)).to(cuda)
    return plan, mats, mats_host, key, A_round, pool, pool_host


def _schedule(seed, count, rate):
    from lattica_b200.serve import sample_requests
    return sample_requests(seed, count, rate, commit_n=(1, 512), ranks=(8, 16),
                           gram_r=(2, 4, 8), gram_n=128, round_shape=(4, 128),
                           commit_arena=4096, pool_polys=8192)


def test_results_identical_alone_and_in_mix(cuda, oracle):
    from lattica_b200.serve import Request, RingServer, run_load
    plan, mats, mats_host, key, A_round, pool, pool_host = _server_parts(cuda)
    sched = _schedule(5, 120, 40000.0)
    kinds = {r.kind for _, r in sched}
    assert kinds == {"commit", "gramjl", "round"}
    with RingServer(plan, mats, key, pool, mode="continuous", streams=4, k_split=64) as srv:
        stats = run_load(srv, sched)
        batches = srv.batches
    assert stats["requests"] == 120
    n_commit = sum(1 for _, r in sched if r.kind == "commit")
    assert batches < n_commit          # commitments were batched, not issued one by one
    mixed = [r.future.result() for _, r in sched]

    with RingServer(plan, mats, key, pool, mode="plain") as alone:
        for (_, r), got in zip(sched, mixed):
            solo = alone.submit(Request(r.kind, r.offset, r.shape)).result(timeout=60)
            assert len(solo) == len(got)
            for a, b in zip(solo, got):
                assert np.array_equal(a, b), (r.kind, r.offset, r.shape)

    P = oracle.Plan(Q, D)
    F = P.field
    seed = bytes(range(32))
    checked = {"commit": 0, "gramjl": 0, "round": 0}
    for (_, r), got in zip(sched, mixed):
        if checked[r.kind] >= 4:
            continue
        checked[r.kind] += 1
        if r.kind == "commit":
            m, n = r.shape
            A = np.ascontiguousarray(mats_host[m][:, :n, :])
            want = P.matvec(A, m, n, pool_host[r.offset:r.offset + n], 1).reshape(m, D)
            assert np.array_equal(got[0], want)
        else:
            rr, n = r.shape
            S = pool_host[r.offset:r.offset + rr * n]
            g = P.gram(S, rr, n).reshape(-1, D)
            p, _ = oracle.jl_project(F, seed, 256, S.reshape(rr, n * D), rr, n * D, D,
                                     want_flat=False)
            if r.kind == "gramjl":
                assert np.array_equal(got[0], g) and np.array_equal(got[1], p)
            else:
                t = P.matvec(A_round, key.kappa, n, S, rr)
                assert np.array_equal(got[0], oracle.decompose_polys(F, D, t, 256, 4).reshape(-1, D))
                assert np.array_equal(got[1], g)
                assert np.array_equal(got[3], p)
    assert all(v > 0 for v in checked.values())
    plan.check_device()


def test_budget_admission_and_bad_request(cuda):
    from lattica_b200.serve import Request, RingServer
    plan, mats, _, key, _, pool, _ = _server_parts(cuda, seed=3)
    # a budget below one request's footprint still admits it when nothing is in flight
    with RingServer(plan, mats, key, pool, hbm_budget=1024) as srv:
        futs = [srv.submit(Request("commit", 17 * i, (8, 100))) for i in range(6)]
        outs = [f.result(timeout=60) for f in futs]
    assert all(o[0].shape == (8, D) for o in outs)
    with pytest.raises(ValueError):
        RingServer(plan, mats, key, pool, mode="other")
    srv = RingServer(plan, mats, key, pool).start()
    fut = srv.submit(Request("round", 0, (4, 64)))     # length differs from the key
    with pytest.raises(ValueError):
        fut.result(timeout=60)
    with pytest.raises(ValueError):
        srv.stop()
