"""Host-side logic of the batching and serving layers, on CPU: the open-loop
request stream (mix, arrival rate, witness offsets, determinism), the
grouping of queued commitments into contiguous runs for one batched launch,
and the uneven-batch instance sampler."""
import numpy as np
import pytest

from lattica_b200.serve import KINDS, Request, RingServer, sample_requests


def test_request_stream_mix_rate_and_offsets():
    rate, count, arena, pool = 5000.0, 20000, 1 << 14, 1 << 18
    out = sample_requests(7, count, rate, commit_arena=arena, pool_polys=pool,
                          commit_n=(64, 4096), gram_r=(8, 16, 32, 64), gram_n=1024,
                          round_shape=(64, 2048))
    assert len(out) == count
    times = np.array([a for a, _ in out])
    assert times[0] == 0.0 and np.all(np.diff(times) >= 0)
    assert abs(count / times[-1] - rate) / rate < 0.03          # Poisson at the offered rate
    kinds = [r.kind for _, r in out]
    share = {k: kinds.count(k) / count for k in KINDS}
    assert abs(share["commit"] - 0.70) < 0.02 and abs(share["gramjl"] - 0.25) < 0.02
    assert abs(share["round"] - 0.05) < 0.01
    cursor = 0
    for _, r in out:
        if r.kind == "commit":
            m, n = r.shape
            assert m in (8, 16, 32) and 64 <= n <= 4096
            if cursor + n > arena:                                # the arena wraps
                cursor = 0
            assert r.offset == cursor and r.offset + n <= arena    # consecutive slices
            cursor += n
        else:
            rr, n = r.shape
            assert r.offset >= arena and r.offset + rr * n <= pool
            assert (n == 1024 and rr in (8, 16, 32, 64)) if r.kind == "gramjl" else (rr, n) == (64, 2048)
    again = sample_requests(7, count, rate, commit_arena=arena, pool_polys=pool)
    assert [(a, r.kind, r.offset, r.shape) for a, r in again[:50]] == \
           [(a, r.kind, r.offset, r.shape) for a, r in out[:50]]


def test_request_stream_rejects_a_pool_too_small():
    with pytest.raises(ValueError):
        sample_requests(1, 10, 100.0, commit_arena=1 << 10, pool_polys=1 << 11)


def test_queued_commitments_group_into_contiguous_runs():
    reqs = [Request("commit", off, (8, n)) for off, n in
            [(0, 100), (100, 50), (3000, 10), (150, 20), (5000, 64), (3010, 5)]]
    runs = RingServer._runs(reqs, gap=1024)
    spans = [sorted(reqs[i].offset for i in run) for run in runs]
    assert spans == [[0, 100, 150], [3000, 3010], [5000]]
    assert sorted(i for run in runs for i in run) == list(range(len(reqs)))
    # a larger gap joins everything into one launch
    assert len(RingServer._runs(reqs, gap=1 << 20)) == 1


def test_uneven_batch_instances_match_the_workload():
    """Config 3's instances: n log-uniform in [64, 8192] (mean ~1675), rank
    uniform over {8, 16, 32}, witness and output offsets packed in order."""
    import math
    from lattica_b200.batch import sample_uneven_instances
    items, s_polys, t_polys = sample_uneven_instances(4096, 7)
    assert len(items) == 4096
    ns = np.array([it[2] for it in items])
    ms = np.array([(8, 16, 32)[it[3]] for it in items])
    assert ns.min() >= 64 and ns.max() <= 8192
    assert abs(ns.mean() - (8192 - 64) / math.log(8192 / 64)) / 1675 < 0.06
    assert abs(np.log(ns).mean() - (math.log(64) + math.log(8192)) / 2) < 0.1
    assert all(abs((ms == m).mean() - 1 / 3) < 0.03 for m in (8, 16, 32))
    so = np.cumsum([0] + ns.tolist()[:-1])
    to = np.cumsum([0] + ms.tolist()[:-1])
    assert [it[0] for it in items] == so.tolist() and [it[1] for it in items] == to.tolist()
    assert s_polys == ns.sum() and t_polys == ms.sum()
