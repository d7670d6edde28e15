"""Seeded commitment-key expansion on the GPU (CommitKey::from_seed,
labrador/src/crs.rs:136-198, 308-326; PrimeField::rand, prime.rs:730-743)
against the oracle's restatement of ChaCha20Rng + u64 rejection sampling,
word for word, including a lowered threshold that makes rejections frequent
enough to exercise the device compaction."""
import numpy as np
import pytest

Q = 4294966657

pytestmark = pytest.mark.gpu


def _host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("q,npolys", [(Q, 1), (Q, 33), (Q, 1000), (12289, 77)])
def test_uniform_polys_match_oracle(cuda, oracle, q, npolys):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import sample_uniform_polys
    plan = TwistedNttPlan(q, 64)
    seed = bytes((7 * i + npolys) & 0xFF for i in range(32))
    want = oracle.sample_uniform_polys(oracle.Field(q), seed, npolys, 64).reshape(npolys, 64)
    assert np.array_equal(sample_uniform_polys(plan, seed, npolys), want)
    assert np.array_equal(_host(sample_uniform_polys(plan, seed, npolys, device=cuda)), want)
    plan.check_device()


def test_rejections_compact_like_the_sequential_sampler(cuda, oracle):
    """accept_max = 2^64 - 2^60 rejects about 1 in 16 samples."""
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import sample_uniform_polys
    plan = TwistedNttPlan(Q, 64)
    seed, npolys, amax = bytes(range(32)), 5000, (1 << 64) - (1 << 60)
    want = oracle.sample_uniform_polys(oracle.Field(Q), seed, npolys, 64, accept_max=amax)
    got = sample_uniform_polys(plan, seed, npolys, device=cuda, accept_max=amax)
    plan.check_device()
    assert np.array_equal(_host(got).reshape(-1), want)
    plain = oracle.sample_uniform_polys(oracle.Field(Q), seed, npolys, 64)
    assert not np.array_equal(plain, want)  # the planted threshold did reject


def test_exhausted_margin_is_reported(cuda):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200._lib import GridGpuError
    from lattica_b200.labrador import sample_uniform_polys
    plan = TwistedNttPlan(Q, 64)
    with pytest.raises(GridGpuError):  # half the samples rejected: more than the margin
        sample_uniform_polys(plan, bytes(32), 4000, accept_max=1 << 63)


def test_commit_key_from_seed_spans(cuda, oracle):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import commit_key_from_seed
    plan = TwistedNttPlan(Q, 64)
    r, n, kappa, k1, k2, t1, t2 = 3, 10, 2, 2, 3, 2, 2
    seed = bytes(range(100, 132))
    key, outer = commit_key_from_seed(plan, seed, r, n, kappa, k1, k2, t1, t2, device=cuda)
    g = r * (r + 1) // 2
    sizes = [kappa * n, k1 * r * t1 * kappa, k1 * t2 * g, k2 * t1 * g]
    allp = oracle.sample_uniform_polys(oracle.Field(Q), seed, sum(sizes), 64).reshape(-1, 64)
    # the inner key commits like the oracle with A = the first span
    P = oracle.Plan(Q, 64)
    rng = np.random.default_rng(5)
    s = rng.integers(0, Q, (1, n, 64), dtype=np.uint64).astype(np.uint32)
    want = P.matvec(allp[:kappa * n], kappa, n, s, 1).reshape(kappa, 64)
    assert np.array_equal(key.inner_commit_slice(s).reshape(kappa, 64), want)
    # u2 = D h with D the last span
    h = rng.integers(0, Q, (t1 * g, 64), dtype=np.uint64).astype(np.uint32)
    D = allp[sum(sizes[:3]):]
    assert np.array_equal(outer.outer_commit_u2_slice(h), P.matvec(D, k2, t1 * g, h, 1).reshape(k2, 64))
    plan.check_device()
