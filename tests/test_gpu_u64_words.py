"""The reference's default limb, PrimeField<Q, u64> (value * 2^64 mod q,
algebra/src/arith/prime.rs:24-29), at the boundary: u64 words convert to this
library's u32 words (value * 2^32 mod q) and back, and a u64 caller's
commitment over the LaBRADOR modulus 2^32 - 5 returns the reference's u64 words."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

Q = 4294966657
LABRADOR_Q = 4294967291


def _words(values, q, bits):
    return np.array([(int(v) << bits) % q for v in values], dtype=np.uint64)


@pytest.mark.parametrize("q", [Q, LABRADOR_Q, 12289, 17])
def test_u64_words_round_trip(cuda, q):
    import torch
    from lattica_b200.ntt import RingPlan
    plan = RingPlan(q, 64)
    rng = np.random.default_rng(q % 1000)
    vals = [0, 1, q - 1, q // 2] + [int(x) for x in rng.integers(0, q, 5000, dtype=np.uint64)]
    w64 = _words(vals, q, 64)
    w32 = _words(vals, q, 32).astype(np.uint32)
    t64 = torch.from_numpy(w64.view(np.int64)).to(cuda)
    got32 = plan.words_from_u64(t64)
    assert np.array_equal(got32.cpu().numpy().view(np.uint32), w32)
    back = plan.words_to_u64(got32)
    assert np.array_equal(back.cpu().numpy().view(np.uint64), w64)
    bad = torch.from_numpy(np.array([1, q, 2], dtype=np.uint64).view(np.int64)).to(cuda)
    with pytest.raises(ValueError):
        plan.words_from_u64(bad)
    plan.check_device()


def test_u64_caller_commit_on_labrador_modulus(cuda, oracle):
    """A caller holding PrimeField<2^32 - 5> (u64) words: convert, commit on the
    ring plan, convert back; equals the oracle's schoolbook commitment in u64 words."""
    import torch
    from lattica_b200.commit import PreparedMatrix
    from lattica_b200.ntt import RingPlan
    q, d, rows, cols, batch = LABRADOR_Q, 64, 4, 20, 3
    plan = RingPlan(q, d)
    F = oracle.Field(q)
    rng = np.random.default_rng(64)
    A_vals = rng.integers(0, q, rows * cols * d, dtype=np.uint64)
    s_vals = rng.integers(0, q, batch * cols * d, dtype=np.uint64)
    A64 = _words(A_vals, q, 64)
    s64 = _words(s_vals, q, 64)
    to_dev = lambda a: torch.from_numpy(a.view(np.int64)).to(cuda)
    A32 = plan.words_from_u64(to_dev(A64)).view(rows, cols, d)
    s32 = plan.words_from_u64(to_dev(s64)).view(batch, cols, d)
    t64 = plan.words_to_u64(PreparedMatrix(plan, A32, rows, cols).mul_vec(s32))
    want32 = F.ring_matvec(d, _words(A_vals, q, 32).astype(np.uint32), rows, cols,
                           _words(s_vals, q, 32).astype(np.uint32), batch)
    rinv = pow(1 << 32, -1, q)
    want64 = np.array([(int(w) * rinv % q << 64) % q for w in want32], dtype=np.uint64)
    assert np.array_equal(t64.cpu().numpy().view(np.uint64).reshape(-1), want64)
    plan.check_device()
