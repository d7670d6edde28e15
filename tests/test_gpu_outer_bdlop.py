"""GPU parity of the LaBRADOR outer commitments u1 = B t + C g, u2 = D h
(crs.rs:264-304) and the BDLOP parts u = A_mask r, v = A_msg m + A_open r
(recompute_bdlop_parts_runtime, commit/src/linear.rs:552-573, 800-938)
against compositions of the oracle's pinned matvec and linear commitment."""
import numpy as np
import pytest

Q = 4294966657
Q256 = 4294962689

pytestmark = pytest.mark.gpu


def _rand(q, shape, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, q, shape, dtype=np.uint64).astype(np.uint32)


def _dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(cuda)


def _host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("q,d,rows,mlen,olen,batch", [
    (Q, 64, 8, 64, 16, 1), (Q, 64, 5, 33, 7, 3), (12289, 64, 3, 5, 9, 2), (Q256, 256, 4, 12, 6, 2)])
def test_bdlop_parts_match_oracle(cuda, oracle, q, d, rows, mlen, olen, batch):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.commit import BdlopCommitmentKey
    plan, P = TwistedNttPlan(q, d), oracle.Plan(q, d)
    a_mask = _rand(q, (rows, olen, d), 1)
    a_msg = _rand(q, (rows, mlen, d), 2)
    a_open = _rand(q, (rows, olen, d), 3)
    m = _rand(q, (batch, mlen, d), 4)
    r = _rand(q, (batch, olen, d), 5)
    key = BdlopCommitmentKey(plan, a_mask, a_msg, a_open, rows, mlen, olen)
    want_u = P.matvec(a_mask, rows, olen, r, batch).reshape(batch, rows, d)
    want_v = np.stack([P.linear_commit(a_msg, rows, mlen, a_open, olen, m[b], r[b]).reshape(rows, d)
                       for b in range(batch)])
    u, v = key.recompute_parts(m, r)
    assert np.array_equal(u, want_u) and np.array_equal(v, want_v)
    du, dv = key.recompute_parts(_dev(m, cuda), _dev(r, cuda))
    assert np.array_equal(_host(du), want_u) and np.array_equal(_host(dv), want_v)
    plan.check_device()


def test_bdlop_rejects_bad_shapes(cuda):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.commit import BdlopCommitmentKey
    from lattica_b200.ntt import CommitmentError
    plan = TwistedNttPlan(Q, 64)
    key = BdlopCommitmentKey(plan, _rand(Q, (2, 3, 64), 1), _rand(Q, (2, 4, 64), 2),
                             _rand(Q, (2, 3, 64), 3), 2, 4, 3)
    with pytest.raises(CommitmentError):
        key.recompute_parts(_rand(Q, (4, 64), 4), _rand(Q, (2, 64), 5))
    with pytest.raises(CommitmentError):
        BdlopCommitmentKey(plan, _rand(Q, (2, 5, 64), 1), _rand(Q, (2, 4, 64), 2),
                           _rand(Q, (2, 3, 64), 3), 2, 4, 3)


@pytest.mark.parametrize("kappa1,kappa2,t_len,g_len,h_len", [(4, 3, 48, 20, 20), (16, 8, 1024, 528, 528)])
def test_outer_commitments_match_oracle(cuda, oracle, kappa1, kappa2, t_len, g_len, h_len):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import OuterCommitKey
    plan, P = TwistedNttPlan(Q, 64), oracle.Plan(Q, 64)
    b = _rand(Q, (kappa1, t_len, 64), 11)
    c = _rand(Q, (kappa1, g_len, 64), 12)
    dm = _rand(Q, (kappa2, h_len, 64), 13)
    t, g, h = _rand(Q, (t_len, 64), 14), _rand(Q, (g_len, 64), 15), _rand(Q, (h_len, 64), 16)
    key = OuterCommitKey(plan, b, c, dm, kappa1, kappa2, t_len, g_len, h_len)
    want_u1 = P.linear_commit(b, kappa1, t_len, c, g_len, t, g).reshape(kappa1, 64)
    want_u2 = P.matvec(dm, kappa2, h_len, h, 1).reshape(kappa2, 64)
    assert np.array_equal(key.outer_commit_u1_slice(t, g), want_u1)
    assert np.array_equal(key.outer_commit_u2_slice(h), want_u2)
    assert np.array_equal(_host(key.outer_commit_u1_slice(_dev(t, cuda), _dev(g, cuda))), want_u1)
    assert np.array_equal(_host(key.outer_commit_u2_slice(_dev(h, cuda))), want_u2)
    plan.check_device()
