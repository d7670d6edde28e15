"""GPU parity of the garbage h (compute_garbage_h, garbage.rs:101-133) and the
amortized witness z = sum_i c_i s_i (amortization.rs:61-84) against the CPU
oracle, bit-exact, through the device and the host-buffer entry points; and
at the round's size through properties that need no oracle."""
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


@pytest.mark.parametrize("q,d,r,n", [(Q, 64, 1, 5), (Q, 64, 3, 17), (Q, 64, 17, 130),
                                     (Q, 64, 40, 33), (12289, 64, 5, 9), (Q256, 256, 6, 20),
                                     (Q, 64, 64, 50), (Q, 64, 33, 40)])
def test_garbage_h_matches_oracle(cuda, oracle, q, d, r, n):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import compute_garbage_h
    plan, P = TwistedNttPlan(q, d), oracle.Plan(q, d)
    S, Phi = _rand(q, (r, n, d), r * 31 + n), _rand(q, (r, n, d), r * 37 + n)
    want = P.garbage_h(S, Phi, r, n).reshape(-1, d)
    got = compute_garbage_h(plan, _dev(S, cuda), _dev(Phi, cuda))
    assert np.array_equal(_host(got), want)
    assert np.array_equal(compute_garbage_h(plan, S, Phi), want)
    plan.check_device()


@pytest.mark.parametrize("q,d,r,n", [(Q, 64, 1, 5), (Q, 64, 3, 17), (Q, 64, 64, 100),
                                     (12289, 64, 5, 9), (Q256, 256, 6, 20)])
def test_amortize_matches_oracle(cuda, oracle, q, d, r, n):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import amortize_witness
    plan, P = TwistedNttPlan(q, d), oracle.Plan(q, d)
    S, c = _rand(q, (r, n, d), r * 41 + n), _rand(q, (r, d), r * 43 + n)
    want = P.amortize(S, c, r, n).reshape(n, d)
    got = amortize_witness(plan, _dev(S, cuda), _dev(c, cuda))
    assert np.array_equal(_host(got), want)
    assert np.array_equal(amortize_witness(plan, S, c), want)
    plan.check_device()


def test_round_sized_properties(cuda):
    """r = 64, n = 2048: h with phi = s is the Gram matrix, and amortizing with
    challenges (1, 0, ..., 0) returns s_0."""
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import amortize_witness, compute_garbage_g, compute_garbage_h
    plan = TwistedNttPlan(Q, 64)
    r, n = 64, 2048
    g = torch.Generator(device=cuda).manual_seed(21)
    S = torch.randint(0, Q, (r, n, 64), dtype=torch.int64, device=cuda, generator=g).to(torch.int32)
    assert torch.equal(compute_garbage_h(plan, S, S), compute_garbage_g(plan, S))
    c = torch.zeros((r, 64), dtype=torch.int64, device=cuda)
    c[0, 0] = (1 << 32) % Q  # the Montgomery word of the constant 1
    assert torch.equal(amortize_witness(plan, S, c.to(torch.int32)), S[0])
    plan.check_device()
