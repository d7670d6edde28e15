"""GPU parity of the aggregation-side JL evaluations
evals[m] = sum_{i,j} conj(pi_{m,i,j}) s_{i,j} (jl_rows_flat_to_conjugated_polys +
jl_evals, main_protocol/mod.rs:885-923, step_prover.rs:185-206), computed on the
tensor cores straight from the keystream, against the oracle's restatement
over the int8 entries; and at the round's size against the JL projection
(coefficient 0) without an oracle."""
import numpy as np
import pytest

Q = 4294966657

pytestmark = pytest.mark.gpu


def _rand(q, shape, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, q, shape, dtype=np.uint64).astype(np.uint32)


def _dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(cuda)


def _host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("num_parts,n", [(1, 1), (2, 3), (3, 5), (1, 13)])
def test_jl_evals_match_oracle(cuda, oracle, num_parts, n):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import JLMatrix
    d, rows = 64, 256
    plan, P = TwistedNttPlan(Q, d), oracle.Plan(Q, d)
    parts = _rand(Q, (num_parts, n * d), 100 + n)
    parts[0, :5] = [0, 1, Q - 1, 0, Q - 2]  # zero coefficients and their negations
    seed = bytes(range(7, 39))
    _, flat = oracle.jl_project(P.field, seed, rows, parts, num_parts, n * d, d)
    want = P.jl_evals(flat, rows, parts, num_parts, n).reshape(rows, d)
    jl = JLMatrix(seed, rows, n * d)
    assert np.array_equal(jl.conjugated_evals(plan, parts, num_parts, d), want)
    assert np.array_equal(_host(jl.conjugated_evals(plan, _dev(parts, cuda), num_parts, d)), want)
    plan.check_device()


def test_jl_evals_constant_term_is_the_projection_at_round_size(cuda):
    """r = 64 parts of n = 2048 polys: coefficient 0 of every evaluation is the
    JL projection p of the same witness (the identity the verifier checks)."""
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import JLMatrix
    plan = TwistedNttPlan(Q, 64)
    r, n = 64, 2048
    g = torch.Generator(device=cuda).manual_seed(8)
    S = torch.randint(0, Q, (r, n * 64), dtype=torch.int64, device=cuda, generator=g).to(torch.int32)
    jl = JLMatrix(bytes(range(32)), 256, n * 64)
    ev = jl.conjugated_evals(plan, S, r, 64)
    p = jl.project_multi(plan, _host(S), r, 64)
    assert np.array_equal(_host(ev)[:, 0], p)
    plan.check_device()


def test_jl_evals_rejects_unsupported_shapes(cuda):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import JLMatrix
    from lattica_b200.ntt import NttError
    plan = TwistedNttPlan(Q, 64)
    with pytest.raises(NttError):  # GRID_ERR_UNSUPPORTED_SIZE
        JLMatrix(bytes(32), 128, 64).conjugated_evals(plan, _rand(Q, (1, 64), 1), 1, 64)
