"""GPU parity of the contractions over point-major evaluations (emm_pm.cu: the
forward transform stores [point][row][k], TMA loads the operand boxes, the
tensor cores contract): commitments, the Gram matrix, garbage h and the fused
prover round against the oracle, and bit-equality with the poly-major kernels
that gather their operands (a plan created with GRID_GPU_CONTRACTION=gather).
Shapes cover ragged K (a partial last 32-word chunk), K splits, the largest
operand boxes (128 X rows, 64 Y rows) and one row; the int32 bound at 8192
words per CTA is in test_gpu_config_sizes.py."""
import os

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


def _gather_plan(q, d):
    """A plan whose contractions gather poly-major operands."""
    from lattica_b200 import TwistedNttPlan
    old = os.environ.get("GRID_GPU_CONTRACTION")
    os.environ["GRID_GPU_CONTRACTION"] = "gather"
    try:
        return TwistedNttPlan(q, d)
    finally:
        if old is None:
            del os.environ["GRID_GPU_CONTRACTION"]
        else:
            os.environ["GRID_GPU_CONTRACTION"] = old


@pytest.mark.parametrize("rows,cols,batch", [
    (16, 2048, 64),   # the LaBRADOR round's inner commitment shape
    (16, 260, 5),     # ragged K: 8 whole chunks and 4 words
    (64, 512, 128),   # largest boxes: 128 X rows, 64 Y rows (NP 64)
    (1, 132, 1),      # one row, one vector
    (40, 1024, 33),   # NP 48
    (17, 4100, 3),    # NP 32, K split over several CTAs
])
def test_point_major_commit_matches_oracle(cuda, oracle, rows, cols, batch):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.commit import PreparedMatrix
    plan = TwistedNttPlan(Q, 64)
    P = oracle.Plan(Q, 64)
    A = _rand(Q, (rows, cols, 64), rows + cols)
    s = _rand(Q, (batch, cols, 64), batch + 1)
    got = _host(PreparedMatrix(plan, A, rows, cols).mul_vec(_dev(s, cuda)))
    gplan = _gather_plan(Q, 64)
    ref = _host(PreparedMatrix(gplan, A, rows, cols).mul_vec(_dev(s, cuda)))
    assert np.array_equal(got, ref)
    # the oracle on a sample of vectors (all of them when the batch is small)
    pick = list(range(batch)) if batch <= 5 else [0, batch // 2, batch - 1]
    want = P.matvec(A, rows, cols, s[pick], len(pick), threads=0).reshape(len(pick), rows, 64)
    assert np.array_equal(got.reshape(batch, rows, 64)[pick], want)
    plan.check_device()


@pytest.mark.parametrize("r,n", [(64, 2048), (7, 132), (1, 4), (33, 260), (64, 8196)])
def test_point_major_gram_matches_oracle(cuda, oracle, r, n):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import compute_garbage_g
    plan = TwistedNttPlan(Q, 64)
    S = _rand(Q, (r, n, 64), 3 * r + n)
    got = _host(compute_garbage_g(plan, _dev(S, cuda)))
    ref = _host(compute_garbage_g(_gather_plan(Q, 64), _dev(S, cuda)))
    assert np.array_equal(got, ref)
    if r * n <= 40000:
        want = oracle.Plan(Q, 64).gram(S, r, n, threads=0).reshape(-1, 64)
        assert np.array_equal(got.reshape(-1, 64), want)
    plan.check_device()


def test_point_major_garbage_h_matches_oracle(cuda, oracle):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import compute_garbage_h
    plan = TwistedNttPlan(Q, 64)
    r, n = 24, 132
    S = _rand(Q, (r, n, 64), 5)
    Phi = _rand(Q, (r, n, 64), 6)
    got = _host(compute_garbage_h(plan, _dev(S, cuda), _dev(Phi, cuda)))
    want = oracle.Plan(Q, 64).garbage_h(S, Phi, r, n).reshape(got.shape)
    assert np.array_equal(got, want)
    plan.check_device()


def test_point_major_round_equals_gather_round(cuda):
    """The fused round at the LaBRADOR size (r = 64, n = 2048, kappa = 16): t
    limbs, g and g limbs identical on both contraction paths."""
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import CommitKey, prover_round_dev
    r, n, kappa = 64, 2048, 16
    rng = np.random.default_rng(8)
    S = _dev(rng.integers(0, Q, (r, n, 64), dtype=np.uint64).astype(np.uint32), cuda)
    A = _rand(Q, (kappa, n, 64), 9)
    outs = []
    for plan in (TwistedNttPlan(Q, 64), _gather_plan(Q, 64)):
        out = prover_round_dev(CommitKey(plan, A, kappa, n), S, 256, 4, 256, 4, None, 0)
        outs.append([_host(x) for x in (out.t_limbs, out.g, out.g_limbs)])
        plan.check_device()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
