"""GPU parity of commitments, the Gram matrix, decompositions and the JL
projection against the CPU oracle (bit-exact)."""
import numpy as np
import pytest

Q = 4294966657
Q256 = 4294962689

pytestmark = pytest.mark.gpu


def _rand(q, shape, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, q, shape, dtype=np.uint64).astype(np.uint32)


def _ternary(F, shape, seed):
    rng = np.random.default_rng(seed)
    v = rng.integers(-1, 2, shape)
    return F.to_mont(np.where(v < 0, F.q + v, v).astype(np.uint64).ravel()).reshape(shape)


def _dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(cuda)


def _host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("q,d,rows,cols,batch", [
    (Q, 64, 8, 64, 64),         # plain Ajtai commit shape
    (Q, 64, 16, 3000, 1),       # one vector, long K: the matrix-vector kernel with K splits
    (Q, 64, 16, 300, 5),
    (12289, 64, 3, 5, 7),
    (17, 8, 2, 9, 3),
    (Q256, 256, 4, 40, 6),
    (Q, 32, 33, 17, 2),
    # tensor-core contraction: Y rows padded to 16 / 32 / 48 / 64, X rows <= 64 or <= 128
    (Q, 64, 17, 40, 64),        # NP 32, X 64 rows
    (Q, 64, 24, 50, 70),        # NP 32, X 128-row buffers
    (Q, 64, 40, 70, 100),       # NP 48
    (Q, 64, 49, 20, 65),        # NP 64, just past 64 X rows
    (Q, 64, 64, 33, 128),       # NP 64, 128 X rows
    # one-launch small commitments (rows <= 32, cols <= 128, batch <= 1024)
    (Q, 64, 1, 1, 1),
    (Q, 64, 5, 100, 2),         # a second group of 64 columns, partly filled
    (Q, 64, 32, 128, 3),        # largest rows and cols
    (Q, 64, 31, 65, 7),
    (Q, 64, 8, 64, 1024),       # largest batch
])
def test_commit_matches_oracle(cuda, oracle, q, d, rows, cols, batch):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.commit import PreparedMatrix
    plan = TwistedNttPlan(q, d)
    P = oracle.Plan(q, d)
    A = _rand(q, (rows, cols, d), rows * 7 + cols)
    s = _ternary(P.field, (batch, cols, d), batch) if q == Q else _rand(q, (batch, cols, d), 3)
    want = P.matvec(A, rows, cols, s, batch, threads=0).reshape(batch, rows, d)
    M = PreparedMatrix(plan, A, rows, cols)
    assert np.array_equal(M.mul_vec(s), want)
    assert np.array_equal(_host(M.mul_vec(_dev(s, cuda))), want)
    # A given directly in the evaluation domain (TwistedNttPoly::from_evals)
    Ah = P.forward(A).reshape(rows, cols, d)
    M2 = PreparedMatrix(plan, Ah, rows, cols, is_evals=True)
    assert np.array_equal(M2.mul_vec(s), want)


def test_prepared_linear_commit_matches_coefficient_path(cuda, oracle):
    """Port of linear.rs test_prepared_linear_recompute_matches_coefficient_path
    (commit/src/linear.rs:1128): Poly8 over F17."""
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.commit import CommitmentDimensions, LinearCommitmentKey
    q, d = 17, 8
    P = oracle.Plan(q, d)
    F = P.field
    i = np.arange(d)
    one = F.to_mont([1] + [0] * (d - 1))
    zero = F.to_mont([0] * d)
    lin = lambda a: F.to_mont(((a * i + 1) % q).tolist())
    a_msg = np.stack([one, zero, lin(1), lin(2)])
    a_open = np.stack([zero, one, lin(3), lin(4)])
    m = np.stack([one, lin(5)])
    r = np.stack([zero, lin(6)])
    dims = CommitmentDimensions(2, 2, 2)
    key = LinearCommitmentKey(TwistedNttPlan(q, d), a_msg, a_open, dims)
    got = key.recompute(m, r)
    want = P.linear_commit(a_msg, 2, 2, a_open, 2, m, r).reshape(2, d)
    # coefficient-domain schoolbook reference of the same commitment
    naive = np.zeros((2, d), np.uint32)
    for row in range(2):
        acc = np.zeros(d, np.uint32)
        for k in range(2):
            for prod in (P.naive_negacyclic(a_msg[row * 2 + k], m[k]),
                         P.naive_negacyclic(a_open[row * 2 + k], r[k])):
                acc = np.array([F.add(int(x), int(y)) for x, y in zip(acc, prod)], np.uint32)
        naive[row] = acc
    assert np.array_equal(want, naive)
    assert np.array_equal(got, want)


def test_linear_commit_rejects_bad_shapes(cuda):
    from lattica_b200 import CommitmentError, TwistedNttPlan
    from lattica_b200.commit import CommitmentDimensions, LinearCommitmentKey
    plan = TwistedNttPlan(Q, 64)
    dims = CommitmentDimensions(2, 3, 2)
    key = LinearCommitmentKey(plan, np.zeros((2, 2, 64), np.uint32), np.zeros((2, 3, 64), np.uint32), dims)
    with pytest.raises(CommitmentError) as ei:
        key.recompute(np.zeros((1, 64), np.uint32), np.zeros((3, 64), np.uint32))
    assert ei.value.kind == "DimensionMismatch"
    with pytest.raises(CommitmentError) as ei:
        CommitmentDimensions(0, 1, 1).validate()
    assert ei.value.kind == "InvalidParameters"


@pytest.mark.parametrize("q,d,r,n", [(Q, 64, 1, 4), (Q, 64, 3, 70), (Q, 64, 5, 130),
                                     (12289, 64, 33, 9), (Q256, 256, 6, 12), (17, 8, 4, 3),
                                     (Q, 64, 40, 1100), (Q, 64, 20, 30), (Q, 64, 64, 40),
                                     (Q, 64, 16, 77), (Q, 64, 17, 9)])
def test_gram_matches_oracle(cuda, oracle, q, d, r, n):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import compute_garbage_g
    plan = TwistedNttPlan(q, d)
    P = oracle.Plan(q, d)
    S = _rand(q, (r, n, d), r + n)
    want = P.gram(S, r, n, threads=0).reshape(-1, d)
    if r * n <= 64:
        assert np.array_equal(P.gram(S, r, n, naive=True).reshape(-1, d), want)
    assert np.array_equal(compute_garbage_g(plan, S), want)
    assert np.array_equal(_host(compute_garbage_g(plan, _dev(S, cuda))), want)


@pytest.mark.parametrize("base,limbs", [(256, 4), (8, 3), (10, 12), (2, 32)])
def test_balanced_decomposition_matches_oracle(cuda, oracle, base, limbs):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import decompose_polys
    plan = TwistedNttPlan(Q, 64)
    F = oracle.Field(Q)
    polys = _rand(Q, (9, 64), base)
    polys[0, :10] = F.to_mont([0, 1, Q - 1, Q // 2, Q // 2 + 1, 127, 128, 129, base // 2, Q - base // 2])
    want = oracle.decompose_polys(F, 64, polys, base, limbs).reshape(-1, 64)
    got = decompose_polys(plan, polys, base, limbs)
    assert got.num_polys == 9 and got.num_limbs == limbs
    assert np.array_equal(got.flat, want)


def test_balanced_decomposition_kats_on_gpu(cuda, oracle, kats):
    """decompose_coeff_balanced KATs (main_protocol/mod.rs:1107-1118), through the GPU."""
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import decompose_polys
    for c in kats["decompose_coeff_balanced"]:
        q, d = c["q"], 64
        plan = TwistedNttPlan(q, d)
        F = oracle.Field(q)
        poly = F.to_mont([c["value"]] * d).reshape(1, d)
        out = decompose_polys(plan, poly, c["base"], c["num_limbs"]).flat
        vals = F.from_mont(out[:, 0]).astype(np.int64)
        signed = np.where(vals > q // 2, vals - q, vals)
        assert signed.tolist() == c["limbs"], c["source"]


def test_gadget_decompose_matches_oracle(cuda, oracle):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.commit import gadget_decompose, gadget_digits
    plan = TwistedNttPlan(Q, 64)
    F = oracle.Field(Q)
    x = _rand(Q, 5 * 64, 9)
    x[:3] = F.to_mont([0, 1, Q - 1])
    for base in (256, 16, 3):
        assert gadget_digits(Q, base) == oracle.gadget_digits(Q, base)
        want = oracle.gadget_decompose(F, x, base)
        assert np.array_equal(gadget_decompose(plan, x, base, digit_major=True), want)
        per_poly = gadget_decompose(plan, x, base, digit_major=False)
        k = want.shape[0]
        assert np.array_equal(per_poly, want.reshape(k, 5, 64).transpose(1, 0, 2))


@pytest.mark.parametrize("rows,num_parts,n,d", [(256, 3, 5, 64), (100, 2, 3, 64),
                                                (256, 1, 130, 64), (7, 4, 2, 8),
                                                # entries written by the projection kernel
                                                # (whole blocks, n % 32 == 0, d % 8 == 0)
                                                (256, 3, 32, 64), (253, 2, 64, 64),
                                                (256, 2, 96, 8), (255, 1, 32, 16)])
def test_jl_projection_matches_oracle(cuda, oracle, rows, num_parts, n, d):
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import JLMatrix
    q = 17 if d == 8 else Q
    plan = TwistedNttPlan(q, d)
    F = oracle.Field(q)
    seed = bytes((7 * i + rows) & 0xFF for i in range(32))
    cols = n * d
    parts = _rand(q, (num_parts, cols), rows + n)
    want_p, want_flat = oracle.jl_project(F, seed, rows, parts, num_parts, cols, d)
    jl = JLMatrix.from_seed(rows, cols, seed)
    p, flat = jl.project_and_extract_jl_rows(plan, parts, num_parts, d)
    assert np.array_equal(p, want_p)
    assert np.array_equal(flat, want_flat)
    assert np.array_equal(jl.project_multi(plan, parts, num_parts, d), want_p)


def test_prover_round_matches_oracle(cuda, oracle):
    """Fused round (commit + limbs, Gram + limbs, JL) on a small LaBRADOR witness."""
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import CommitKey, prover_round_dev, verify_norm
    q, d, r, n, kappa = Q, 64, 6, 64, 4  # n % 32 == 0: entries from the projection kernel
    plan = TwistedNttPlan(q, d)
    P = oracle.Plan(q, d)
    F = P.field
    rng = np.random.default_rng(77)
    coeffs = rng.integers(-2048, 2049, (r, n, d))
    S = F.to_mont(np.where(coeffs < 0, q + coeffs, coeffs).astype(np.uint64).ravel()).reshape(r, n, d)
    A = _rand(q, (kappa, n, d), 5)
    seed = bytes(range(32))
    key = CommitKey(plan, A, kappa, n)
    out = prover_round_dev(key, _dev(S, cuda), 256, 4, 256, 4, seed, 256, extract=True)
    torch.cuda.synchronize()
    t = P.matvec(A, kappa, n, S, r)
    assert np.array_equal(_host(out.t_limbs),
                          oracle.decompose_polys(F, d, t, 256, 4).reshape(-1, d))
    g = P.gram(S, r, n, threads=0)
    assert np.array_equal(_host(out.g), g.reshape(-1, d))
    assert np.array_equal(_host(out.g_limbs), oracle.decompose_polys(F, d, g, 256, 4).reshape(-1, d))
    p, flat = oracle.jl_project(F, seed, 256, S.reshape(r, n * d), r, n * d, d)
    assert np.array_equal(_host(out.p), p)
    assert np.array_equal(out.jl_flat.cpu().numpy(), flat)
    # the checks verify_step applies to these outputs, on the GPU's own words:
    # limbs reconstruct to t = A s and to g (reconstruct_from_limbs,
    # main_protocol/mod.rs:331-359), and p passes the JL norm gate (jl.rs:533-547)
    # for a bound above the witness norm (E ||p||^2 = 128 ||s||^2) and fails below it
    tl, gl = _host(out.t_limbs), _host(out.g_limbs)
    for i in range(r * kappa):
        rec = oracle.reconstruct_from_limbs(F, d, tl[i * 4:(i + 1) * 4].reshape(-1), 256)
        assert np.array_equal(rec, t.reshape(-1, d)[i])
    for i in range(0, g.reshape(-1, d).shape[0], 97):
        rec = oracle.reconstruct_from_limbs(F, d, gl[i * 4:(i + 1) * 4].reshape(-1), 256)
        assert np.array_equal(rec, g.reshape(-1, d)[i])
    s_norm = float(np.sqrt(np.sum(coeffs.astype(np.float64) ** 2)))
    assert verify_norm(_host(out.p), q, 1.5 * s_norm)
    assert not verify_norm(_host(out.p), q, 0.5 * s_norm)
    plan.check_device()


@pytest.mark.parametrize("extract", [False, True])
def test_prover_round_with_jl_evals(cuda, oracle, extract):
    """The round's JL evaluations; without extraction p comes from their coefficient 0."""
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import CommitKey, prover_round_dev
    q, d, r, n, kappa = Q, 64, 3, 20, 4
    plan = TwistedNttPlan(q, d)
    P = oracle.Plan(q, d)
    F = P.field
    S = _rand(q, (r, n, d), 41)
    A = _rand(q, (kappa, n, d), 43)
    seed = bytes((5 * i + 1) & 0xFF for i in range(32))
    key = CommitKey(plan, A, kappa, n)
    out = prover_round_dev(key, _dev(S, cuda), 256, 4, 256, 4, seed, 256, extract=extract,
                           jl_evals=True)
    torch.cuda.synchronize()
    p, flat = oracle.jl_project(F, seed, 256, S.reshape(r, n * d), r, n * d, d)
    assert np.array_equal(_host(out.p), p)
    assert np.array_equal(_host(out.jl_evals),
                          P.jl_evals(flat, 256, S.reshape(r, n * d), r, n).reshape(256, d))
    assert (out.jl_flat is not None) == extract
    t = P.matvec(A, kappa, n, S, r)
    assert np.array_equal(_host(out.t_limbs),
                          oracle.decompose_polys(F, d, t, 256, 4).reshape(-1, d))
    assert np.array_equal(_host(out.g), P.gram(S, r, n, threads=0).reshape(-1, d))
    with pytest.raises(ValueError):
        prover_round_dev(key, _dev(S, cuda), 256, 4, 256, 4, None, 256, jl_evals=True)
    plan.check_device()
