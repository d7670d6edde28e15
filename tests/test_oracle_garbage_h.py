"""Pin the oracle's garbage h and amortization (CPU only) against the
reference's definitions restated with one naive negacyclic product per term
(poly/ring.rs:226-228), and against the reference tests' properties: zero phi
gives zero h (garbage.rs test_garbage_h_zero_phi), zero witness gives zero z
(amortization.rs test_amortization_zero_witness), and x 2^-1 2 = x
(test_garbage_division_by_2)."""
import numpy as np

Q = 4294966657
D = 64


def _rand(rng, shape):
    return rng.integers(0, Q, shape, dtype=np.uint64).astype(np.uint32)


def _naive_dot(P, F, a, b):
    """sum_k a[k] * b[k] as ring products, one naive negacyclic product each."""
    acc = np.zeros(D, dtype=np.uint32)
    for k in range(a.shape[0]):
        prod = P.naive_negacyclic(a[k], b[k])
        acc = np.array([F.add(int(x), int(y)) for x, y in zip(acc, prod)], dtype=np.uint32)
    return acc


def test_garbage_h_matches_naive_products(oracle):
    P, F = oracle.Plan(Q, D), oracle.Field(Q)
    rng = np.random.default_rng(11)
    r, n = 3, 4
    S, Phi = _rand(rng, (r, n, D)), _rand(rng, (r, n, D))
    got = P.garbage_h(S, Phi, r, n).reshape(-1, D)
    two_inv = int(F.to_mont(Q // 2 + 1)[0])
    idx = 0
    for i in range(r):
        for j in range(i, r):
            t = _naive_dot(P, F, Phi[i], S[j])
            u = _naive_dot(P, F, Phi[j], S[i])
            want = [F.mul(F.add(int(x), int(y)), two_inv) for x, y in zip(t, u)]
            assert np.array_equal(got[idx], np.array(want, dtype=np.uint32)), (i, j)
            assert idx == oracle.garbage_index(r, i, j)
            idx += 1
    # garbage.rs test_garbage_h_zero_phi
    assert not P.garbage_h(S, np.zeros_like(Phi), r, n).any()


def test_two_inverse_roundtrip(oracle):
    """garbage.rs test_garbage_division_by_2: x * 2^-1 * 2 = x."""
    F = oracle.Field(Q)
    two_inv, two = int(F.to_mont(Q // 2 + 1)[0]), int(F.to_mont(2)[0])
    for v in range(100):
        w = F.mul(F.mul(int(F.to_mont(v)[0]), two_inv), two)
        assert int(F.from_mont(w)[0]) == v


def test_amortize_matches_naive_products(oracle):
    P, F = oracle.Plan(Q, D), oracle.Field(Q)
    rng = np.random.default_rng(12)
    r, n = 3, 5
    S, c = _rand(rng, (r, n, D)), _rand(rng, (r, D))
    got = P.amortize(S, c, r, n).reshape(n, D)
    for k in range(n):
        want = _naive_dot(P, F, c, S[:, k, :])
        assert np.array_equal(got[k], want), k
    # amortization.rs test_amortization_zero_witness
    assert not P.amortize(np.zeros_like(S), c, r, n).any()


def test_jl_evals_are_projections_of_rotated_witnesses(oracle):
    """Coefficient t of evals[m] = sum conj(pi_{m,i,j}) s_{i,j} (the oracle's
    restatement of mod.rs:885-923 and step_prover.rs:185-206) equals the JL
    projection p[m] of the witness with every polynomial multiplied by X^-t;
    t = 0 is the projection itself (the constant-term identity LaBRADOR uses)."""
    q = Q
    P, F = oracle.Plan(q, D), oracle.Field(q)
    rng = np.random.default_rng(13)
    r, n = 2, 3
    parts = _rand(rng, (r, n, D))
    seed = bytes(range(32))
    _, flat = oracle.jl_project(F, seed, 256, parts.reshape(r, n * D), r, n * D, D)
    ev = P.jl_evals(flat, 256, parts.reshape(r, n * D), r, n).reshape(256, D)
    for t in (0, 1, 17, 63):
        # X^-t s: coefficient u is s[u + t] when u + t < d, else -s[u + t - d]
        idx = np.arange(D) + t
        rot = np.where(idx < D, parts[..., idx % D], 0).astype(np.uint32)
        wrap = parts[..., idx % D]
        neg = np.where(wrap == 0, 0, q - wrap.astype(np.uint64)).astype(np.uint32)
        rot = np.where(idx < D, rot, neg)
        p_t, _ = oracle.jl_project(F, seed, 256, rot.reshape(r, n * D), r, n * D, D, want_flat=False)
        assert np.array_equal(ev[:, t], p_t), t
