"""CPU checks of the oracle's schoolbook ring contractions and slice hooks.

The reference multiplies in R_q through the twisted NTT only when q has a
2d-th root of unity, and otherwise by the schoolbook rule
(naive_negacyclic_mul_coeffs, algebra/src/poly/ring.rs:60-100); its own
LaBRADOR primes (2^32 - 5, 12281) take that branch. The oracle's fused
schoolbook contractions (orc_ring_*) are pinned here three ways: against a
term-by-term restatement over orc_naive_negacyclic and field additions (the
reference's operation order), against Python big-integer arithmetic, and, for
NTT-friendly primes, against the oracle's NTT-domain Gram and matvec.
"""
import numpy as np
import pytest

Q = 4294966657
LABRADOR_Q = 4294967291  # 2^32 - 5: no 128th root of unity
SMALL_Q = 12281          # examples/fibonacci_round_trip.rs: no 128th root either


def _words(rng, q, shape):
    return rng.integers(0, q, shape, dtype=np.uint64).astype(np.uint32)


@pytest.mark.parametrize("q", [LABRADOR_Q, SMALL_Q, 12289, Q])
def test_ring_gram_matches_term_by_term_schoolbook(oracle, q):
    F = oracle.Field(q)
    d, r, n = 64, 4, 5
    rng = np.random.default_rng(q % 1000)
    S = _words(rng, q, (r, n, d))
    S[0, 0] = q - 1  # all-maximal words: the largest integer sums
    G = F.ring_gram(d, S, r, n, threads=2).reshape(-1, d)
    idx = 0
    for i in range(r):
        for j in range(i, r):
            want = np.zeros(d, np.uint32)
            for k in range(n):
                want = F.add_slice(want, F.naive_negacyclic(S[i, k], S[j, k]))
            assert np.array_equal(G[idx], want), (i, j)
            idx += 1


@pytest.mark.parametrize("q,d", [(LABRADOR_Q, 64), (SMALL_Q, 64), (LABRADOR_Q, 16),
                                 (LABRADOR_Q, 256)])
def test_ring_matvec_matches_python_integers(oracle, q, d):
    F = oracle.Field(q)
    rows, cols, batch = 3, 4, 2
    rng = np.random.default_rng(d)
    A = _words(rng, q, (rows, cols, d))
    s = _words(rng, q, (batch, cols, d))
    t = F.ring_matvec(d, A, rows, cols, s, batch, threads=2).reshape(batch, rows, d)
    rinv = pow(2 ** 32, -1, q)
    for b in range(batch):
        for i in range(rows):
            acc = [0] * d
            for k in range(cols):
                x, y = [int(v) for v in A[i, k]], [int(v) for v in s[b, k]]
                for u in range(d):
                    for v in range(d):
                        term = x[u] * y[v] * rinv
                        if u + v < d:
                            acc[u + v] += term
                        else:
                            acc[u + v - d] -= term
            assert [a % q for a in acc] == [int(w) for w in t[b, i]], (b, i)


@pytest.mark.parametrize("q", [12289, Q])
def test_ring_contractions_match_ntt_domain_oracle(oracle, q):
    d, r, n = 64, 6, 9
    P = oracle.Plan(q, d)
    F = P.field
    rng = np.random.default_rng(7)
    S = _words(rng, q, (r, n, d))
    assert np.array_equal(F.ring_gram(d, S, r, n), P.gram(S, r, n))
    A = _words(rng, q, (5, n, d))
    assert np.array_equal(F.ring_matvec(d, A, 5, n, S, r), P.matvec(A, 5, n, S, r))
    Phi = _words(rng, q, (r, n, d))
    assert np.array_equal(F.ring_garbage_h(d, S, Phi, r, n), P.garbage_h(S, Phi, r, n))
    c = _words(rng, q, (r, d))
    assert np.array_equal(F.ring_amortize(d, S, c, r, n), P.amortize(S, c, r, n))


@pytest.mark.parametrize("q", [LABRADOR_Q, SMALL_Q, Q])
def test_ring_garbage_h_and_amortize_term_by_term(oracle, q):
    F = oracle.Field(q)
    d, r, n = 16, 3, 4
    rng = np.random.default_rng(11)
    S = _words(rng, q, (r, n, d))
    Phi = _words(rng, q, (r, n, d))
    two_inv = int(F.to_mont([q // 2 + 1])[0])
    H = F.ring_garbage_h(d, S, Phi, r, n).reshape(-1, d)
    idx = 0
    for i in range(r):
        for j in range(i, r):
            t1 = np.zeros(d, np.uint32)
            t2 = np.zeros(d, np.uint32)
            for k in range(n):
                t1 = F.add_slice(t1, F.naive_negacyclic(Phi[i, k], S[j, k]))
                t2 = F.add_slice(t2, F.naive_negacyclic(Phi[j, k], S[i, k]))
            assert np.array_equal(H[idx], F.scalar_mul_slice(F.add_slice(t1, t2), two_inv))
            idx += 1
    c = _words(rng, q, (r, d))
    Z = F.ring_amortize(d, S, c, r, n).reshape(n, d)
    for k in range(n):
        want = np.zeros(d, np.uint32)
        for i in range(r):
            want = F.add_slice(want, F.naive_negacyclic(c[i], S[i, k]))
        assert np.array_equal(Z[k], want)


@pytest.mark.parametrize("q", [17, 12289, LABRADOR_Q, Q])
def test_slice_hooks_match_python_integers(oracle, q):
    F = oracle.Field(q)
    rng = np.random.default_rng(q % 97)
    n = 300
    a = _words(rng, q, n)
    b = _words(rng, q, n)
    a[:3] = [0, 1, q - 1]
    b[:3] = [q - 1, q - 1, q - 1]
    sc = int(_words(rng, q, 1)[0])
    rinv = pow(2 ** 32, -1, q)
    ai, bi = [int(x) for x in a], [int(x) for x in b]
    assert [int(x) for x in F.add_slice(a, b)] == [(x + y) % q for x, y in zip(ai, bi)]
    assert [int(x) for x in F.sub_slice(a, b)] == [(x - y) % q for x, y in zip(ai, bi)]
    assert [int(x) for x in F.scalar_mul_slice(a, sc)] == [x * sc * rinv % q for x in ai]
    assert [int(x) for x in F.pointwise_mul_slice(a, b)] == [x * y * rinv % q
                                                             for x, y in zip(ai, bi)]
    assert [int(x) for x in F.add_scaled_slice(a, b, sc)] == [
        (x + y * sc * rinv) % q for x, y in zip(ai, bi)]
    assert F.dot_product(a, b) == sum(x * y for x, y in zip(ai, bi)) * rinv % q
