"""The AVX2 restatement of the reference's x86 NTT path (oracle/oracle_avx2.c,
the timed CPU baseline) gives the scalar oracle's words exactly: both moduli
branches of the Montgomery reduction (q >= 2^31 and q < 2^31), degrees whose
stages are all vector, mixed or all scalar, and edge words."""
import numpy as np
import pytest

Q, Q256 = 4294966657, 4294962689


@pytest.mark.parametrize("q,d", [(Q, 64), (Q, 8), (Q256, 256), (12289, 64), (12289, 512),
                                 (17, 8), (Q, 16)])
def test_avx2_port_matches_scalar_oracle(oracle, q, d):
    P = oracle.Plan(q, d)
    rng = np.random.default_rng(d + q % 1000)
    count = 37
    a = rng.integers(0, q, count * d, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, q, count * d, dtype=np.uint64).astype(np.uint32)
    edge = np.array([0, 1, q - 1, q // 2, q // 2 + 1, q - 2], dtype=np.uint32)
    a[:edge.size] = edge
    b[d:d + edge.size] = edge
    a[2 * d:3 * d] = q - 1                     # all-(q-1) polynomial
    b[2 * d:3 * d] = q - 1
    want = P.ntt_mul_inverse(a, b)
    assert np.array_equal(P.ntt_mul_inverse(a, b, avx2=True), want)
    assert np.array_equal(P.ntt_mul_inverse(a, b, threads=4, avx2=True), want)


@pytest.mark.parametrize("q,d,rows,cols,batch", [(Q, 64, 8, 64, 5), (Q, 64, 3, 7, 2),
                                                 (12289, 64, 5, 9, 3), (Q256, 256, 4, 10, 2),
                                                 (17, 8, 2, 9, 3)])
def test_avx2_prepared_commit_matches_scalar_oracle(oracle, q, d, rows, cols, batch):
    P = oracle.Plan(q, d)
    rng = np.random.default_rng(rows * 31 + cols)
    A = rng.integers(0, q, rows * cols * d, dtype=np.uint64).astype(np.uint32)
    s = rng.integers(0, q, batch * cols * d, dtype=np.uint64).astype(np.uint32)
    A[:4] = [0, 1, q - 1, q - 2]
    want = P.matvec(A, rows, cols, s, batch)
    assert np.array_equal(P.matvec(A, rows, cols, s, batch, threads=3, avx2=True), want)
    a_hat = P.forward(A.reshape(rows * cols, d)).reshape(-1)   # cached evaluations
    assert np.array_equal(P.matvec(a_hat, rows, cols, s, batch, a_is_eval=True, threads=1,
                                   avx2=True), want)
