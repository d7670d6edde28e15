"""Ring plans for moduli without a 2d-th root of unity, against the oracle's
schoolbook products (the reference's path for such q,
naive_negacyclic_mul_coeffs, algebra/src/poly/ring.rs:60-77): single products,
commitments, linear and BDLOP commitments, the Gram matrix, garbage h, the
amortized witness and the fused prover round, for the reference's own LaBRADOR
moduli 2^32 - 5 and 12281, bit-exact; up to the prover round at r = 64,
n = 2048, kappa = 16 for 2^32 - 5."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LABRADOR_Q = 4294967291  # 2^32 - 5 (labrador/src/params/builder.rs)
SMALL_Q = 12281          # examples/fibonacci_round_trip.rs
Q = 4294966657           # NTT-friendly: a ring plan is the ordinary plan


def _rand(q, shape, seed, edge=True):
    rng = np.random.default_rng(seed)
    x = rng.integers(0, q, shape, dtype=np.uint64).astype(np.uint32)
    if edge:
        flat = x.reshape(-1)
        flat[: min(flat.size, 70)] = q - 1  # largest words: the largest integer sums
    return x


def _mont(q, values):
    """Signed integers -> Montgomery words v * 2^32 mod q (two exact 16-bit steps)."""
    v = (np.asarray(values, dtype=np.int64) % q).astype(np.uint64)
    return ((v * np.uint64(1 << 16)) % np.uint64(q) * np.uint64(1 << 16) % np.uint64(q)).astype(np.uint32)


def _dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).to(cuda)


def _host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("q", [LABRADOR_Q, SMALL_Q])
def test_ring_plan_kind_and_ntt_refusal(cuda, q):
    import ctypes as C
    from lattica_b200 import _lib
    from lattica_b200.ntt import NttError, RingPlan, TwistedNttPlan
    lib = _lib.load()
    with pytest.raises(NttError) as ei:
        TwistedNttPlan(q, 64)
    plan = RingPlan(q, 64)
    assert plan.uses_aux_primes
    aux = (C.c_uint32 * 3)()
    kind = C.c_int()
    assert lib.grid_gpu_plan_ring_kind(plan.handle, C.byref(kind), aux) == 0
    assert kind.value == 1 and list(aux) == [4294962689, 4294957057, 4294955009]
    x = _dev(_rand(q, (4, 64), 1), cuda)
    with pytest.raises(NttError) as ej:
        plan.forward_in_place(x)
    assert ej.value.kind == ei.value.kind
    assert not RingPlan(Q, 64).uses_aux_primes
    plan.check_device()


@pytest.mark.parametrize("q,d,n", [(LABRADOR_Q, 64, 300), (SMALL_Q, 64, 5), (LABRADOR_Q, 16, 33),
                                   (LABRADOR_Q, 256, 17), (LABRADOR_Q, 8, 1)])
def test_ring_products_match_schoolbook(cuda, oracle, q, d, n):
    from lattica_b200.ntt import RingPlan
    plan = RingPlan(q, d)
    F = oracle.Field(q)
    a = _rand(q, (n, d), n)
    b = _rand(q, (n, d), n + 1)
    want = np.stack([F.naive_negacyclic(a[i], b[i]) for i in range(n)])
    ta = _dev(a, cuda)
    plan.multiply_in_place(ta, _dev(b, cuda))
    assert np.array_equal(_host(ta), want)
    ha = a.copy()
    plan.multiply_in_place(ha, b)  # host-buffer path
    assert np.array_equal(ha, want)
    plan.check_device()


@pytest.mark.parametrize("q,rows,cols,batch", [(LABRADOR_Q, 8, 64, 64), (LABRADOR_Q, 16, 300, 6),
                                               (SMALL_Q, 3, 40, 5), (LABRADOR_Q, 1, 2, 1),
                                               (LABRADOR_Q, 33, 70, 3)])
def test_ring_commit_matches_schoolbook(cuda, oracle, q, rows, cols, batch):
    from lattica_b200.commit import PreparedMatrix
    from lattica_b200.ntt import RingPlan
    d = 64
    plan = RingPlan(q, d)
    F = oracle.Field(q)
    A = _rand(q, (rows, cols, d), rows + cols)
    s = _rand(q, (batch, cols, d), batch)
    want = F.ring_matvec(d, A, rows, cols, s, batch).reshape(batch, rows, d)
    M = PreparedMatrix(plan, _dev(A, cuda), rows, cols)
    assert np.array_equal(_host(M.mul_vec(_dev(s, cuda))), want)
    M2 = PreparedMatrix(plan, A, rows, cols)  # host-buffer create and commit
    assert np.array_equal(M2.mul_vec(s), want)
    plan.check_device()


def test_ring_linear_and_bdlop_commits_match_schoolbook(cuda, oracle):
    from lattica_b200.commit import BdlopCommitmentKey, CommitmentDimensions, LinearCommitmentKey
    from lattica_b200.ntt import RingPlan
    q, d = LABRADOR_Q, 64
    plan = RingPlan(q, d)
    F = oracle.Field(q)
    rows, mc, oc, batch = 4, 6, 5, 3
    a_msg, a_open = _rand(q, (rows, mc, d), 1), _rand(q, (rows, oc, d), 2)
    a_mask = _rand(q, (rows, oc, d), 3)
    m, r = _rand(q, (batch, mc, d), 4), _rand(q, (batch, oc, d), 5)
    t_msg = F.ring_matvec(d, a_msg, rows, mc, m, batch)
    t_open = F.ring_matvec(d, a_open, rows, oc, r, batch)
    want_v = F.add_slice(t_msg, t_open).reshape(batch, rows, d)
    key = LinearCommitmentKey(plan, a_msg, a_open, CommitmentDimensions(mc, oc, rows))
    for i in range(batch):
        assert np.array_equal(key.recompute(m[i], r[i]).reshape(rows, d), want_v[i])
    bd = BdlopCommitmentKey(plan, _dev(a_mask, cuda), _dev(a_msg, cuda), _dev(a_open, cuda),
                            rows, mc, oc)
    u, v = bd.recompute_parts(_dev(m, cuda), _dev(r, cuda))
    assert np.array_equal(_host(v).reshape(batch, rows, d), want_v)
    want_u = F.ring_matvec(d, a_mask, rows, oc, r, batch).reshape(batch, rows, d)
    assert np.array_equal(_host(u).reshape(batch, rows, d), want_u)
    plan.check_device()


@pytest.mark.parametrize("q,r,n", [(LABRADOR_Q, 5, 130), (LABRADOR_Q, 16, 77), (SMALL_Q, 9, 20),
                                   (LABRADOR_Q, 64, 40), (LABRADOR_Q, 1, 1)])
def test_ring_gram_garbage_h_amortize_match_schoolbook(cuda, oracle, q, r, n):
    from lattica_b200.labrador import amortize_witness, compute_garbage_g, compute_garbage_h
    from lattica_b200.ntt import RingPlan
    d = 64
    plan = RingPlan(q, d)
    F = oracle.Field(q)
    S = _rand(q, (r, n, d), r * n)
    Phi = _rand(q, (r, n, d), r * n + 1)
    c = _rand(q, (r, d), r + 2)
    assert np.array_equal(_host(compute_garbage_g(plan, _dev(S, cuda))).reshape(-1),
                          F.ring_gram(d, S, r, n))
    assert np.array_equal(compute_garbage_g(plan, S).reshape(-1), F.ring_gram(d, S, r, n))
    assert np.array_equal(_host(compute_garbage_h(plan, _dev(S, cuda), _dev(Phi, cuda))).reshape(-1),
                          F.ring_garbage_h(d, S, Phi, r, n))
    assert np.array_equal(_host(amortize_witness(plan, _dev(S, cuda), _dev(c, cuda))).reshape(-1),
                          F.ring_amortize(d, S, c, r, n))
    plan.check_device()


def _round_check(cuda, oracle, q, r, n, kappa, seed_words):
    import torch
    from lattica_b200.labrador import CommitKey, prover_round_dev, verify_norm
    from lattica_b200.ntt import RingPlan
    d = 64
    plan = RingPlan(q, d)
    F = oracle.Field(q)
    rng = np.random.default_rng(seed_words)
    bound = min(1 << 11, q // 4)
    coeffs = rng.integers(-bound, bound + 1, (r, n, d))
    S = _mont(q, coeffs)
    A = _rand(q, (kappa, n, d), seed_words + 1)
    seed = bytes((3 * i + seed_words) & 0xFF for i in range(32))
    key = CommitKey(plan, A, kappa, n)
    base = 256 if q > 1 << 20 else 16  # base^4 covers q
    limbs = 4
    out = prover_round_dev(key, _dev(S, cuda), base, limbs, base, limbs, seed, 256)
    torch.cuda.synchronize()
    t = F.ring_matvec(d, A, kappa, n, S, r)
    g = F.ring_gram(d, S, r, n)
    assert np.array_equal(_host(out.t_limbs).reshape(-1),
                          oracle.decompose_polys(F, d, t, base, limbs))
    assert np.array_equal(_host(out.g).reshape(-1), g)
    assert np.array_equal(_host(out.g_limbs).reshape(-1),
                          oracle.decompose_polys(F, d, g, base, limbs))
    p, _ = oracle.jl_project(F, seed, 256, S.reshape(r, n * d), r, n * d, d, want_flat=False)
    assert np.array_equal(_host(out.p), p)
    if q > 1 << 31:  # p does not wrap mod q: the JL norm gate applies
        s_norm = float(np.sqrt(np.sum(coeffs.astype(np.float64) ** 2)))
        assert verify_norm(_host(out.p), q, 1.5 * s_norm)
    plan.check_device()


@pytest.mark.parametrize("q", [LABRADOR_Q, SMALL_Q])
def test_ring_prover_round_matches_schoolbook(cuda, oracle, q):
    _round_check(cuda, oracle, q, 6, 64, 4, 17)


def test_ring_prover_round_at_round_size(cuda, oracle):
    """r = 64, n = 2048, kappa = 16 with q = 2^32 - 5: every word against the
    oracle's schoolbook products (~26 G word products on the host cores)."""
    _round_check(cuda, oracle, LABRADOR_Q, 64, 2048, 16, 29)


def test_ring_plan_refuses_what_needs_evaluations(cuda):
    import ctypes as C
    from lattica_b200 import _lib
    from lattica_b200.commit import PreparedMatrix
    from lattica_b200.ntt import NttError, RingPlan
    lib = _lib.load()
    plan = RingPlan(LABRADOR_Q, 64)
    A = np.zeros((2, 3, 64), np.uint32)
    with pytest.raises(NttError):
        PreparedMatrix(plan, A, 2, 3, is_evals=True)
    M = PreparedMatrix(plan, A, 2, 3)
    ev = C.c_void_p()
    assert lib.grid_gpu_matrix_device_evals(M.handle, C.byref(ev)) in (3, 4)
    items = (_lib.BatchItem * 1)(_lib.BatchItem(0, 0, 3, 0))
    hs = (C.c_void_p * 1)(M.handle.value)
    b = C.c_void_p()
    assert lib.grid_gpu_batch_create(plan.handle, hs, 1, items, 1, C.byref(b)) in (3, 4)
    z = np.zeros(64, np.uint32)
    assert lib.grid_gpu_plan_get_twiddles(plan.handle, z.ctypes.data, z.ctypes.data) in (3, 4)
    # the exactness bound: 2^24 terms of d = 64 products of words near 2^32 reach
    # 2^93 (2^23 stay below); rejected before any device memory is touched
    nb = C.c_size_t()
    assert lib.grid_gpu_gram_workspace(plan.handle, 1, 1 << 24, C.byref(nb)) == 0
    assert lib.grid_gpu_gram_dev(plan.handle, 16, 1, 1 << 24, 16, 16, 0, None) == 5
