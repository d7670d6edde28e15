"""Parity at the configurations' own sizes, where the kernels pick geometries
(split K, tensor-core tiles, fused JL entries) that small cases never reach.

* The LaBRADOR prover round at r = 64, n = 2048, kappa = 16 (every word of the
  t limbs, g, g limbs and p; sampled rows of the 2 GiB JL entries) and the
  checks verify_step applies to those outputs.
* The tensor-core contractions' int32 bound: one CTA accumulates at most 8192
  K words, D_l = sum_{k,i} byte_i(x_k) byte_l(2^(8i) y_k mod q) < 4 * 8192 *
  255^2 = 2,130,739,200 < 2^31. Words are chosen so that one byte plane comes
  within 1.2 % of 2^31 at exactly 8192 words per CTA, and past it (the split
  boundary: one word, which only the gathering kernel takes, K not a multiple
  of 4; four words, a last range of one partial chunk), on the point-major
  kernel and on the gathering one.
* The uneven batch (4096 instances, n log-uniform in [64, 8192]) at full size,
  32 instances against the oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

Q = 4294966657
R_INV = pow(1 << 32, -1, Q)


def _dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).to(cuda)


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def _mont(q, values):
    """Signed integers -> Montgomery words v * 2^32 mod q (two exact 16-bit steps)."""
    v = (np.asarray(values, dtype=np.int64) % q).astype(np.uint64)
    return ((v * np.uint64(1 << 16)) % np.uint64(q) * np.uint64(1 << 16) % np.uint64(q)).astype(np.uint32)


def test_prover_round_at_round_size_matches_oracle(cuda, oracle):
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import CommitKey, prover_round_dev, verify_norm
    q, d, r, n, kappa = Q, 64, 64, 2048, 16
    plan = TwistedNttPlan(q, d)
    P = oracle.Plan(q, d)
    F = P.field
    rng = np.random.default_rng(2048)
    coeffs = rng.integers(-(1 << 11), (1 << 11) + 1, (r, n, d))
    S = _mont(q, coeffs).reshape(r, n, d)
    A = rng.integers(0, q, (kappa, n, d), dtype=np.uint64).astype(np.uint32)
    seed = bytes((11 * i + 3) & 0xFF for i in range(32))
    key = CommitKey(plan, A, kappa, n)
    out = prover_round_dev(key, _dev(S, cuda), 256, 4, 256, 4, seed, 256, extract=True)
    torch.cuda.synchronize()
    t = P.matvec(A, kappa, n, S, r, threads=0)
    g = P.gram(S, r, n, threads=0)
    assert np.array_equal(_host(out.t_limbs).reshape(-1),
                          oracle.decompose_polys(F, d, t, 256, 4))
    assert np.array_equal(_host(out.g).reshape(-1), g)
    assert np.array_equal(_host(out.g_limbs).reshape(-1), oracle.decompose_polys(F, d, g, 256, 4))
    p, flat = oracle.jl_project(F, seed, 256, S.reshape(r, n * d), r, n * d, d)
    assert np.array_equal(_host(out.p), p)
    plane = r * n * d
    for row in (0, 1, 63, 64, 127, 128, 200, 254, 255):
        got = out.jl_flat[row * plane:(row + 1) * plane].cpu().numpy()
        assert np.array_equal(got, flat[row * plane:(row + 1) * plane]), row
    del flat
    # what verify_step checks on these words: limbs reconstruct to t and g,
    # and p passes the JL norm gate above the witness norm, not below it
    tl, gl = _host(out.t_limbs), _host(out.g_limbs)
    tt, gg = t.reshape(-1, d), g.reshape(-1, d)
    for i in range(0, tt.shape[0], 37):
        assert np.array_equal(oracle.reconstruct_from_limbs(F, d, tl[4 * i:4 * i + 4], 256), tt[i])
    for i in range(0, gg.shape[0], 53):
        assert np.array_equal(oracle.reconstruct_from_limbs(F, d, gl[4 * i:4 * i + 4], 256), gg[i])
    s_norm = float(np.sqrt(np.sum(coeffs.astype(np.float64) ** 2)))
    assert verify_norm(_host(out.p), q, 1.5 * s_norm)
    assert not verify_norm(_host(out.p), q, 0.5 * s_norm)
    plan.check_device()


def _const_polys(word, count, d=64):
    x = np.zeros((count, d), np.uint32)
    x[:, 0] = word  # a constant polynomial: every twisted evaluation is the word itself
    return x


def _k_per_cta_8192(cuda, groups):
    """K at which the contraction gives every CTA exactly 8192 words: the
    gathering geometry splits K over num_sms // groups CTAs per evaluation
    group; the point-major one caps every range at 8192 words, fewer ranges
    than this K needs (2 num_sms / 64 per point)."""
    import torch
    sms = torch.cuda.get_device_properties(cuda).multi_processor_count
    return max(1, sms // groups) * 8192


def _plan(gather):
    import os
    from lattica_b200 import TwistedNttPlan
    if not gather:
        return TwistedNttPlan(Q, 64)
    os.environ["GRID_GPU_CONTRACTION"] = "gather"
    try:
        return TwistedNttPlan(Q, 64)
    finally:
        del os.environ["GRID_GPU_CONTRACTION"]


@pytest.mark.parametrize("gather", [False, True])
@pytest.mark.parametrize("extra", [0, 1, 4])
def test_contraction_bound_commit_at_8192_words_per_cta(cuda, extra, gather):
    """t = A s with every evaluation of s equal to x = 0xFEFFFFFF (bytes FF FF FF
    FE) and of A equal to y = 0xFEFEFD82, whose byte-3 plane sums to 99.6 % of
    4 * 255^2 per word: 98.8 % of 2^31 in each CTA."""
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.commit import PreparedMatrix
    x, y = 0xFEFFFFFF, 0xFEFEFD82
    plan_sc = [(y * pow(2, 8 * i, Q)) % Q for i in range(4)]
    plane3 = sum(((x >> (8 * i)) & 255) * ((plan_sc[i] >> 24) & 255) for i in range(4))
    assert plane3 * 8192 > 0.988 * 2 ** 31 and 4 * 8192 * 255 ** 2 < 2 ** 31
    rows, batch = 16, 8          # Y rows <= 16: 4 evaluation points per CTA, 16 groups
    K = _k_per_cta_8192(cuda, 16) + extra
    plan = _plan(gather)
    A = _dev(_const_polys(y, rows * K), cuda).view(rows, K, 64)
    M = PreparedMatrix(plan, A, rows, K)
    del A
    s = _dev(_const_polys(x, batch * K), cuda).view(batch, K, 64)
    t = M.mul_vec(s)
    torch.cuda.synchronize()
    want = np.zeros((batch, rows, 64), np.uint32)
    want[:, :, 0] = K * (x * y * R_INV % Q) % Q
    assert np.array_equal(_host(t), want)
    plan.check_device()


@pytest.mark.parametrize("gather", [False, True])
@pytest.mark.parametrize("extra", [0, 1, 4])
def test_contraction_bound_gram_at_8192_words_per_cta(cuda, extra, gather):
    """Gram (X = Y) with every evaluation equal to c = 3488348921, the word whose
    largest byte plane is highest among 4 * 10^7 sampled words (89 % of 2^31 per
    CTA)."""
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import compute_garbage_g
    c = 3488348921
    r = 16
    K = _k_per_cta_8192(cuda, 16) + extra
    plan = _plan(gather)
    S = _dev(_const_polys(c, r * K), cuda).view(r, K, 64)
    g = compute_garbage_g(plan, S)
    torch.cuda.synchronize()
    want = np.zeros((r * (r + 1) // 2, 64), np.uint32)
    want[:, 0] = K * (c * c * R_INV % Q) % Q
    assert np.array_equal(_host(g), want)
    plan.check_device()


def test_uneven_batch_full_size_sampled_against_oracle(cuda, oracle):
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.batch import UnevenCommitBatch, sample_uneven_instances
    from lattica_b200.commit import PreparedMatrix
    q, d, ranks = Q, 64, (8, 16, 32)
    plan = TwistedNttPlan(q, d)
    rng = np.random.default_rng(4096)
    mats_host = [rng.integers(0, q, (m, 8192, d), dtype=np.uint64).astype(np.uint32)
                 for m in ranks]
    mats = [PreparedMatrix(plan, _dev(A, cuda), A.shape[0], 8192) for A in mats_host]
    items, s_polys, t_polys = sample_uneven_instances(4096, 7)
    g = torch.Generator(device=cuda).manual_seed(3)
    s = ((torch.randint(-1, 2, (s_polys, d), dtype=torch.int64, device=cuda, generator=g) % q)
         * ((1 << 32) % q) % q).to(torch.int32)
    t = torch.zeros((t_polys, d), dtype=torch.int32, device=cuda)
    batch = UnevenCommitBatch(plan, mats, items)
    batch.commit_dev(s, t)
    torch.cuda.synchronize()
    P = oracle.Plan(q, d)
    order = sorted(range(len(items)), key=lambda i: items[i][2])
    pick = sorted(set([order[0], order[-1]] + order[:: len(order) // 30][:30]))
    assert max(items[i][2] for i in pick) > 7000
    for i in pick:
        so, to, nn, m = items[i]
        rows = ranks[m]
        want = P.matvec(np.ascontiguousarray(mats_host[m][:, :nn]), rows, nn,
                        _host(s[so:so + nn]), 1).reshape(rows, d)
        assert np.array_equal(_host(t[to:to + rows]), want), (i, nn, rows)
    plan.check_device()
