"""CPU checks of the verifier restatement (oracle/labrador_verify.py) on a level
the oracle itself proves: honest outputs pass verify_all's equations and the
b'' check, and a changed word of any message is rejected. This pins the
restatement before it judges the GPU's outputs."""
import numpy as np
import pytest

Q = 4294966657


def _mont(q, values):
    v = (np.asarray(values, dtype=np.int64) % q).astype(np.uint64)
    return ((v * np.uint64(1 << 16)) % np.uint64(q) * np.uint64(1 << 16) % np.uint64(q)).astype(np.uint32)


def _honest_level(oracle, r=5, n=12, kappa=3, k1=2, k2=2, seed=3):
    q, d = Q, 64
    b1 = b2 = 256
    t1 = t2 = 4
    gar = r * (r + 1) // 2
    P = oracle.Plan(q, d)
    F = P.field
    rng = np.random.default_rng(seed)
    S = _mont(q, rng.integers(-2048, 2049, (r, n, d)))
    rand = lambda *shape: rng.integers(0, q, shape, dtype=np.uint64).astype(np.uint32)
    A, B, C, D = rand(kappa, n, d), rand(k1, r * kappa * t1, d), rand(k1, gar * t2, d), \
        rand(k2, gar * t1, d)
    phis = rand(r, n, d)
    challenges = _mont(q, rng.integers(-2, 3, (r, d)))
    t_limbs = oracle.decompose_polys(F, d, P.matvec(A, kappa, n, S, r), b1, t1)
    g_limbs = oracle.decompose_polys(F, d, P.gram(S, r, n), b2, t2)
    h_limbs = oracle.decompose_polys(F, d, P.garbage_h(S, phis, r, n), b1, t1)
    z = P.amortize(S, challenges, r, n)
    u1 = F.add_slice(P.matvec(B, k1, r * kappa * t1, t_limbs, 1),
                     P.matvec(C, k1, gar * t2, g_limbs, 1))
    u2 = P.matvec(D, k2, gar * t1, h_limbs, 1)
    return dict(A=A, B=B, C=C, D=D, u1=u1, u2=u2, z=z, challenges=challenges, t_limbs=t_limbs,
                g_limbs=g_limbs, h_limbs=h_limbs, phis=phis, r=r, n=n, kappa=kappa, b1=b1,
                t1=t1, b2=b2, t2=t2)


def test_verifier_accepts_an_honest_level_and_rejects_changes(oracle):
    from oracle.labrador_verify import VerifyError, verify_all
    level = _honest_level(oracle)
    verify_all(Q, 64, gamma=float(2 ** 30), **level)
    for name in ("t_limbs", "g_limbs", "h_limbs", "z", "u1", "u2", "challenges"):
        bad = dict(level)
        arr = np.array(bad[name], dtype=np.uint32, copy=True).reshape(-1)
        arr[arr.size // 3] = (int(arr[arr.size // 3]) + 1) % Q
        bad[name] = arr
        with pytest.raises(VerifyError):
            verify_all(Q, 64, **bad)
    short = dict(level)
    short["t_limbs"] = level["t_limbs"][:-64]
    with pytest.raises(VerifyError, match="shape"):
        verify_all(Q, 64, **short)
    with pytest.raises(VerifyError, match="2b"):
        verify_all(Q, 64, gamma=1.0, **level)


def test_limb_reconstruction_matches_oracle(oracle):
    from oracle.labrador_verify import EvalRing, reconstruct_from_limbs
    F = oracle.Field(Q)
    rng = np.random.default_rng(8)
    polys = rng.integers(0, Q, (7, 64), dtype=np.uint64).astype(np.uint32)
    limbs = oracle.decompose_polys(F, 64, polys, 256, 4)
    rec = reconstruct_from_limbs(EvalRing(Q, 64), limbs, 7, 4, 256)
    assert np.array_equal(rec.astype(np.uint32), polys)
    for i in range(7):
        assert np.array_equal(oracle.reconstruct_from_limbs(F, 64, limbs[i * 256:(i + 1) * 256], 256),
                              polys[i])


def test_b_double_prime_check(oracle):
    from oracle.labrador_verify import VerifyError, verify_b_double_prime
    q = Q
    rng = np.random.default_rng(2)
    p = [int(x) for x in rng.integers(0, q, 256)]
    b0 = [int(x) for x in rng.integers(0, q, 3)]
    psi = rng.integers(0, q, (2, 3))
    omega = rng.integers(0, q, (2, 256))
    ct = [(sum(int(a) * b for a, b in zip(psi[k], b0)) + sum(int(o) * x for o, x in zip(omega[k], p)))
          % q for k in range(2)]
    verify_b_double_prime(q, ct, psi, omega, p, b0)
    with pytest.raises(VerifyError):
        verify_b_double_prime(q, [ct[0], (ct[1] + 1) % q], psi, omega, p, b0)
