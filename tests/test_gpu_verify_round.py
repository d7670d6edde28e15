"""The verifier's checks on a prover level whose hot calls ran on the GPU, at the
LaBRADOR round's size (r = 64, n = 2048, kappa = kappa1 = kappa2 = 16, base 2^8
with 4 limbs): the GPU's t limbs, g limbs, p and JL evaluations from one fused
round, the GPU's garbage h and its limbs, the GPU's amortized witness z and the
GPU's outer commitments u1, u2 pass the restated verify_all equations (1), (2a),
(2b), (3a), (3b), (4), the limb-shortness and shape checks, the b'' constant-term
check and the JL norm gate (oracle/labrador_verify.py); one flipped limb, one
changed word of z, g or p is rejected."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

Q = 4294966657


def _mont(q, values):
    v = (np.asarray(values, dtype=np.int64) % q).astype(np.uint64)
    return ((v * np.uint64(1 << 16)) % np.uint64(q) * np.uint64(1 << 16) % np.uint64(q)).astype(np.uint32)


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def _dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).to(cuda)


def test_gpu_level_passes_verifier_and_tampering_is_rejected(cuda):
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import (CommitKey, OuterCommitKey, amortize_witness,
                                       compute_garbage_h, decompose_polys, prover_round_dev,
                                       verify_norm)
    from oracle.labrador_verify import VerifyError, verify_all, verify_b_double_prime
    q, d, r, n, kappa, k1, k2 = Q, 64, 64, 2048, 16, 16, 16
    b1 = b2 = 256
    t1 = t2 = 4
    gar = r * (r + 1) // 2
    plan = TwistedNttPlan(q, d)
    rng = np.random.default_rng(31)
    coeffs = rng.integers(-(1 << 11), (1 << 11) + 1, (r, n, d))
    S = _mont(q, coeffs)
    rand = lambda *shape: rng.integers(0, q, shape, dtype=np.uint64).astype(np.uint32)
    A, B, C, D = rand(kappa, n, d), rand(k1, r * kappa * t1, d), rand(k1, gar * t2, d), \
        rand(k2, gar * t1, d)
    seed = bytes((13 * i + 5) & 0xFF for i in range(32))
    key = CommitKey(plan, A, kappa, n)
    S_dev = _dev(S, cuda)
    out = prover_round_dev(key, S_dev, b1, t1, b2, t2, seed, 256, jl_evals=True)
    # garbage h over aggregated phis, its limbs; amortized witness; outer commitments
    phis = rand(r, n, d)
    challenges = _mont(q, rng.integers(-2, 3, (r, d)))  # small challenge polynomials
    h = compute_garbage_h(plan, S_dev, _dev(phis, cuda))
    h_limbs = decompose_polys(plan, _host(h), b1, t1).flat
    z = amortize_witness(plan, S_dev, _dev(challenges, cuda))
    outer = OuterCommitKey(plan, B, C, D, k1, k2, r * kappa * t1, gar * t2, gar * t1)
    u1 = outer.outer_commit_u1_slice(out.t_limbs, out.g_limbs)
    u2 = outer.outer_commit_u2_slice(_dev(h_limbs, cuda))
    torch.cuda.synchronize()
    level = dict(A=A, B=B, C=C, D=D, u1=_host(u1), u2=_host(u2), z=_host(z),
                 challenges=challenges, t_limbs=_host(out.t_limbs), g_limbs=_host(out.g_limbs),
                 h_limbs=h_limbs, phis=phis, r=r, n=n, kappa=kappa, b1=b1, t1=t1, b2=b2, t2=t2)
    # ||z|| for small challenges: at most 2 * r * 2^11 * d per coefficient, loose gamma
    verify_all(q, d, gamma=float(2 ** 40), **level)

    # b'' constant terms against p: b''_k = sum_m omega_km conj(pi_m) s (F' empty)
    rinv = pow(1 << 32, -1, q)
    val = lambda w: int(w) * rinv % q
    p_vals = [val(w) for w in _host(out.p)]
    ev0 = [val(w) for w in _host(out.jl_evals)[:, 0]]
    omega = rng.integers(0, q, (4, 256), dtype=np.uint64)
    bdp_ct = [sum(int(om) * e for om, e in zip(omega[k], ev0)) % q for k in range(4)]
    verify_b_double_prime(q, bdp_ct, [[] for _ in range(4)], omega, p_vals, [])
    s_norm = float(np.sqrt(np.sum(coeffs.astype(np.float64) ** 2)))
    assert verify_norm(_host(out.p), q, 1.5 * s_norm)

    # one changed word anywhere is rejected
    def tampered(name, index, delta=1):
        bad = dict(level)
        arr = np.array(bad[name], dtype=np.uint32, copy=True).reshape(-1)
        arr[index] = (int(arr[index]) + delta) % q
        bad[name] = arr
        return bad

    for name, index in (("t_limbs", 12345), ("g_limbs", 777), ("h_limbs", 4242), ("z", 99),
                        ("u1", 5), ("u2", 17)):
        with pytest.raises(VerifyError):
            verify_all(q, d, **tampered(name, index))
    with pytest.raises(VerifyError, match="shortness"):  # a limb far outside [-b/2, b/2]
        verify_all(q, d, **tampered("t_limbs", 3, delta=1 << 20))
    bad_p = list(p_vals)
    bad_p[7] = (bad_p[7] + 1) % q
    with pytest.raises(VerifyError):
        verify_b_double_prime(q, bdp_ct, [[] for _ in range(4)], omega, bad_p, [])
    plan.check_device()
