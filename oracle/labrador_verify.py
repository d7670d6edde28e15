"""Restatement of the LaBRADOR verifier's checks on one prover level
(TEST INFRASTRUCTURE ONLY: used by tests/ to decide whether outputs the GPU
produced would be accepted; nothing in lattica_b200/ imports it).

Restated from the reference:
  * verify_all (labrador/src/main_protocol/verify_equations.rs:271-344):
    shape validation (:59-209), limb shortness (:30-55), equation (1)
    u1 = B t + C g (:347-365), (2a) A z = sum_i c_i t_i with t reconstructed from
    its limbs (:368-394, reconstruct_t_vecs main_protocol/mod.rs:702-727),
    (2b) ||z|| <= gamma (:397-414), (3a) <z, z> = sum g_ij c_i c_j (:417-450),
    (3b) sum_i <phi_i, z> c_i = sum h_ij c_i c_j (:453-491) and (4) u2 = D h
    (:531-548). Equation (3c) and the opening-norm bounds need the statement's
    a_ij / b and the parameter set's gamma1 / gamma2, which a prover level's
    hot path does not produce; they are not restated.
  * verify_b_double_prime (labrador/src/main_protocol/aggregation.rs:143-181):
    the constant terms of b'' against psi, omega, p and the F' constants.
  * The JL norm gate is lattica_b200.labrador.verify_norm (jl.rs:533-547).

Ring arithmetic runs in the oracle's twisted evaluation domain with numpy
(Montgomery words; a product is a * b * 2^-32 mod q, exact in uint64), the same
field elements as the reference's coefficient-domain products. The modulus must
have an NTT for the ring degree (the oracle's Plan).
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


class VerifyError(AssertionError):
    """A check of the verifier failed (the reference returns Err(String))."""


class EvalRing:
    """R_q in the evaluation domain: polys (..., d) of Montgomery words."""

    def __init__(self, q: int, d: int):
        self.P = O.Plan(q, d)
        self.q, self.d = q, d
        self.rinv = np.uint64(pow(1 << 32, -1, q))
        self.Q = np.uint64(q)

    def evals(self, polys):
        a = np.ascontiguousarray(polys, dtype=np.uint32).reshape(-1, self.d)
        return self.P.forward(a).reshape(a.shape).astype(np.uint64)

    def mul(self, a, b):
        return (a * b % self.Q) * self.rinv % self.Q

    def dot(self, a, b, axis):
        """sum over `axis` of the products a * b (both broadcast), mod q."""
        return (self.mul(a, b) % self.Q).sum(axis=axis, dtype=np.uint64) % self.Q

    def scale(self, a, k: int):
        """a times the integer k (Montgomery words are linear)."""
        return a * np.uint64(k % self.q) % self.Q


def reconstruct_from_limbs(ring: EvalRing, flat, num_polys: int, num_limbs: int, base: int):
    """reconstruct_from_limbs (main_protocol/mod.rs:331-359) of every poly of a
    DecomposedPolys: sum_k limb_k * base^k, limbs stored as residues. Returns
    coefficient-domain Montgomery words (num_polys, d), uint64."""
    limbs = np.asarray(flat, dtype=np.uint64).reshape(num_polys, num_limbs, ring.d)
    acc = np.zeros((num_polys, ring.d), dtype=np.uint64)
    for k in range(num_limbs):
        acc = (acc + ring.scale(limbs[:, k, :], pow(base, k, ring.q))) % ring.Q
    return acc


def squared_l2_norm(words, q: int) -> int:
    """squared_l2_norm (main_protocol/mod.rs:225-247): sum of squares of the
    centered values (v > q / 2 counts as v - q) of Montgomery words, exact."""
    rinv = pow(1 << 32, -1, q)
    total = 0
    for w in np.asarray(words, dtype=np.uint64).tolist():
        v = w * rinv % q
        c = v - q if v > q // 2 else v
        total += c * c
    return total


def _check_short(flat, base: int, q: int, label: str):
    """validate_decomposed_limbs: every limb's canonical value v (to_u64 of the
    field element, here w * 2^-32 mod q) is <= base/2 or >= q - base/2."""
    w = np.asarray(flat, dtype=np.uint64).reshape(-1)
    v = w * np.uint64(pow(1 << 32, -1, q)) % np.uint64(q)
    half = base // 2
    bad = np.nonzero(~((v <= half) | (v >= q - half)))[0]
    if bad.size:
        raise VerifyError(f"limb shortness: {label} word {int(bad[0])} = {int(v[bad[0]])}")


def _sym_sum(ring: EvalRing, garbage_hat, c_hat, r: int):
    """sum over i <= j of x_ij c_i c_j, off-diagonal terms doubled (eq. 3a / 3b)."""
    total = np.zeros(ring.d, dtype=np.uint64)
    idx = 0
    for i in range(r):
        for j in range(i, r):
            term = ring.mul(ring.mul(garbage_hat[idx], c_hat[i]), c_hat[j])
            total = (total + term * np.uint64(1 if i == j else 2)) % ring.Q
            idx += 1
    return total


def verify_all(q: int, d: int, *, A, B, C, D, u1, u2, z, challenges, t_limbs, g_limbs, h_limbs,
               phis, r: int, n: int, kappa: int, b1: int, t1: int, b2: int, t2: int,
               gamma: float | None = None):
    """Raise VerifyError unless the level's outputs satisfy verify_all's checks.
    A (kappa, n, d); B (kappa1, r kappa t1, d); C (kappa1, garbage t2, d);
    D (kappa2, garbage t1, d); u1 (kappa1, d); u2 (kappa2, d); z (n, d);
    challenges (r, d); t_limbs (r kappa t1, d); g_limbs (garbage t2, d);
    h_limbs (garbage t1, d); phis (r, n, d). All Montgomery words."""
    ring = EvalRing(q, d)
    gar = r * (r + 1) // 2
    # shapes (validate_proof_shapes, validate_decomposed_shapes)
    shapes = {"challenges": (challenges, r), "z": (z, n), "t_limbs": (t_limbs, r * kappa * t1),
              "g_limbs": (g_limbs, gar * t2), "h_limbs": (h_limbs, gar * t1)}
    for name, (arr, polys) in shapes.items():
        if np.asarray(arr).size != polys * d:
            raise VerifyError(f"shape: {name} holds {np.asarray(arr).size // d} polys, "
                              f"expected {polys}")
    # limb shortness (validate_decomposed_limbs): t and h in base b1, g in b2
    _check_short(t_limbs, b1, q, "t")
    _check_short(g_limbs, b2, q, "g")
    _check_short(h_limbs, b1, q, "h")
    if gamma is not None and squared_l2_norm(np.asarray(z).reshape(-1), q) > gamma * gamma:
        raise VerifyError("equation (2b): ||z|| exceeds gamma")
    t_hat = ring.evals(t_limbs)
    g_limb_hat = ring.evals(g_limbs)
    h_limb_hat = ring.evals(h_limbs)
    # (1) u1 = B t + C g over the decomposed flats
    u1_want = (ring.dot(ring.evals(B).reshape(-1, r * kappa * t1, d)[:, :, :], t_hat[None], 1)
               + ring.dot(ring.evals(C).reshape(-1, gar * t2, d), g_limb_hat[None], 1)) % ring.Q
    if not np.array_equal(ring.evals(u1).reshape(u1_want.shape), u1_want):
        raise VerifyError("equation (1): u1 != B t + C g")
    # (4) u2 = D h
    u2_want = ring.dot(ring.evals(D).reshape(-1, gar * t1, d), h_limb_hat[None], 1)
    if not np.array_equal(ring.evals(u2).reshape(u2_want.shape), u2_want):
        raise VerifyError("equation (4): u2 != D h")
    # reconstructed t_i (reconstruct_t_vecs), g_ij, h_ij
    t_rec = ring.evals(reconstruct_from_limbs(ring, t_limbs, r * kappa, t1, b1).astype(np.uint32))
    t_rec = t_rec.reshape(r, kappa, d)
    g_hat = ring.evals(reconstruct_from_limbs(ring, g_limbs, gar, t2, b2).astype(np.uint32))
    h_hat = ring.evals(reconstruct_from_limbs(ring, h_limbs, gar, t1, b1).astype(np.uint32))
    z_hat = ring.evals(z)
    c_hat = ring.evals(challenges)
    # (2a) A z = sum_i c_i t_i
    left = ring.dot(ring.evals(A).reshape(kappa, n, d), z_hat[None], 1)
    right = ring.dot(c_hat[:, None, :], t_rec, 0)
    if not np.array_equal(left, right):
        raise VerifyError("equation (2a): A z != sum c_i t_i")
    # (3a) <z, z> = sum g_ij c_i c_j
    if not np.array_equal(ring.dot(z_hat, z_hat, 0), _sym_sum(ring, g_hat, c_hat, r)):
        raise VerifyError("equation (3a): <z,z> != sum g_ij c_i c_j")
    # (3b) sum_i <phi_i, z> c_i = sum h_ij c_i c_j
    phi_z = ring.dot(ring.evals(phis).reshape(r, n, d), z_hat[None], 1)
    if not np.array_equal(ring.dot(phi_z, c_hat, 0), _sym_sum(ring, h_hat, c_hat, r)):
        raise VerifyError("equation (3b): sum <phi_i,z> c_i != sum h_ij c_i c_j")


def verify_b_double_prime(q: int, b_double_prime_ct, psi, omega, p, b0_primes):
    """verify_b_double_prime (aggregation.rs:143-181) on canonical integer values:
    for every batch k, the constant term of b''_k must equal
    sum_l psi[k][l] b0'_l + sum_m omega[k][m] p_m (mod q)."""
    for k, actual in enumerate(b_double_prime_ct):
        expected = 0
        for l, b0 in enumerate(b0_primes):
            expected = (expected + int(psi[k][l]) * int(b0) % q) % q
        for m, pm in enumerate(p):
            expected = (expected + int(omega[k][m]) * int(pm) % q) % q
        if int(actual) != expected:
            raise VerifyError(f"b''[{k}] constant term mismatch: expected {expected}, "
                              f"got {int(actual)}")
