"""CPU model of the exact reconstruction behind ring plans without an NTT for q
(lattica_b200/csrc/ring_crt.cu), checked before the kernel runs: residue words
w_j = V * 2^-32 mod p_j of an integer |V| < 2^93 go back to V * 2^-32 mod q by
Garner's mixed radix with the same Montgomery-folded constants and the same
sign rule (top digit above p2 / 2 means V < 0)."""
import numpy as np
import pytest

AUX = (4294962689, 4294957057, 4294955009)
R = 1 << 32


def mont(a, b, m):
    return a * b * pow(R, -1, m) % m


def consts(q):
    p0, p1, p2 = AUX
    i0 = pow(p0, -1, p1)
    i01 = pow(p0 * p1, -1, p2)
    i1 = pow(p1, -1, p2)
    return {
        "r2_0": R * R % p0, "c1a": R * R * i0 % p1, "c1b": R * i0 % p1,
        "c2a": R * R * i01 % p2, "c2b": R * i01 % p2, "c2c": R * i1 % p2,
        "m1": p0 % q, "m2": p0 * p1 % q, "p_rinv": p0 * p1 * p2 * pow(R, -1, q) % q,
    }


def crt_word(w, c, q):
    p0, p1, p2 = AUX
    x1 = mont(w[0], c["r2_0"], p0)
    x2 = (mont(w[1], c["c1a"], p1) - mont(x1, c["c1b"], p1)) % p1
    t3 = (mont(w[2], c["c2a"], p2) - mont(x1, c["c2b"], p2)) % p2
    x3 = (t3 - mont(x2, c["c2c"], p2)) % p2
    r = (mont(x1, 1, q) + mont(x2, c["m1"], q) + mont(x3, c["m2"], q)) % q
    return (r - c["p_rinv"]) % q if x3 > p2 // 2 else r


def test_aux_primes_support_every_compiled_degree():
    from sympy import isprime
    for p in AUX:
        assert isprime(p) and p % 512 == 1 and p > 2 ** 31
    assert AUX[0] * AUX[1] * AUX[2] > 2 ** 95


@pytest.mark.parametrize("q", [4294967291, 12281, 4294966657, 3, 17])
def test_reconstruction_recovers_montgomery_word(q):
    c = consts(q)
    rng = np.random.default_rng(q)
    bound = 1 << 93
    vals = [0, 1, -1, bound - 1, -(bound - 1), q, -q, AUX[0], -AUX[0] * AUX[1]]
    vals += [int(x) for x in rng.integers(-(1 << 62), 1 << 62, 200)]
    vals += [int(rng.integers(0, 1 << 62)) << 31 for _ in range(100)]
    vals += [-(int(rng.integers(0, 1 << 62)) << 31) for _ in range(100)]
    for v in vals:
        assert abs(v) < bound
        w = [v * pow(R, -1, p) % p for p in AUX]
        assert crt_word(w, c, q) == v * pow(R, -1, q) % q, v


def test_bound_admits_the_labrador_round():
    """n = 2048 terms of d = 64 products of words below 2^32 - 5."""
    q = 4294967291
    assert 2048 * 64 * (q - 1) ** 2 < 2 ** 93
    assert (1 << 23) * 64 * (q - 1) ** 2 < 2 ** 93 <= (1 << 24) * 64 * (q - 1) ** 2
