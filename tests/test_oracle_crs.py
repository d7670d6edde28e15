"""The oracle's seeded commitment-key expansion against an independent Python
restatement of the same published algorithm: ChaCha20Rng(seed) (the RFC 8439
block function with a 64-bit block counter in words 12-13 and stream 0 in
words 14-15; rand_core's block RNG reads each u64 as two consecutive
little-endian words, low word first) and PrimeField::rand's u64 rejection
(prime.rs:730-743: accept s <= u64::MAX - ((u64::MAX % q + 1) % q), value s % q).
A lowered acceptance threshold makes rejections frequent."""
import numpy as np

Q = 4294966657
M32 = 0xFFFFFFFF


def _rotl(x, r):
    return ((x << r) | (x >> (32 - r))) & M32


def _chacha_block(key_words, counter):
    s = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574] + list(key_words) + \
        [counter & M32, counter >> 32, 0, 0]
    x = s[:]

    def qr(a, b, c, d):
        x[a] = (x[a] + x[b]) & M32; x[d] = _rotl(x[d] ^ x[a], 16)
        x[c] = (x[c] + x[d]) & M32; x[b] = _rotl(x[b] ^ x[c], 12)
        x[a] = (x[a] + x[b]) & M32; x[d] = _rotl(x[d] ^ x[a], 8)
        x[c] = (x[c] + x[d]) & M32; x[b] = _rotl(x[b] ^ x[c], 7)
    for _ in range(10):
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15)
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14)
    return [(x[i] + s[i]) & M32 for i in range(16)]


def _sample(seed, count, accept_max=0):
    key = [int.from_bytes(seed[4 * i:4 * i + 4], "little") for i in range(8)]
    upper = accept_max or (2 ** 64 - 1) - (((2 ** 64 - 1) % Q + 1) % Q)
    out, block = [], 0
    while len(out) < count:
        w = _chacha_block(key, block)
        block += 1
        for c in range(8):
            s = w[2 * c] | (w[2 * c + 1] << 32)
            if s <= upper and len(out) < count:
                out.append((s % Q) * (1 << 32) % Q)  # from_u64(s % q), Montgomery word
    return np.array(out, dtype=np.uint64).astype(np.uint32)


def test_seeded_expansion_matches_an_independent_restatement(oracle):
    F = oracle.Field(Q)
    seed = bytes(range(3, 35))
    for npolys, accept_max in ((3, 0), (2, 1 << 62), (2, (1 << 63) + 12345)):
        want = _sample(seed, npolys * 64, accept_max)
        got = oracle.sample_uniform_polys(F, seed, npolys, 64, accept_max)
        assert np.array_equal(got, want), (npolys, accept_max)
