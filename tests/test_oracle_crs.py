"""Two oracle paths against independent Python restatements of the published
algorithms they follow. The JL projection and its int8 entries
(labrador/src/jl.rs). The seeded commitment-key expansion: ChaCha20Rng(seed)
(the RFC 8439 block function with a 64-bit block counter in words 12-13 and
stream 0 in words 14-15; rand_core's block RNG reads each u64 as two consecutive
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


def _chacha_ietf_block(key_words, counter, nonce_words):
    """RFC 8439 block: 32-bit counter in word 12, 96-bit nonce in words 13-15."""
    s = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574] + list(key_words) + \
        [counter & M32] + list(nonce_words)
    x = s[:]

    def qr(a, b, c, d):
        x[a] = (x[a] + x[b]) & M32; x[d] = _rotl(x[d] ^ x[a], 16)
        x[c] = (x[c] + x[d]) & M32; x[b] = _rotl(x[b] ^ x[c], 12)
        x[a] = (x[a] + x[b]) & M32; x[d] = _rotl(x[d] ^ x[a], 8)
        x[c] = (x[c] + x[d]) & M32; x[b] = _rotl(x[b] ^ x[c], 7)
    for _ in range(10):
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15)
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14)
    return b"".join(((x[i] + s[i]) & M32).to_bytes(4, "little") for i in range(16))


def _jl_reference(seed, rows, parts_words, parts, cols, d):
    """project_multi_into (labrador/src/jl.rs:206-256) with the extraction layout
    [row][part][k][j] for col = j * d + k: one ChaCha20 stream per part (nonce =
    part index, little endian, in the first 4 bytes), ceil(rows / 4) keystream
    bytes per column in order, entry (row) = bits 2 (row % 4) of byte row / 4:
    00 -> +1, 01 -> -1, otherwise 0."""
    key = [int.from_bytes(seed[4 * i:4 * i + 4], "little") for i in range(8)]
    packed = (rows + 3) // 4
    p = [0] * rows
    flat = np.zeros((rows, parts, cols), dtype=np.int8)
    n = cols // d
    for part in range(parts):
        stream = b"".join(_chacha_ietf_block(key, blk, [part, 0, 0])
                          for blk in range((cols * packed + 63) // 64))
        for col in range(cols):
            chunk = stream[col * packed:(col + 1) * packed]
            coeff = int(parts_words[part, col])
            j, k = divmod(col, d)
            for row in range(rows):
                v = (chunk[row // 4] >> (2 * (row % 4))) & 3
                if v == 0:
                    p[row] = (p[row] + coeff) % Q
                    flat[row, part, k * n + j] = 1
                elif v == 1:
                    p[row] = (p[row] - coeff) % Q
                    flat[row, part, k * n + j] = -1
    return np.array(p, dtype=np.uint64).astype(np.uint32), flat.reshape(-1)


def test_jl_projection_and_entries_match_an_independent_restatement(oracle):
    F = oracle.Field(Q)
    seed = bytes((11 * i + 2) & 0xFF for i in range(32))
    rng = np.random.default_rng(9)
    for rows, parts, n, d in ((256, 2, 3, 8), (100, 3, 5, 8), (7, 2, 9, 4)):
        cols = n * d
        parts_words = rng.integers(0, Q, (parts, cols), dtype=np.uint64).astype(np.uint32)
        want_p, want_flat = _jl_reference(seed, rows, parts_words, parts, cols, d)
        got_p, got_flat = oracle.jl_project(F, seed, rows, parts_words, parts, cols, d)
        assert np.array_equal(got_p, want_p), (rows, parts, n, d)
        assert np.array_equal(np.asarray(got_flat).view(np.int8).reshape(-1), want_flat), rows
