"""LaBRADOR prover hot calls on the GPU, mirroring the reference surface:
`CommitKey::inner_commit_slice / inner_commit_decomposed` (labrador/src/crs.rs),
`compute_garbage_g` (labrador/src/main_protocol/garbage.rs), `JLMatrix`
(labrador/src/jl.rs) and `decompose_polys` (labrador/src/main_protocol/mod.rs).

Witness layout: r parts x n polys x d Montgomery words (LabradorWitness parts,
each a slice of CyclotomicPolyRing<R, d>).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .commit import PreparedMatrix
from .ntt import TwistedNttPlan, _is_torch, _stream_ptr, raise_status

JL_MAX_RETRY = 100  # labrador/src/jl.rs:27


def garbage_index(r: int, i: int, j: int) -> int:
    """Upper-triangular index (main_protocol/mod.rs:664-670)."""
    return i * r - (i * (i - 1)) // 2 + (j - i)


def garbage_count(r: int) -> int:
    return r * (r + 1) // 2


@dataclass
class DecomposedPolys:
    """DecomposedPolys (main_protocol/mod.rs:361-375): flat[poly][limb] polys."""

    flat: np.ndarray
    num_polys: int
    num_limbs: int
    base: int


def decompose_polys(plan: TwistedNttPlan, polys, base: int, num_limbs: int) -> DecomposedPolys:
    """Balanced base-`base` decomposition (decompose_polys, main_protocol/mod.rs:731-747)."""
    p = np.ascontiguousarray(polys, dtype=np.uint32).reshape(-1, plan.d)
    out = np.empty((p.shape[0], num_limbs, plan.d), dtype=np.uint32)
    st = _lib.load().grid_gpu_decompose_balanced(plan.handle, p.ctypes.data, p.shape[0], base,
                                                 num_limbs, out.ctypes.data)
    raise_status(st, "grid_gpu_decompose_balanced")
    return DecomposedPolys(out.reshape(-1, plan.d), p.shape[0], num_limbs, base)


def compute_garbage_g(plan: TwistedNttPlan, witness):
    """g_ij = <s_i, s_j> for i <= j in garbage_index order (garbage.rs:76-93).
    witness: (r, n, d) numpy uint32 or a CUDA tensor."""
    r, n, d = (int(x) for x in witness.shape)
    if d != plan.d:
        raise ValueError("witness ring degree does not match the plan")
    lib = _lib.load()
    if _is_torch(witness):
        import torch
        g = torch.empty((garbage_count(r), d), dtype=witness.dtype, device=witness.device)
        nb = C.c_size_t()
        raise_status(lib.grid_gpu_gram_workspace(plan.handle, r, n, C.byref(nb)), "gram_ws")
        ws = torch.empty(max(16, nb.value), dtype=torch.uint8, device=witness.device)
        st = lib.grid_gpu_gram_dev(plan.handle, witness.data_ptr(), r, n, g.data_ptr(),
                                   ws.data_ptr(), ws.numel(), _stream_ptr(witness))
    else:
        w = np.ascontiguousarray(witness, dtype=np.uint32)
        g = np.empty((garbage_count(r), d), dtype=np.uint32)
        st = lib.grid_gpu_gram(plan.handle, w.ctypes.data, r, n, g.ctypes.data)
    raise_status(st, "grid_gpu_gram")
    return g


def compute_garbage_g_batch(plan: TwistedNttPlan, pool, items, k_split: int = 0,
                            workspace=None):
    """compute_garbage_g for many witnesses of different rank r <= 64 and
    length n in one launch sequence. pool: CUDA tensor (polys, d) of witness
    words; items: [(s_offset, r, n)], witness i = r x n polys at poly s_offset.
    Returns a CUDA tensor (sum_i r_i (r_i + 1) / 2, d): item i's Gram polys in
    garbage_index order after item i-1's. Equals one compute_garbage_g per item."""
    import torch
    lib = _lib.load()
    d = plan.d
    arr = (_lib.GramItem * len(items))()
    total = 0
    for i, (so, r, n) in enumerate(items):
        arr[i] = _lib.GramItem(int(so), int(r), int(n))
        total += garbage_count(int(r))
    G = torch.empty((total, d), dtype=torch.int32, device=pool.device)
    if workspace is None:
        nb = C.c_size_t()
        raise_status(lib.grid_gpu_batch_gram_workspace(plan.handle, arr, len(items), int(k_split),
                                                       C.byref(nb)), "batch_gram_workspace")
        workspace = torch.empty(max(256, nb.value), dtype=torch.uint8, device=pool.device)
    st = lib.grid_gpu_batch_gram_dev(plan.handle, pool.data_ptr(), arr, len(items), int(k_split),
                                     G.data_ptr(), workspace.data_ptr(), workspace.numel(),
                                     _stream_ptr(pool))
    raise_status(st, "grid_gpu_batch_gram_dev")
    return G


def compute_garbage_h(plan: TwistedNttPlan, witness, aggregated_phis):
    """h_ij = (<phi_i, s_j> + <phi_j, s_i>) * 2^-1 for i <= j in garbage_index
    order (garbage.rs:101-133). witness, aggregated_phis: (r, n, d) numpy
    uint32 or CUDA tensors (both the same kind)."""
    r, n, d = (int(x) for x in witness.shape)
    if d != plan.d or tuple(aggregated_phis.shape) != (r, n, d):
        raise ValueError("witness and phis must both be (r, n, d) with the plan's d")
    lib = _lib.load()
    if _is_torch(witness):
        import torch
        h = torch.empty((garbage_count(r), d), dtype=witness.dtype, device=witness.device)
        nb = C.c_size_t()
        raise_status(lib.grid_gpu_garbage_h_workspace(plan.handle, r, n, C.byref(nb)),
                     "garbage_h_ws")
        ws = torch.empty(max(16, nb.value), dtype=torch.uint8, device=witness.device)
        st = lib.grid_gpu_garbage_h_dev(plan.handle, witness.data_ptr(),
                                        aggregated_phis.data_ptr(), r, n, h.data_ptr(),
                                        ws.data_ptr(), ws.numel(), _stream_ptr(witness))
    else:
        w = np.ascontiguousarray(witness, dtype=np.uint32)
        ph = np.ascontiguousarray(aggregated_phis, dtype=np.uint32)
        h = np.empty((garbage_count(r), d), dtype=np.uint32)
        st = lib.grid_gpu_garbage_h(plan.handle, w.ctypes.data, ph.ctypes.data, r, n,
                                    h.ctypes.data)
    raise_status(st, "grid_gpu_garbage_h")
    return h


def amortize_witness(plan: TwistedNttPlan, witness, challenges):
    """z[k] = sum_i c_i * s_i[k], the product part of compute_amortized_witness
    (amortization.rs:61-84); the challenges c_i (r polys) come from the
    caller's transcript. witness: (r, n, d), challenges: (r, d), numpy uint32
    or CUDA tensors (both the same kind). Returns z: (n, d)."""
    r, n, d = (int(x) for x in witness.shape)
    if d != plan.d or tuple(challenges.shape) != (r, d):
        raise ValueError("witness must be (r, n, d) and challenges (r, d) with the plan's d")
    lib = _lib.load()
    if _is_torch(witness):
        import torch
        z = torch.empty((n, d), dtype=witness.dtype, device=witness.device)
        nb = C.c_size_t()
        raise_status(lib.grid_gpu_amortize_workspace(plan.handle, r, n, C.byref(nb)),
                     "amortize_ws")
        ws = torch.empty(max(16, nb.value), dtype=torch.uint8, device=witness.device)
        st = lib.grid_gpu_amortize_dev(plan.handle, witness.data_ptr(), challenges.data_ptr(),
                                       r, n, z.data_ptr(), ws.data_ptr(), ws.numel(),
                                       _stream_ptr(witness))
    else:
        w = np.ascontiguousarray(witness, dtype=np.uint32)
        c = np.ascontiguousarray(challenges, dtype=np.uint32)
        z = np.empty((n, d), dtype=np.uint32)
        st = lib.grid_gpu_amortize(plan.handle, w.ctypes.data, c.ctypes.data, r, n, z.ctypes.data)
    raise_status(st, "grid_gpu_amortize")
    return z


class CommitKey:
    """The inner-commitment matrix A (kappa x n) of a LaBRADOR CommitKey
    (labrador/src/crs.rs:111-216), kept resident on the device."""

    def __init__(self, plan: TwistedNttPlan, a, kappa: int, n: int, is_evals: bool = False):
        self.plan, self.kappa, self.n = plan, kappa, n
        self.a = PreparedMatrix(plan, a, kappa, n, is_evals)

    def inner_commit_slice(self, s_i):
        """t_i = A * s_i (crs.rs:211-216); s_i (n, d) or a batch (r, n, d)."""
        return self.a.mul_vec(s_i)

    def inner_commit_decomposed(self, witness, b1: int, t1: int) -> DecomposedPolys:
        """t_i = A s_i for every part, balanced limbs (crs.rs:225-256)."""
        t = self.inner_commit_slice(witness)
        return decompose_polys(self.plan, np.asarray(t).reshape(-1, self.plan.d), b1, t1)


class OuterCommitKey:
    """The outer-commitment matrices of a LaBRADOR CommitKey (crs.rs:111-123):
    B (kappa1 x t_len), C (kappa1 x g_len), D (kappa2 x h_len), prepared on the
    device."""

    def __init__(self, plan: TwistedNttPlan, b, c, d, kappa1: int, kappa2: int, t_len: int,
                 g_len: int, h_len: int):
        from .commit import CommitmentDimensions, LinearCommitmentKey
        self.plan = plan
        self.bc = LinearCommitmentKey(plan, b, c, CommitmentDimensions(t_len, g_len, kappa1))
        if not _is_torch(d):
            d = np.ascontiguousarray(d, dtype=np.uint32)
        self.d = PreparedMatrix(plan, d, kappa2, h_len)

    def outer_commit_u1_slice(self, t, g):
        """u1 = B t + C g (crs.rs:272-285); t (t_len, d), g (g_len, d): numpy
        uint32 or CUDA tensors (both the same kind)."""
        return self.bc.recompute(t, g)

    def outer_commit_u2_slice(self, h):
        """u2 = D h (crs.rs:297-303); h (h_len, d), numpy uint32 or a CUDA tensor."""
        return self.d.mul_vec(h)


def sample_uniform_polys(plan: TwistedNttPlan, seed: bytes, npolys: int, device=None,
                         accept_max: int = 0):
    """npolys uniform ring elements (Montgomery words, shape (npolys, d)) drawn
    in order from ChaCha20Rng(seed), as sample_uniform_mat does
    (crs.rs:308-326, prime.rs:730-743). device: a CUDA device for a tensor on
    the device, else a numpy array. accept_max 0 keeps the reference's
    rejection threshold."""
    if len(seed) != 32:
        raise ValueError("seed must be 32 bytes")
    lib = _lib.load()
    sd = (C.c_uint8 * 32).from_buffer_copy(bytes(seed))
    d = plan.d
    if device is not None:
        import torch
        out = torch.empty((npolys, d), dtype=torch.int32, device=device)
        nb = C.c_size_t()
        raise_status(lib.grid_gpu_sample_uniform_polys_workspace(plan.handle, npolys, accept_max,
                                                                 C.byref(nb)), "sample_ws")
        ws = torch.empty(max(16, nb.value), dtype=torch.uint8, device=device)
        st = lib.grid_gpu_sample_uniform_polys_dev(plan.handle, sd, npolys, accept_max,
                                                   out.data_ptr(), ws.data_ptr(), ws.numel(),
                                                   _stream_ptr(out))
    else:
        out = np.empty((npolys, d), dtype=np.uint32)
        st = lib.grid_gpu_sample_uniform_polys(plan.handle, sd, npolys, accept_max,
                                               out.ctypes.data)
    raise_status(st, "grid_gpu_sample_uniform_polys")
    return out


def commit_key_from_seed(plan: TwistedNttPlan, seed: bytes, r: int, n: int, kappa: int,
                         kappa1: int, kappa2: int, t1: int, t2: int, device):
    """CommitKey::from_seed (crs.rs:136-198) expanded on the device: A
    (kappa x n), B (kappa1 x r*t1*kappa), C (kappa1 x t2*g), D (kappa2 x t1*g)
    with g = r(r+1)/2, consecutive draws of one ChaCha20Rng(seed). Returns
    (CommitKey for A, OuterCommitKey for B, C, D)."""
    for name, v in (("n", n), ("r", r), ("kappa", kappa), ("kappa1", kappa1),
                    ("kappa2", kappa2), ("t1", t1), ("t2", t2)):
        if v <= 0:
            raise ValueError(f"CommitKey dimension {name}={v} must be positive")
    g = r * (r + 1) // 2
    cols_b, cols_c, cols_d = r * t1 * kappa, t2 * g, t1 * g
    sizes = [kappa * n, kappa1 * cols_b, kappa1 * cols_c, kappa2 * cols_d]
    polys = sample_uniform_polys(plan, seed, sum(sizes), device=device)
    offs = np.cumsum([0] + sizes)
    a, b, c, dm = (polys[offs[i]:offs[i + 1]] for i in range(4))
    return (CommitKey(plan, a, kappa, n),
            OuterCommitKey(plan, b, c, dm, kappa1, kappa2, cols_b, cols_c, cols_d))


class JLMatrix:
    """Seeded JL projection (labrador/src/jl.rs:34-509): ChaCha20 keystream,
    key = seed, nonce = part index."""

    def __init__(self, seed: bytes, rows: int, cols: int):
        if cols <= 0:
            raise ValueError("JL projection columns must be > 0 (n * d)")
        if len(seed) != 32:
            raise ValueError("JL seed must be 32 bytes")
        self.seed, self.rows, self._cols = bytes(seed), rows, cols

    @classmethod
    def from_seed(cls, rows: int, cols: int, seed: bytes) -> "JLMatrix":
        return cls(seed, rows, cols)

    def cols(self) -> int:
        return self._cols

    def project_and_extract_jl_rows(self, plan: TwistedNttPlan, parts, num_parts: int, d: int,
                                    extract: bool = True):
        """(p, jl_rows_flat) like project_and_extract_jl_rows (jl.rs:267-303).
        parts: (num_parts, cols) words; flat: rows*num_parts*cols int8."""
        if d <= 0 or self._cols % d:
            raise ValueError(f"cols ({self._cols}) must be divisible by ring degree d ({d})")
        parts = np.ascontiguousarray(parts, dtype=np.uint32).reshape(-1)
        if parts.size != num_parts * self._cols:
            raise ValueError("parts count / length mismatch")
        p = np.empty(self.rows, dtype=np.uint32)
        flat = np.empty(self.rows * num_parts * self._cols, dtype=np.int8) if extract else None
        seed = (C.c_uint8 * 32).from_buffer_copy(self.seed)
        st = _lib.load().grid_gpu_jl_project(plan.handle, seed, self.rows, parts.ctypes.data,
                                             num_parts, self._cols, d, p.ctypes.data,
                                             flat.ctypes.data if extract else None)
        raise_status(st, "grid_gpu_jl_project")
        return p, flat

    def project_multi(self, plan: TwistedNttPlan, parts, num_parts: int, d: int):
        return self.project_and_extract_jl_rows(plan, parts, num_parts, d, extract=False)[0]

    def conjugated_evals(self, plan: TwistedNttPlan, parts, num_parts: int, d: int):
        """jl_evals[m] = sum_{i,j} conj(pi_{m,i,j}) * s_{i,j}: the polynomials
        prove_step builds from jl_rows_flat_to_conjugated_polys
        (main_protocol/mod.rs:885-923, step_prover.rs:185-206), computed from
        the keystream without the int8 entries. parts: (num_parts, cols)
        numpy uint32 or a CUDA tensor; returns (rows, d). The kernel covers
        rows = 256 and d = 64."""
        if d <= 0 or self._cols % d:
            raise ValueError(f"cols ({self._cols}) must be divisible by ring degree d ({d})")
        lib = _lib.load()
        seed = (C.c_uint8 * 32).from_buffer_copy(self.seed)
        if _is_torch(parts):
            import torch
            if parts.numel() != num_parts * self._cols:
                raise ValueError("parts count / length mismatch")
            ev = torch.empty((self.rows, d), dtype=parts.dtype, device=parts.device)
            nb = C.c_size_t()
            raise_status(lib.grid_gpu_jl_evals_workspace(C.byref(nb)), "jl_evals_ws")
            ws = torch.empty(max(16, nb.value), dtype=torch.uint8, device=parts.device)
            st = lib.grid_gpu_jl_evals_dev(plan.handle, seed, self.rows, parts.data_ptr(),
                                           num_parts, self._cols, d, ev.data_ptr(), ws.data_ptr(),
                                           ws.numel(), _stream_ptr(parts))
        else:
            parts = np.ascontiguousarray(parts, dtype=np.uint32).reshape(-1)
            if parts.size != num_parts * self._cols:
                raise ValueError("parts count / length mismatch")
            ev = np.empty((self.rows, d), dtype=np.uint32)
            st = lib.grid_gpu_jl_evals(plan.handle, seed, self.rows, parts.ctypes.data,
                                       num_parts, self._cols, d, ev.ctypes.data)
        raise_status(st, "grid_gpu_jl_evals")
        return ev


@dataclass
class RoundOutputs:
    t_limbs: object   # (r*kappa*t1, d)
    g: object         # (r(r+1)/2, d)
    g_limbs: object   # (r(r+1)/2*t2, d) or None
    p: object         # (jl_rows,) or None
    jl_flat: object   # int8 or None
    jl_evals: object = None  # (256, d) conjugated JL evaluations, or None


def prover_round_dev(key: CommitKey, witness, b1: int, t1: int, b2: int, t2: int,
                     jl_seed: bytes | None, jl_rows: int = 256, extract: bool = False,
                     workspace=None, jl_evals: bool = False) -> RoundOutputs:
    """The GPU hot calls of one prove_step (step_prover.rs:118-170) on a CUDA
    witness tensor (r, n, d): inner commitments + limbs, Gram + limbs, JL.

    jl_evals=True also returns the 256 conjugated JL evaluations that
    prove_step aggregates later (step_prover.rs:185-206). Coefficient 0 of
    evals[m] is sum_u pi_{m,u} s[u], the projection p_m itself, so without
    `extract` the round runs the evaluation kernel in place of the projection
    and reads p from it: one keystream pass instead of two."""
    import torch
    r, n, d = (int(x) for x in witness.shape)
    if jl_evals and (not jl_seed or jl_rows != 256 or d != 64):
        raise ValueError("jl_evals needs a JL seed, 256 rows and d = 64")
    if jl_evals and not extract:
        out = prover_round_dev(key, witness, b1, t1, b2, t2, None, jl_rows, False, workspace)
        jl = JLMatrix.from_seed(jl_rows, n * d, jl_seed)
        ev = jl.conjugated_evals(key.plan, witness.reshape(r, n * d), r, d)
        out.p = ev[:, 0].contiguous()
        out.jl_evals = ev
        return out
    plan = key.plan
    lib = _lib.load()
    dev = witness.device
    kappa = key.kappa
    t_limbs = torch.empty((r * kappa * t1, d), dtype=torch.int32, device=dev)
    g = torch.empty((garbage_count(r), d), dtype=torch.int32, device=dev)
    g_limbs = torch.empty((garbage_count(r) * t2, d), dtype=torch.int32, device=dev) if t2 else None
    p = torch.empty(jl_rows, dtype=torch.int32, device=dev) if jl_seed else None
    flat = (torch.empty(jl_rows * r * n * d, dtype=torch.int8, device=dev)
            if (jl_seed and extract) else None)
    if workspace is None:
        nb = C.c_size_t()
        raise_status(lib.grid_gpu_prover_round_workspace(key.a.handle, r, jl_rows, C.byref(nb)),
                     "prover_round_workspace")
        workspace = torch.empty(max(16, nb.value), dtype=torch.uint8, device=dev)
    seed = (C.c_uint8 * 32).from_buffer_copy(jl_seed) if jl_seed else None
    st = lib.grid_gpu_prover_round_dev(
        key.a.handle, witness.data_ptr(), r, b1, t1, b2, t2, seed, jl_rows, t_limbs.data_ptr(),
        g.data_ptr(), g_limbs.data_ptr() if g_limbs is not None else None,
        p.data_ptr() if p is not None else None, flat.data_ptr() if flat is not None else None,
        workspace.data_ptr(), workspace.numel(), _stream_ptr(witness))
    raise_status(st, "grid_gpu_prover_round_dev")
    out = RoundOutputs(t_limbs, g, g_limbs, p, flat)
    if jl_evals:
        jl = JLMatrix.from_seed(jl_rows, n * d, jl_seed)
        out.jl_evals = jl.conjugated_evals(plan, witness.reshape(r, n * d), r, d)
    return out


def _canonical(words, q: int):
    """Montgomery words -> canonical integers (value = word * 2^-32 mod q)."""
    rinv = pow(1 << 32, -1, q)
    w = np.asarray(words, dtype=np.uint64).ravel()
    return [(int(x) * rinv) % q for x in w]


def squared_l2_norm_u128(words, q: int) -> int:
    """Centered squared L2 norm, exact (main_protocol/mod.rs:225-247)."""
    half = q // 2
    total = 0
    for v in _canonical(words, q):
        a = q - v if v > half else v
        total += a * a
    if total >= 1 << 128:
        raise OverflowError("norm overflow: sum exceeds u128")
    return total


def verify_norm(p_words, q: int, beta: float, rows: int = 256,
                verify_factor: float = 128.0 ** 0.5) -> bool:
    """||p||^2 <= (verify_factor * beta)^2 (jl.rs:533-547, JLProfile::paper_default)."""
    import math
    if not math.isfinite(beta) or beta <= 0.0:
        return False
    if len(np.asarray(p_words).ravel()) != rows:
        return False
    try:
        norm_sq = float(squared_l2_norm_u128(p_words, q))
    except OverflowError:
        return False
    threshold = (verify_factor * beta) * (verify_factor * beta)
    return norm_sq <= threshold
