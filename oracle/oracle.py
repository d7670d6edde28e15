"""ctypes wrapper around the C oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module. Arrays are numpy uint32 Montgomery words (PrimeField<Q, u32>).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_u32p = C.POINTER(C.c_uint32)
_i64p = C.POINTER(C.c_int64)
_i8p = C.POINTER(C.c_int8)
_u8p = C.POINTER(C.c_uint8)

_LIB = None


class OracleError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        super().__init__(f"oracle error {code} {what}")
        self.code = code


class _Field(C.Structure):
    _fields_ = [("q", C.c_uint32), ("r_mod_q", C.c_uint32), ("r2_mod_q", C.c_uint32),
                ("q_inv", C.c_uint32)]


class _Plan(C.Structure):
    _fields_ = [("f", _Field), ("n", C.c_uint32), ("generator", C.c_uint32),
                ("omega", C.c_uint32), ("psi", C.c_uint32), ("inv_scale", C.c_uint32),
                ("fwd_tw", _u32p), ("inv_tw", _u32p), ("twists", _u32p), ("untwists", _u32p)]


def lib():
    global _LIB
    if _LIB is None:
        path = _build.build()
        L = C.CDLL(path)
        fp = C.POINTER(_Field)
        pp = C.POINTER(_Plan)
        sig = {
            "orc_field_init": (C.c_int, [fp, C.c_uint64]),
            "orc_to_mont": (C.c_uint32, [fp, C.c_uint64]),
            "orc_from_mont": (C.c_uint32, [fp, C.c_uint32]),
            "orc_add": (C.c_uint32, [fp, C.c_uint32, C.c_uint32]),
            "orc_sub": (C.c_uint32, [fp, C.c_uint32, C.c_uint32]),
            "orc_mul": (C.c_uint32, [fp, C.c_uint32, C.c_uint32]),
            "orc_pow": (C.c_uint32, [fp, C.c_uint32, C.c_uint64]),
            "orc_inv": (C.c_uint32, [fp, C.c_uint32]),
            "orc_is_prime_u64": (C.c_int, [C.c_uint64]),
            "orc_plan_create": (C.c_int, [pp, C.c_uint64, C.c_uint64]),
            "orc_plan_destroy": (None, [pp]),
            "orc_max_ntt_size": (C.c_uint64, [C.c_uint64]),
            "orc_find_generator": (C.c_uint32, [fp]),
            "orc_ntt_forward": (None, [pp, _u32p]),
            "orc_ntt_inverse": (None, [pp, _u32p]),
            "orc_twisted_forward": (None, [pp, _u32p, C.c_size_t]),
            "orc_twisted_inverse": (None, [pp, _u32p, C.c_size_t]),
            "orc_ntt_mul_inverse": (None, [pp, _u32p, _u32p, _u32p, C.c_size_t]),
            "orc_ntt_mul_inverse_mt": (None, [pp, _u32p, _u32p, _u32p, C.c_size_t, C.c_int]),
            "orc_ntt_mul_inverse_avx2": (None, [pp, _u32p, _u32p, _u32p, C.c_size_t]),
            "orc_matvec_avx2": (C.c_int, [pp, _u32p, C.c_size_t, C.c_size_t, C.c_int, _u32p,
                                          C.c_size_t, _u32p, C.c_int]),
            "orc_ntt_mul_inverse_avx2_mt": (None, [pp, _u32p, _u32p, _u32p, C.c_size_t,
                                                   C.c_int]),
            "orc_poly_mul_ntt": (None, [pp, _u32p, _u32p, _u32p]),
            "orc_naive_negacyclic": (None, [fp, C.c_uint32, _u32p, _u32p, _u32p]),
            "orc_pointwise_mul": (None, [fp, _u32p, _u32p, C.c_size_t]),
            "orc_matvec": (C.c_int, [pp, _u32p, C.c_size_t, C.c_size_t, C.c_int, _u32p,
                                     C.c_size_t, _u32p]),
            "orc_matvec_mt": (C.c_int, [pp, _u32p, C.c_size_t, C.c_size_t, C.c_int, _u32p,
                                        C.c_size_t, _u32p, C.c_int]),
            "orc_linear_commit": (C.c_int, [pp, _u32p, C.c_size_t, C.c_size_t, _u32p,
                                            C.c_size_t, _u32p, _u32p, _u32p]),
            "orc_gram": (C.c_int, [pp, _u32p, C.c_size_t, C.c_size_t, _u32p, C.c_int]),
            "orc_gram_naive": (C.c_int, [pp, _u32p, C.c_size_t, C.c_size_t, _u32p]),
            "orc_garbage_h": (C.c_int, [pp, _u32p, _u32p, C.c_size_t, C.c_size_t, _u32p]),
            "orc_jl_evals": (C.c_int, [pp, _i8p, C.c_size_t, _u32p, C.c_size_t, C.c_size_t,
                                       _u32p]),
            "orc_sample_uniform_polys": (C.c_int, [fp, _u8p, C.c_size_t, C.c_uint32, C.c_uint64,
                                                   _u32p]),
            "orc_amortize": (C.c_int, [pp, _u32p, _u32p, C.c_size_t, C.c_size_t, _u32p]),
            "orc_garbage_index": (C.c_size_t, [C.c_size_t, C.c_size_t, C.c_size_t]),
            "orc_decompose_coeff_balanced": (None, [C.c_uint64, C.c_uint64, C.c_size_t,
                                                    C.c_uint64, _i64p]),
            "orc_centered_mod": (C.c_int64, [C.c_int64, C.c_int64]),
            "orc_decompose_polys": (C.c_int, [fp, C.c_uint32, _u32p, C.c_size_t, C.c_uint64,
                                              C.c_size_t, _u32p]),
            "orc_reconstruct_from_limbs": (C.c_int, [fp, C.c_uint32, _u32p, C.c_size_t,
                                                     C.c_uint64, _u32p]),
            "orc_gadget_digits": (C.c_size_t, [C.c_uint64, C.c_uint64]),
            "orc_gadget_decompose": (C.c_int, [fp, _u32p, C.c_size_t, C.c_uint64, _u32p]),
            "orc_chacha20_block": (None, [_u8p, C.c_uint32, _u8p, _u8p]),
            "orc_chacha20_quarter": (None, [_u32p, _u32p, _u32p, _u32p]),
            "orc_jl_project": (C.c_int, [fp, _u8p, C.c_size_t, C.c_size_t, _u32p, C.c_size_t,
                                         C.c_size_t, _u32p, _i8p, C.c_int]),
            "orc_add_assign_slice": (None, [fp, _u32p, _u32p, C.c_size_t]),
            "orc_sub_assign_slice": (None, [fp, _u32p, _u32p, C.c_size_t]),
            "orc_scalar_mul_slice": (None, [fp, _u32p, C.c_uint32, C.c_size_t]),
            "orc_add_assign_scaled_slice": (None, [fp, _u32p, _u32p, C.c_uint32, C.c_size_t]),
            "orc_dot_product": (C.c_uint32, [fp, _u32p, _u32p, C.c_size_t]),
            "orc_ring_matvec": (C.c_int, [fp, C.c_uint32, _u32p, C.c_size_t, C.c_size_t, _u32p,
                                          C.c_size_t, _u32p, C.c_int]),
            "orc_ring_gram": (C.c_int, [fp, C.c_uint32, _u32p, C.c_size_t, C.c_size_t, _u32p,
                                        C.c_int]),
            "orc_ring_garbage_h": (C.c_int, [fp, C.c_uint32, _u32p, _u32p, C.c_size_t,
                                             C.c_size_t, _u32p, C.c_int]),
            "orc_ring_amortize": (C.c_int, [fp, C.c_uint32, _u32p, _u32p, C.c_size_t, C.c_size_t,
                                            _u32p, C.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(_u32p)


class Field:
    def __init__(self, q: int):
        self.s = _Field()
        st = lib().orc_field_init(C.byref(self.s), q)
        if st:
            raise OracleError(st, f"q={q}")
        self.q = q

    def to_mont(self, v):
        v = np.asarray(v, dtype=np.uint64).ravel()
        out = np.empty(v.shape, dtype=np.uint32)
        L = lib()
        for i, x in enumerate(v):
            out[i] = L.orc_to_mont(C.byref(self.s), int(x))
        return out

    def from_mont(self, w):
        w = np.asarray(w, dtype=np.uint32).ravel()
        L = lib()
        return np.array([L.orc_from_mont(C.byref(self.s), int(x)) for x in w], dtype=np.uint64)

    def mul(self, a: int, b: int) -> int:
        return lib().orc_mul(C.byref(self.s), a, b)

    def add(self, a: int, b: int) -> int:
        return lib().orc_add(C.byref(self.s), a, b)

    def sub(self, a: int, b: int) -> int:
        return lib().orc_sub(C.byref(self.s), a, b)

    def pow(self, a: int, e: int) -> int:
        return lib().orc_pow(C.byref(self.s), a, e)

    def one(self) -> int:
        return self.s.r_mod_q

    # -- slice hooks of Ring for PrimeField (arith/prime.rs:433-491); new arrays
    def add_slice(self, dst, src):
        d, pd = _u32(np.array(dst, dtype=np.uint32, copy=True))
        s_, ps = _u32(src)
        lib().orc_add_assign_slice(C.byref(self.s), pd, ps, d.size)
        return d

    def sub_slice(self, dst, src):
        d, pd = _u32(np.array(dst, dtype=np.uint32, copy=True))
        s_, ps = _u32(src)
        lib().orc_sub_assign_slice(C.byref(self.s), pd, ps, d.size)
        return d

    def scalar_mul_slice(self, dst, scalar: int):
        d, pd = _u32(np.array(dst, dtype=np.uint32, copy=True))
        lib().orc_scalar_mul_slice(C.byref(self.s), pd, scalar, d.size)
        return d

    def add_scaled_slice(self, dst, src, scalar: int):
        d, pd = _u32(np.array(dst, dtype=np.uint32, copy=True))
        s_, ps = _u32(src)
        lib().orc_add_assign_scaled_slice(C.byref(self.s), pd, ps, scalar, d.size)
        return d

    def dot_product(self, lhs, rhs) -> int:
        a, pa = _u32(lhs)
        b, pb = _u32(rhs)
        return lib().orc_dot_product(C.byref(self.s), pa, pb, a.size)

    def pointwise_mul_slice(self, dst, rhs):
        d, pd = _u32(np.array(dst, dtype=np.uint32, copy=True))
        r_, pr = _u32(rhs)
        lib().orc_pointwise_mul(C.byref(self.s), pd, pr, d.size)
        return d

    # -- ring contractions with schoolbook negacyclic products (any odd prime q)
    def ring_matvec(self, d: int, A, rows: int, cols: int, s, batch: int, threads: int = 0):
        A, pA = _u32(A)
        s, ps = _u32(s)
        t = np.empty(batch * rows * d, dtype=np.uint32)
        st = lib().orc_ring_matvec(C.byref(self.s), d, pA, rows, cols, ps, batch,
                                   t.ctypes.data_as(_u32p), threads or os.cpu_count())
        if st:
            raise OracleError(st)
        return t

    def ring_gram(self, d: int, S, r: int, n: int, threads: int = 0):
        S, pS = _u32(S)
        G = np.empty(r * (r + 1) // 2 * d, dtype=np.uint32)
        st = lib().orc_ring_gram(C.byref(self.s), d, pS, r, n, G.ctypes.data_as(_u32p),
                                 threads or os.cpu_count())
        if st:
            raise OracleError(st)
        return G

    def ring_garbage_h(self, d: int, S, Phi, r: int, n: int, threads: int = 0):
        S, pS = _u32(S)
        Phi, pP = _u32(Phi)
        H = np.empty(r * (r + 1) // 2 * d, dtype=np.uint32)
        st = lib().orc_ring_garbage_h(C.byref(self.s), d, pS, pP, r, n, H.ctypes.data_as(_u32p),
                                      threads or os.cpu_count())
        if st:
            raise OracleError(st)
        return H

    def ring_amortize(self, d: int, S, c, r: int, n: int, threads: int = 0):
        S, pS = _u32(S)
        c, pc = _u32(c)
        Z = np.empty(n * d, dtype=np.uint32)
        st = lib().orc_ring_amortize(C.byref(self.s), d, pS, pc, r, n, Z.ctypes.data_as(_u32p),
                                     threads or os.cpu_count())
        if st:
            raise OracleError(st)
        return Z

    def naive_negacyclic(self, a, b):
        a, pa = _u32(a)
        b, pb = _u32(b)
        out = np.empty(a.size, dtype=np.uint32)
        lib().orc_naive_negacyclic(C.byref(self.s), a.size, pa, pb, out.ctypes.data_as(_u32p))
        return out


class Plan:
    """Twisted negacyclic plan of length n (mirrors TwistedNttPlan::build)."""

    def __init__(self, q: int, n: int):
        self.s = _Plan()
        st = lib().orc_plan_create(C.byref(self.s), q, n)
        if st:
            lib().orc_plan_destroy(C.byref(self.s))
            raise OracleError(st, f"q={q} n={n}")
        self.q, self.n = q, n
        self.field = Field(q)

    def __del__(self):
        try:
            lib().orc_plan_destroy(C.byref(self.s))
        except Exception:
            pass

    def _ref(self):
        return C.byref(self.s)

    def tables(self):
        n = self.n
        get = lambda p, k: np.ctypeslib.as_array(p, shape=(k,)).copy() if k else np.empty(0, np.uint32)
        return {
            "fwd_tw": get(self.s.fwd_tw, n - 1), "inv_tw": get(self.s.inv_tw, n - 1),
            "twists": get(self.s.twists, n), "untwists": get(self.s.untwists, n),
            "generator": self.s.generator, "omega": self.s.omega, "psi": self.s.psi,
            "inv_scale": self.s.inv_scale,
        }

    def forward(self, polys):
        a, p = _u32(np.array(polys, dtype=np.uint32, copy=True))
        lib().orc_twisted_forward(self._ref(), p, a.size // self.n)
        return a

    def inverse(self, evals):
        a, p = _u32(np.array(evals, dtype=np.uint32, copy=True))
        lib().orc_twisted_inverse(self._ref(), p, a.size // self.n)
        return a

    def ntt_forward_cyclic(self, v):
        a, p = _u32(np.array(v, dtype=np.uint32, copy=True))
        lib().orc_ntt_forward(self._ref(), p)
        return a

    def ntt_inverse_cyclic(self, v):
        a, p = _u32(np.array(v, dtype=np.uint32, copy=True))
        lib().orc_ntt_inverse(self._ref(), p)
        return a

    def ntt_mul_inverse(self, a, b, threads: int = 1, avx2: bool = False):
        """INTT(NTT(a) * b) per polynomial; avx2 runs the AVX2 restatement of
        the reference's x86 path (same words)."""
        a, pa = _u32(a)
        b, pb = _u32(b)
        out = np.empty_like(a)
        cnt = a.size // self.n
        po = out.ctypes.data_as(_u32p)
        if threads == 1:
            (lib().orc_ntt_mul_inverse_avx2 if avx2 else lib().orc_ntt_mul_inverse)(
                self._ref(), pa, pb, po, cnt)
        else:
            (lib().orc_ntt_mul_inverse_avx2_mt if avx2 else lib().orc_ntt_mul_inverse_mt)(
                self._ref(), pa, pb, po, cnt, threads)
        return out

    def poly_mul(self, a, b):
        a, pa = _u32(a)
        b, pb = _u32(b)
        out = np.empty(self.n, dtype=np.uint32)
        lib().orc_poly_mul_ntt(self._ref(), pa, pb, out.ctypes.data_as(_u32p))
        return out

    def naive_negacyclic(self, a, b):
        a, pa = _u32(a)
        b, pb = _u32(b)
        out = np.empty(self.n, dtype=np.uint32)
        lib().orc_naive_negacyclic(C.byref(self.s.f), self.n, pa, pb, out.ctypes.data_as(_u32p))
        return out

    def matvec(self, A, rows, cols, s, batch, a_is_eval=False, threads=1, avx2=False):
        A, pA = _u32(A)
        s, ps = _u32(s)
        t = np.empty(batch * rows * self.n, dtype=np.uint32)
        if avx2:  # the AVX2 restatement of the reference's x86 path, same words
            st = lib().orc_matvec_avx2(self._ref(), pA, rows, cols, int(a_is_eval), ps, batch,
                                       t.ctypes.data_as(_u32p), threads)
        elif threads == 1:
            st = lib().orc_matvec(self._ref(), pA, rows, cols, int(a_is_eval), ps, batch,
                                  t.ctypes.data_as(_u32p))
        else:
            st = lib().orc_matvec_mt(self._ref(), pA, rows, cols, int(a_is_eval), ps, batch,
                                     t.ctypes.data_as(_u32p), threads)
        if st:
            raise OracleError(st)
        return t

    def linear_commit(self, a_msg, rows, msg_cols, a_open, open_cols, m, r):
        am, pam = _u32(a_msg)
        ao, pao = _u32(a_open)
        mm, pm = _u32(m)
        rr, pr = _u32(r)
        t = np.empty(rows * self.n, dtype=np.uint32)
        st = lib().orc_linear_commit(self._ref(), pam, rows, msg_cols, pao, open_cols, pm, pr,
                                     t.ctypes.data_as(_u32p))
        if st:
            raise OracleError(st)
        return t

    def gram(self, S, r, n, threads=0, naive=False):
        S, pS = _u32(S)
        G = np.empty(r * (r + 1) // 2 * self.n, dtype=np.uint32)
        if naive:
            st = lib().orc_gram_naive(self._ref(), pS, r, n, G.ctypes.data_as(_u32p))
        else:
            st = lib().orc_gram(self._ref(), pS, r, n, G.ctypes.data_as(_u32p), threads)
        if st:
            raise OracleError(st)
        return G


    def garbage_h(self, S, Phi, r, n):
        """h_ij = (<phi_i, s_j> + <phi_j, s_i>) 2^-1, i <= j (garbage.rs:101-133)."""
        S, pS = _u32(S)
        Phi, pP = _u32(Phi)
        H = np.empty(r * (r + 1) // 2 * self.n, dtype=np.uint32)
        st = lib().orc_garbage_h(self._ref(), pS, pP, r, n, H.ctypes.data_as(_u32p))
        if st:
            raise OracleError(st)
        return H

    def jl_evals(self, flat, rows, parts, num_parts, n):
        """evals[m] = sum_{i,j} conj(pi_{m,i,j}) s_{i,j} from the flat int8 JL
        entries (mod.rs:885-923, step_prover.rs:185-206)."""
        fl = np.ascontiguousarray(flat, dtype=np.int8)
        pa, pp = _u32(parts)
        out = np.empty(rows * self.n, dtype=np.uint32)
        st = lib().orc_jl_evals(self._ref(), fl.ctypes.data_as(_i8p), rows, pp, num_parts, n,
                                out.ctypes.data_as(_u32p))
        if st:
            raise OracleError(st)
        return out

    def amortize(self, S, c, r, n):
        """z[k] = sum_i c_i s_i[k] (amortization.rs:75-81); c: r challenge polys."""
        S, pS = _u32(S)
        c, pc = _u32(c)
        Z = np.empty(n * self.n, dtype=np.uint32)
        st = lib().orc_amortize(self._ref(), pS, pc, r, n, Z.ctypes.data_as(_u32p))
        if st:
            raise OracleError(st)
        return Z


def sample_uniform_polys(field: Field, seed: bytes, npolys: int, d: int, accept_max: int = 0):
    """npolys uniform ring elements from ChaCha20Rng(seed) in CommitKey::from_seed
    order (crs.rs:136-198, 308-326; prime.rs:730-743), Montgomery words."""
    out = np.empty(npolys * d, dtype=np.uint32)
    sd = (C.c_uint8 * 32).from_buffer_copy(seed)
    st = lib().orc_sample_uniform_polys(C.byref(field.s), sd, npolys, d, accept_max,
                                        out.ctypes.data_as(_u32p))
    if st:
        raise OracleError(st)
    return out


def decompose_coeff_balanced(c: int, base: int, num_limbs: int, q: int):
    out = (C.c_int64 * num_limbs)()
    lib().orc_decompose_coeff_balanced(c, base, num_limbs, q, out)
    return list(out)


def centered_mod(v: int, base: int) -> int:
    return lib().orc_centered_mod(v, base)


def garbage_index(r: int, i: int, j: int) -> int:
    return lib().orc_garbage_index(r, i, j)


def max_ntt_size(q: int) -> int:
    return lib().orc_max_ntt_size(q)


def is_prime(q: int) -> bool:
    return bool(lib().orc_is_prime_u64(q))


def decompose_polys(field: Field, d: int, polys, base: int, num_limbs: int):
    p, pp = _u32(polys)
    npolys = p.size // d
    out = np.empty(npolys * num_limbs * d, dtype=np.uint32)
    st = lib().orc_decompose_polys(C.byref(field.s), d, pp, npolys, base, num_limbs,
                                   out.ctypes.data_as(_u32p))
    if st:
        raise OracleError(st)
    return out


def reconstruct_from_limbs(field: Field, d: int, limbs, base: int):
    l, pl = _u32(limbs)
    out = np.empty(d, dtype=np.uint32)
    lib().orc_reconstruct_from_limbs(C.byref(field.s), d, pl, l.size // d, base,
                                     out.ctypes.data_as(_u32p))
    return out


def gadget_digits(q: int, base: int) -> int:
    return lib().orc_gadget_digits(q, base)


def gadget_decompose(field: Field, x, base: int):
    x, px = _u32(x)
    k = gadget_digits(field.q, base)
    out = np.empty(k * x.size, dtype=np.uint32)
    st = lib().orc_gadget_decompose(C.byref(field.s), px, x.size, base, out.ctypes.data_as(_u32p))
    if st:
        raise OracleError(st)
    return out.reshape(k, x.size)


def chacha20_block(key: bytes, counter: int, nonce: bytes) -> bytes:
    k = (C.c_uint8 * 32).from_buffer_copy(key)
    n = (C.c_uint8 * 12).from_buffer_copy(nonce)
    out = (C.c_uint8 * 64)()
    lib().orc_chacha20_block(k, counter, n, out)
    return bytes(out)


def chacha20_quarter(a, b, c, d):
    v = [C.c_uint32(x) for x in (a, b, c, d)]
    lib().orc_chacha20_quarter(*[C.byref(x) for x in v])
    return tuple(x.value for x in v)


def jl_project(field: Field, seed: bytes, rows: int, parts, num_parts: int, cols: int, d: int,
               want_flat: bool = True, threads: int = 0):
    parts, pp = _u32(parts)
    assert parts.size == num_parts * cols
    sd = (C.c_uint8 * 32).from_buffer_copy(seed)
    p = np.empty(rows, dtype=np.uint32)
    flat = np.zeros(rows * num_parts * cols, dtype=np.int8) if want_flat else None
    st = lib().orc_jl_project(C.byref(field.s), sd, rows, cols, pp, num_parts, d,
                              p.ctypes.data_as(_u32p),
                              flat.ctypes.data_as(_i8p) if want_flat else None, threads)
    if st:
        raise OracleError(st)
    return p, flat
