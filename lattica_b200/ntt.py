"""Twisted negacyclic NTT plans on the GPU, mirroring the reference's
`TwistedNttPlan` / `twisted_ntt_plan` / `poly_mul_ntt` surface
(algebra/src/poly/ntt.rs:25-319).

Inputs are uint32 PrimeField<Q, u32> Montgomery words shaped (..., d):
numpy arrays use the host-buffer ABI calls, CUDA torch tensors the *_dev calls
on the current torch stream. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import _lib
from ._lib import GridGpuError, PlanInfo, check


class NttError(ValueError):
    """Mirror of NttError (algebra/src/arith/ntt.rs:40-50)."""

    KINDS = {1: "LengthMismatch", 2: "LengthNotPowerOfTwo", 3: "UnsupportedSize",
             4: "UnsupportedTwist"}

    def __init__(self, kind: str, **fields):
        self.kind = kind
        self.fields = fields
        inner = ", ".join(f"{k}: {v}" for k, v in fields.items())
        super().__init__(f"{kind} {{ {inner} }}")

    def __eq__(self, other):
        return isinstance(other, NttError) and (self.kind, self.fields) == (other.kind, other.fields)

    __hash__ = None


class CommitmentError(ValueError):
    """Mirror of CommitmentError (commit/src/error.rs:7-18)."""

    def __init__(self, kind: str):
        self.kind = kind
        super().__init__(kind)

    def __eq__(self, other):
        return isinstance(other, CommitmentError) and self.kind == other.kind

    __hash__ = None


def raise_status(code: int, where: str, length: int = 0) -> None:
    if code == 0:
        return
    if code in (2, 3, 4):
        raise NttError(NttError.KINDS[code], len=length)
    if code == 5:
        raise CommitmentError("InvalidParameters")
    if code == 6:
        raise CommitmentError("DimensionMismatch")
    raise GridGpuError(code, where)


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _stream_ptr(t) -> int:
    import torch
    return torch.cuda.current_stream(t.device).cuda_stream


def _host_u32(a: np.ndarray) -> np.ndarray:
    if not isinstance(a, np.ndarray) or a.dtype != np.uint32 or not a.flags.c_contiguous:
        raise TypeError("expected a C-contiguous numpy uint32 array")
    return a


def _dev_u32(t):
    import torch
    if t.dtype not in (torch.int32, torch.uint32) or not t.is_cuda or not t.is_contiguous():
        raise TypeError("expected a contiguous CUDA tensor of 32-bit words")
    return t


class TwistedNttPlan:
    """Twisted negacyclic NTT of length d over Z_q (TwistedNttPlan::build,
    algebra/src/poly/ntt.rs:139-154); owns device twiddles and scratch."""

    _create = "grid_gpu_plan_create"

    def __init__(self, q: int, d: int):
        lib = _lib.load()
        handle = C.c_void_p()
        st = getattr(lib, self._create)(int(q), int(d), C.byref(handle))
        raise_status(st, self._create, length=int(d))
        self._h = handle
        self._lib = lib
        self.q, self.d = int(q), int(d)
        info = PlanInfo()
        check(lib.grid_gpu_plan_get_info(handle, C.byref(info)), "grid_gpu_plan_get_info")
        self.info = info

    # reference accessors
    def len(self) -> int:
        return self.d

    def is_empty(self) -> bool:
        return self.d == 0

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.grid_gpu_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def twiddles(self):
        z = np.zeros(self.d, np.uint32)
        iz = np.zeros(self.d, np.uint32)
        check(self._lib.grid_gpu_plan_get_twiddles(self._h, z.ctypes.data, iz.ctypes.data),
              "grid_gpu_plan_get_twiddles")
        return z, iz

    def check_device(self, stream=None):
        raise_status(self._lib.grid_gpu_plan_check(self._h, stream), "grid_gpu_plan_check")

    # -- validation mirroring validate_len (poly/ntt.rs:44-52)
    def _npolys(self, x) -> int:
        shape = tuple(x.shape)
        if len(shape) == 0 or shape[-1] != self.d:
            raise NttError("LengthMismatch", left=self.d, right=shape[-1] if shape else 0)
        n = 1
        for s in shape[:-1]:
            n *= int(s)
        return n

    # -- transforms
    def forward_in_place(self, coeffs):
        n = self._npolys(coeffs)
        if _is_torch(coeffs):
            _dev_u32(coeffs)
            st = self._lib.grid_gpu_ntt_forward_dev(self._h, coeffs.data_ptr(), n,
                                                    _stream_ptr(coeffs))
        else:
            _host_u32(coeffs)
            st = self._lib.grid_gpu_ntt_forward(self._h, coeffs.ctypes.data, n)
        raise_status(st, "grid_gpu_ntt_forward")

    def inverse_in_place(self, evals):
        n = self._npolys(evals)
        if _is_torch(evals):
            _dev_u32(evals)
            st = self._lib.grid_gpu_ntt_inverse_dev(self._h, evals.data_ptr(), n,
                                                    _stream_ptr(evals))
        else:
            _host_u32(evals)
            st = self._lib.grid_gpu_ntt_inverse(self._h, evals.ctypes.data, n)
        raise_status(st, "grid_gpu_ntt_inverse")

    def ntt_mul_inverse(self, a, b_evals, out=None):
        """out = INTT(NTT(a) (.) b_evals) for a batch of polys."""
        n = self._npolys(a)
        if tuple(b_evals.shape) != tuple(a.shape):
            raise NttError("LengthMismatch", left=int(np.prod(a.shape)),
                           right=int(np.prod(b_evals.shape)))
        if _is_torch(a):
            import torch
            out = torch.empty_like(a) if out is None else out
            _dev_u32(a), _dev_u32(b_evals), _dev_u32(out)
            st = self._lib.grid_gpu_ntt_mul_inverse_dev(self._h, a.data_ptr(), b_evals.data_ptr(),
                                                        out.data_ptr(), n, _stream_ptr(a))
        else:
            out = np.empty_like(a) if out is None else out
            _host_u32(a), _host_u32(b_evals), _host_u32(out)
            st = self._lib.grid_gpu_ntt_mul_inverse(self._h, a.ctypes.data, b_evals.ctypes.data,
                                                    out.ctypes.data, n)
        raise_status(st, "grid_gpu_ntt_mul_inverse")
        return out

    def multiply_in_place(self, lhs, rhs):
        """lhs <- lhs * rhs mod (X^d + 1) (multiply_in_place, poly/ntt.rs:110-126)."""
        if tuple(lhs.shape) != tuple(rhs.shape):
            raise NttError("LengthMismatch", left=lhs.shape[-1], right=rhs.shape[-1])
        n = self._npolys(lhs)
        if _is_torch(lhs):
            import torch
            words = self._lib.grid_gpu_poly_mul_scratch_words(self._h, n)
            scratch = torch.empty(max(4, words), dtype=torch.int32, device=lhs.device)
            st = self._lib.grid_gpu_poly_mul_dev(self._h, lhs.data_ptr(), rhs.data_ptr(),
                                                 lhs.data_ptr(), scratch.data_ptr(), n,
                                                 _stream_ptr(lhs))
        else:
            _host_u32(lhs), _host_u32(rhs)
            st = self._lib.grid_gpu_poly_mul(self._h, lhs.ctypes.data, rhs.ctypes.data,
                                             lhs.ctypes.data, n)
        raise_status(st, "grid_gpu_poly_mul")

    # -- slice hooks of Ring for PrimeField (algebra/src/arith/prime.rs:433-491),
    #    on CUDA tensors of canonical words, in place on the current torch stream
    def _slice_args(self, dst, src=None):
        _dev_u32(dst)
        if src is not None:
            _dev_u32(src)
            if src.numel() != dst.numel():
                raise NttError("LengthMismatch", left=dst.numel(), right=src.numel())
        return dst.numel(), _stream_ptr(dst)

    def pointwise_mul_assign_slice(self, dst, rhs):
        n, s = self._slice_args(dst, rhs)
        raise_status(self._lib.grid_gpu_pointwise_mul_dev(self._h, dst.data_ptr(), rhs.data_ptr(),
                                                          n, s), "grid_gpu_pointwise_mul_dev")

    def add_assign_slice(self, dst, src):
        n, s = self._slice_args(dst, src)
        raise_status(self._lib.grid_gpu_add_assign_dev(self._h, dst.data_ptr(), src.data_ptr(),
                                                       n, s), "grid_gpu_add_assign_dev")

    def sub_assign_slice(self, dst, src):
        n, s = self._slice_args(dst, src)
        raise_status(self._lib.grid_gpu_sub_assign_dev(self._h, dst.data_ptr(), src.data_ptr(),
                                                       n, s), "grid_gpu_sub_assign_dev")

    def scalar_mul_slice(self, dst, scalar: int):
        n, s = self._slice_args(dst)
        raise_status(self._lib.grid_gpu_scalar_mul_dev(self._h, dst.data_ptr(), int(scalar), n, s),
                     "grid_gpu_scalar_mul_dev")

    def add_assign_scaled_slice(self, dst, src, scalar: int):
        n, s = self._slice_args(dst, src)
        raise_status(self._lib.grid_gpu_add_assign_scaled_dev(
            self._h, dst.data_ptr(), src.data_ptr(), int(scalar), n, s),
            "grid_gpu_add_assign_scaled_dev")

    # -- PrimeField<Q, u64> words (value * 2^64 mod q, the reference's default
    #    limb) to and from this library's u32 words, on CUDA tensors
    def words_from_u64(self, w64):
        """int64 tensor of u64 Montgomery words -> int32 tensor of u32 words;
        raises ValueError if a word is not canonical (>= q)."""
        import torch
        if w64.dtype not in (torch.int64, torch.uint64) or not w64.is_cuda or not w64.is_contiguous():
            raise TypeError("expected a contiguous CUDA tensor of 64-bit words")
        out = torch.empty(w64.shape, dtype=torch.int32, device=w64.device)
        flag = torch.zeros(4, dtype=torch.int32, device=w64.device)
        raise_status(self._lib.grid_gpu_words_from_u64_dev(
            self._h, w64.data_ptr(), w64.numel(), out.data_ptr(), flag.data_ptr(),
            _stream_ptr(w64)), "grid_gpu_words_from_u64_dev")
        if int(flag[0].item()):
            raise ValueError("a u64 word is not canonical (>= q)")
        return out

    def words_to_u64(self, w32):
        """int32 tensor of u32 words -> int64 tensor of u64 Montgomery words."""
        import torch
        _dev_u32(w32)
        out = torch.empty(w32.shape, dtype=torch.int64, device=w32.device)
        raise_status(self._lib.grid_gpu_words_to_u64_dev(
            self._h, w32.data_ptr(), w32.numel(), out.data_ptr(), _stream_ptr(w32)),
            "grid_gpu_words_to_u64_dev")
        return out

    def dot_product(self, lhs, rhs) -> int:
        import torch
        n, s = self._slice_args(lhs, rhs)
        out = torch.empty(4, dtype=torch.int32, device=lhs.device)
        raise_status(self._lib.grid_gpu_dot_product_dev(self._h, lhs.data_ptr(), rhs.data_ptr(),
                                                        n, out.data_ptr(), s),
                     "grid_gpu_dot_product_dev")
        return int(out[0].item()) & 0xFFFFFFFF


class RingPlan(TwistedNttPlan):
    """Arithmetic of CyclotomicPolyRing<PrimeField<q>, d>, whatever q: the NTT
    plan when q has a 2d-th root of unity, else exact products through three
    auxiliary NTT primes with the schoolbook rule's words
    (NegacyclicMulRing::negacyclic_mul_coeffs, algebra/src/poly/ring.rs:60-100).
    Every ring-level call of this package accepts it in place of a
    TwistedNttPlan; NTT calls on a plan without an NTT for q raise the NttError
    TwistedNttPlan::build would."""

    _create = "grid_gpu_ring_plan_create"

    @property
    def uses_aux_primes(self) -> bool:
        kind = C.c_int()
        raise_status(self._lib.grid_gpu_plan_ring_kind(self._h, C.byref(kind), None),
                     "grid_gpu_plan_ring_kind")
        return kind.value == 1


_PLANS: dict = {}
_PLANS_LOCK = threading.Lock()


def twisted_ntt_plan(q: int, d: int) -> TwistedNttPlan:
    """Cached plan per (device, q, d), like cached_twisted_plan (poly/ntt.rs:163-178)."""
    try:
        import torch
        dev = torch.cuda.current_device() if torch.cuda.is_available() else -1
    except Exception:
        dev = -1
    key = (dev, int(q), int(d))
    with _PLANS_LOCK:
        plan = _PLANS.get(key)
        if plan is None:
            plan = TwistedNttPlan(q, d)
            _PLANS[key] = plan
        return plan


def poly_mul_ntt(a, b, q: int):
    """Negacyclic product of equal-length coefficient arrays (poly_mul_ntt, poly/ntt.rs:305-319)."""
    if a.shape[-1] != b.shape[-1]:
        raise NttError("LengthMismatch", left=a.shape[-1], right=b.shape[-1])
    plan = twisted_ntt_plan(q, a.shape[-1])
    lhs = a.clone() if _is_torch(a) else np.array(a, dtype=np.uint32, copy=True)
    plan.multiply_in_place(lhs, b)
    return lhs
