"""Commitments on the GPU, mirroring the reference's linear / Ajtai / gadget
commitment surface (commit/src/linear.rs, commit/src/ajtai/mod.rs,
commit/src/gadget/mod.rs).

A `PreparedMatrix` is the device-resident twisted-domain copy of a ring
matrix: the GPU counterpart of the `PreparedRuntimeCache` that
`PreparedLinearOps::build_linear_key_cache` / `build_matrix_cache` build once
at setup (commit/src/linear.rs:576-715). Ring vectors are numpy uint32 arrays
of Montgomery words shaped (..., len, d) on the host, or CUDA int32 tensors.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .ntt import CommitmentError, TwistedNttPlan, _is_torch, _stream_ptr, raise_status


@dataclass(frozen=True)
class CommitmentDimensions:
    """CommitmentDimensions (commit/src/linear.rs:34-60)."""

    message_len: int
    opening_len: int
    commitment_len: int

    def validate(self) -> None:
        if self.message_len == 0 or self.opening_len == 0 or self.commitment_len == 0:
            raise CommitmentError("InvalidParameters")
        limit = 1 << 64
        if (self.commitment_len * self.message_len >= limit
                or self.commitment_len * self.opening_len >= limit):
            raise CommitmentError("InvalidParameters")


class PreparedMatrix:
    """Device-resident rows x cols ring matrix in the twisted evaluation domain."""

    def __init__(self, plan: TwistedNttPlan, A, rows: int, cols: int, is_evals: bool = False):
        lib = _lib.load()
        h = C.c_void_p()
        if _is_torch(A):
            st = lib.grid_gpu_matrix_create_dev(plan.handle, A.data_ptr(), rows, cols,
                                                int(is_evals), C.byref(h), _stream_ptr(A))
        else:
            A = np.ascontiguousarray(A, dtype=np.uint32)
            if A.size != rows * cols * plan.d:
                raise CommitmentError("DimensionMismatch")
            st = lib.grid_gpu_matrix_create(plan.handle, A.ctypes.data, rows, cols,
                                            int(is_evals), C.byref(h))
        raise_status(st, "grid_gpu_matrix_create")
        self._h, self._lib, self.plan = h, lib, plan
        self.rows, self.cols = rows, cols

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.grid_gpu_matrix_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def workspace_bytes(self, batch: int) -> int:
        n = C.c_size_t()
        raise_status(self._lib.grid_gpu_commit_workspace(self._h, batch, C.byref(n)),
                     "grid_gpu_commit_workspace")
        return n.value

    def mul_vec(self, s):
        """t[b] = A * s[b] for s shaped (batch, cols, d) (RingMat::mul_slice /
        mul_matrix_vector_runtime)."""
        d = self.plan.d
        if tuple(s.shape[-2:]) != (self.cols, d):
            raise CommitmentError("DimensionMismatch")
        batch = int(np.prod(s.shape[:-2])) if len(s.shape) > 2 else 1
        if _is_torch(s):
            import torch
            t = torch.empty((*s.shape[:-2], self.rows, d), dtype=s.dtype, device=s.device)
            ws = torch.empty(max(16, self.workspace_bytes(batch)), dtype=torch.uint8,
                             device=s.device)
            st = self._lib.grid_gpu_commit_dev(self._h, s.data_ptr(), batch, t.data_ptr(),
                                               ws.data_ptr(), ws.numel(), _stream_ptr(s))
        else:
            s = np.ascontiguousarray(s, dtype=np.uint32)
            t = np.empty((*s.shape[:-2], self.rows, d), dtype=np.uint32)
            st = self._lib.grid_gpu_commit(self._h, s.ctypes.data, batch, t.ctypes.data)
        raise_status(st, "grid_gpu_commit")
        return t


class LinearCommitmentKey:
    """LinearCommitmentKey (commit/src/linear.rs:154-160) with its prepared cache."""

    def __init__(self, plan: TwistedNttPlan, a_msg, a_open, dims: CommitmentDimensions):
        dims.validate()
        d = plan.d
        if not _is_torch(a_msg):
            a_msg = np.ascontiguousarray(a_msg, dtype=np.uint32)
        if not _is_torch(a_open):
            a_open = np.ascontiguousarray(a_open, dtype=np.uint32)
        size = lambda a: a.numel() if _is_torch(a) else a.size
        if (size(a_msg) != dims.commitment_len * dims.message_len * d
                or size(a_open) != dims.commitment_len * dims.opening_len * d):
            raise CommitmentError("DimensionMismatch")  # validate_linear_matrices
        self.plan, self.dims = plan, dims
        self.a_msg = PreparedMatrix(plan, a_msg, dims.commitment_len, dims.message_len)
        self.a_open = PreparedMatrix(plan, a_open, dims.commitment_len, dims.opening_len)

    def recompute(self, message, randomness):
        """t = A_msg * m + A_open * r (recompute_linear_commitment_parts_trusted,
        commit/src/linear.rs:476-506); message (batch?, message_len, d),
        randomness (batch?, opening_len, d): numpy uint32 or CUDA tensors."""
        d = self.plan.d
        if tuple(message.shape[-2:]) != (self.dims.message_len, d):
            raise CommitmentError("DimensionMismatch")  # validate_message
        if tuple(randomness.shape[-2:]) != (self.dims.opening_len, d):
            raise CommitmentError("DimensionMismatch")  # validate_opening_randomness
        batch = int(np.prod(message.shape[:-2])) if len(message.shape) > 2 else 1
        if (int(np.prod(randomness.shape[:-2])) if len(randomness.shape) > 2 else 1) != batch:
            raise CommitmentError("DimensionMismatch")
        if _is_torch(message):
            import torch
            lib = _lib.load()
            t = torch.empty((*message.shape[:-2], self.dims.commitment_len, d),
                            dtype=message.dtype, device=message.device)
            nb = C.c_size_t()
            raise_status(lib.grid_gpu_linear_commit_workspace(self.a_msg.handle,
                                                              self.a_open.handle, batch,
                                                              C.byref(nb)),
                         "grid_gpu_linear_commit_workspace")
            ws = torch.empty(max(16, nb.value), dtype=torch.uint8, device=message.device)
            st = lib.grid_gpu_linear_commit_dev(self.a_msg.handle, self.a_open.handle,
                                                message.data_ptr(), randomness.data_ptr(), batch,
                                                t.data_ptr(), ws.data_ptr(), ws.numel(),
                                                _stream_ptr(message))
            raise_status(st, "grid_gpu_linear_commit_dev")
            return t
        m = np.ascontiguousarray(message, dtype=np.uint32)
        r = np.ascontiguousarray(randomness, dtype=np.uint32)
        t = np.empty((*m.shape[:-2], self.dims.commitment_len, d), dtype=np.uint32)
        st = _lib.load().grid_gpu_linear_commit(self.a_msg.handle, self.a_open.handle,
                                                m.ctypes.data, r.ctypes.data, batch,
                                                t.ctypes.data)
        raise_status(st, "grid_gpu_linear_commit")
        return t


class BdlopCommitmentKey:
    """BdlopCommitmentKey (commit/src/bdlop/params.rs:90-135) with its three
    matrices prepared on the device: A_mask (rows x opening_len), A_msg
    (rows x message_len), A_open (rows x opening_len)."""

    def __init__(self, plan: TwistedNttPlan, a_mask, a_msg, a_open, rows: int,
                 message_len: int, opening_len: int):
        d = plan.d
        mats = []
        for a, cols in ((a_mask, opening_len), (a_msg, message_len), (a_open, opening_len)):
            if not _is_torch(a):
                a = np.ascontiguousarray(a, dtype=np.uint32)
            if rows == 0 or cols == 0 or (a.numel() if _is_torch(a) else a.size) != rows * cols * d:
                raise CommitmentError("DimensionMismatch")  # BdlopCommitmentKey::is_valid
            mats.append(PreparedMatrix(plan, a, rows, cols))
        self.plan, self.rows = plan, rows
        self.message_len, self.opening_len = message_len, opening_len
        self.a_mask, self.a_msg, self.a_open = mats

    def recompute_parts(self, message, randomness):
        """(u, v) = (A_mask r, A_msg m + A_open r) per batch entry
        (recompute_bdlop_parts_runtime, commit/src/linear.rs:552-573, 800-938).
        message (batch?, message_len, d), randomness (batch?, opening_len, d):
        numpy uint32 or CUDA tensors (both the same kind)."""
        d = self.plan.d
        if tuple(message.shape[-2:]) != (self.message_len, d):
            raise CommitmentError("DimensionMismatch")
        if tuple(randomness.shape[-2:]) != (self.opening_len, d):
            raise CommitmentError("DimensionMismatch")
        batch = int(np.prod(message.shape[:-2])) if len(message.shape) > 2 else 1
        if (int(np.prod(randomness.shape[:-2])) if len(randomness.shape) > 2 else 1) != batch:
            raise CommitmentError("DimensionMismatch")
        lib = _lib.load()
        shape = (*message.shape[:-2], self.rows, d)
        if _is_torch(message):
            import torch
            u = torch.empty(shape, dtype=message.dtype, device=message.device)
            v = torch.empty(shape, dtype=message.dtype, device=message.device)
            nb = C.c_size_t()
            raise_status(lib.grid_gpu_bdlop_workspace(self.a_mask.handle, self.a_msg.handle,
                                                      self.a_open.handle, batch, C.byref(nb)),
                         "grid_gpu_bdlop_workspace")
            ws = torch.empty(max(16, nb.value), dtype=torch.uint8, device=message.device)
            st = lib.grid_gpu_bdlop_commit_dev(self.a_mask.handle, self.a_msg.handle,
                                               self.a_open.handle, message.data_ptr(),
                                               randomness.data_ptr(), batch, u.data_ptr(),
                                               v.data_ptr(), ws.data_ptr(), ws.numel(),
                                               _stream_ptr(message))
        else:
            m = np.ascontiguousarray(message, dtype=np.uint32)
            r = np.ascontiguousarray(randomness, dtype=np.uint32)
            u = np.empty(shape, dtype=np.uint32)
            v = np.empty(shape, dtype=np.uint32)
            st = lib.grid_gpu_bdlop_commit(self.a_mask.handle, self.a_msg.handle,
                                           self.a_open.handle, m.ctypes.data, r.ctypes.data,
                                           batch, u.ctypes.data, v.ctypes.data)
        raise_status(st, "grid_gpu_bdlop_commit")
        return u, v


class AjtaiCommitment:
    """Ajtai commitment t = A_msg * m + A_open * r with device-resident keys
    (AjtaiCommitmentScheme::commit_with_opening, commit/src/ajtai/mod.rs:443-452).
    The keys are passed in (sampling is host-side and out of the hot path)."""

    def __init__(self, plan: TwistedNttPlan, a_msg, a_open, dims: CommitmentDimensions):
        self.key = LinearCommitmentKey(plan, a_msg, a_open, dims)

    def commit_with_opening(self, message, randomness):
        return self.key.recompute(message, randomness)


def gadget_digits(q: int, base: int) -> int:
    n = C.c_size_t()
    raise_status(_lib.load().grid_gpu_gadget_digits(q, base, C.byref(n)), "grid_gpu_gadget_digits")
    return n.value


def gadget_decompose(plan: TwistedNttPlan, x, base: int, digit_major: bool = True):
    """Unsigned base-`base` digits (gadget_decompose, algebra/src/poly/decomposition.rs:47-61).
    digit_major=True -> shape (k, len); False -> per-polynomial (npolys, k, d) like
    GadgetRing::decompose_element (commit/src/gadget/mod.rs:151-162)."""
    x = np.ascontiguousarray(x, dtype=np.uint32)
    k = gadget_digits(plan.q, base)
    if digit_major:
        out = np.empty((k, x.size), dtype=np.uint32)
    else:
        out = np.empty((x.size // plan.d, k, plan.d), dtype=np.uint32)
    st = _lib.load().grid_gpu_gadget_decompose(plan.handle, x.ctypes.data, x.size, base,
                                               int(digit_major), out.ctypes.data)
    raise_status(st, "grid_gpu_gadget_decompose")
    return out
