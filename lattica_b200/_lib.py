"""ctypes binding of the C ABI in include/grid_gpu.h (libgridgpu.so).

The product path has no CPU fallback: if the shared library is missing or a
GPU is absent, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgridgpu.so")

GRID_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "LengthMismatch", 2: "LengthNotPowerOfTwo", 3: "UnsupportedSize",
    4: "UnsupportedTwist", 5: "InvalidParameters", 6: "DimensionMismatch",
    7: "InvalidModulus", 8: "NullPointer", 9: "OutOfMemory", 10: "Cuda", 11: "Timeout",
    12: "UnsupportedDegree", 13: "Misaligned", 14: "NoDevice", 15: "ScratchLimit",
    16: "SampleExhausted",
}

_u32p = C.POINTER(C.c_uint32)
_vp = C.c_void_p


class BatchItem(C.Structure):
    _fields_ = [("s_offset", C.c_uint64), ("t_offset", C.c_uint64), ("n", C.c_uint32),
                ("matrix", C.c_uint32)]


class BatchConfig(C.Structure):
    _fields_ = [("k_split", C.c_uint32), ("work_items", C.c_uint32), ("tiles", C.c_uint32),
                ("tile_instances", C.c_uint32), ("engine", C.c_uint32),
                ("tensor_cores", C.c_uint32)]


class GramItem(C.Structure):
    _fields_ = [("s_offset", C.c_uint64), ("r", C.c_uint32), ("n", C.c_uint32)]


ENGINE_AUTO, ENGINE_TENSOR, ENGINE_CUDA_CORE, ENGINE_POINT_MAJOR = 0, 1, 2, 3


class PlanInfo(C.Structure):
    _fields_ = [("q", C.c_uint32), ("d", C.c_uint32), ("generator", C.c_uint32),
                ("psi", C.c_uint32), ("omega", C.c_uint32), ("n_inv", C.c_uint32),
                ("r_mod_q", C.c_uint32), ("r2_mod_q", C.c_uint32), ("max_ntt_size", C.c_uint64)]


# name -> (restype, argtypes); every symbol declared in include/grid_gpu.h.
SIGNATURES = {
    "grid_gpu_status_string": (C.c_char_p, [C.c_int]),
    "grid_gpu_abi_version": (C.c_uint32, []),
    "grid_gpu_max_degree": (C.c_uint32, []),
    "grid_gpu_plan_create": (C.c_int, [C.c_uint64, C.c_uint64, C.POINTER(_vp)]),
    "grid_gpu_plan_destroy": (C.c_int, [_vp]),
    "grid_gpu_ring_plan_create": (C.c_int, [C.c_uint64, C.c_uint64, C.POINTER(_vp)]),
    "grid_gpu_plan_ring_kind": (C.c_int, [_vp, C.POINTER(C.c_int), _vp]),
    "grid_gpu_poly_mul_scratch_words": (C.c_size_t, [_vp, C.c_size_t]),
    "grid_gpu_plan_describe": (C.c_int, [C.c_uint64, C.c_uint64, C.POINTER(PlanInfo), _vp, _vp]),
    "grid_gpu_plan_get_info": (C.c_int, [_vp, C.POINTER(PlanInfo)]),
    "grid_gpu_plan_get_twiddles": (C.c_int, [_vp, _vp, _vp]),
    "grid_gpu_plan_check": (C.c_int, [_vp, _vp]),
    "grid_gpu_selftest_wait_timeout_dev": (C.c_int, [_vp, C.c_uint32, _vp]),
    "grid_gpu_ntt_forward_dev": (C.c_int, [_vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_ntt_inverse_dev": (C.c_int, [_vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_ntt_mul_inverse_dev": (C.c_int, [_vp, _vp, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_poly_mul_dev": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_pointwise_mul_dev": (C.c_int, [_vp, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_add_assign_dev": (C.c_int, [_vp, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_sub_assign_dev": (C.c_int, [_vp, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_scalar_mul_dev": (C.c_int, [_vp, _vp, C.c_uint32, C.c_size_t, _vp]),
    "grid_gpu_add_assign_scaled_dev": (C.c_int, [_vp, _vp, _vp, C.c_uint32, C.c_size_t, _vp]),
    "grid_gpu_dot_product_dev": (C.c_int, [_vp, _vp, _vp, C.c_size_t, _vp, _vp]),
    "grid_gpu_words_from_u64_dev": (C.c_int, [_vp, _vp, C.c_size_t, _vp, _vp, _vp]),
    "grid_gpu_words_to_u64_dev": (C.c_int, [_vp, _vp, C.c_size_t, _vp, _vp]),
    "grid_gpu_ntt_forward": (C.c_int, [_vp, _vp, C.c_size_t]),
    "grid_gpu_ntt_inverse": (C.c_int, [_vp, _vp, C.c_size_t]),
    "grid_gpu_ntt_mul_inverse": (C.c_int, [_vp, _vp, _vp, _vp, C.c_size_t]),
    "grid_gpu_poly_mul": (C.c_int, [_vp, _vp, _vp, _vp, C.c_size_t]),
    "grid_gpu_matrix_create": (C.c_int, [_vp, _vp, C.c_size_t, C.c_size_t, C.c_int, C.POINTER(_vp)]),
    "grid_gpu_matrix_create_dev": (C.c_int, [_vp, _vp, C.c_size_t, C.c_size_t, C.c_int,
                                             C.POINTER(_vp), _vp]),
    "grid_gpu_matrix_destroy": (C.c_int, [_vp]),
    "grid_gpu_matrix_view": (C.c_int, [_vp, C.c_size_t, C.POINTER(_vp)]),
    "grid_gpu_matrix_shape": (C.c_int, [_vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "grid_gpu_matrix_device_evals": (C.c_int, [_vp, C.POINTER(_vp)]),
    "grid_gpu_commit_workspace": (C.c_int, [_vp, C.c_size_t, C.POINTER(C.c_size_t)]),
    "grid_gpu_commit_dev": (C.c_int, [_vp, _vp, C.c_size_t, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_commit": (C.c_int, [_vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_linear_commit": (C.c_int, [_vp, _vp, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_gram_workspace": (C.c_int, [_vp, C.c_size_t, C.c_size_t, C.POINTER(C.c_size_t)]),
    "grid_gpu_gram_dev": (C.c_int, [_vp, _vp, C.c_size_t, C.c_size_t, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_gram": (C.c_int, [_vp, _vp, C.c_size_t, C.c_size_t, _vp]),
    "grid_gpu_sample_uniform_polys_workspace": (C.c_int, [_vp, C.c_size_t, C.c_uint64,
                                                          C.POINTER(C.c_size_t)]),
    "grid_gpu_sample_uniform_polys_dev": (C.c_int, [_vp, _vp, C.c_size_t, C.c_uint64, _vp, _vp,
                                                    C.c_size_t, _vp]),
    "grid_gpu_sample_uniform_polys": (C.c_int, [_vp, _vp, C.c_size_t, C.c_uint64, _vp]),
    "grid_gpu_jl_evals_workspace": (C.c_int, [C.POINTER(C.c_size_t)]),
    "grid_gpu_jl_evals_dev": (C.c_int, [_vp, _vp, C.c_size_t, _vp, C.c_size_t, C.c_size_t,
                                        C.c_size_t, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_jl_evals": (C.c_int, [_vp, _vp, C.c_size_t, _vp, C.c_size_t, C.c_size_t,
                                    C.c_size_t, _vp]),
    "grid_gpu_linear_commit_workspace": (C.c_int, [_vp, _vp, C.c_size_t,
                                                   C.POINTER(C.c_size_t)]),
    "grid_gpu_linear_commit_dev": (C.c_int, [_vp, _vp, _vp, _vp, C.c_size_t, _vp, _vp,
                                             C.c_size_t, _vp]),
    "grid_gpu_bdlop_workspace": (C.c_int, [_vp, _vp, _vp, C.c_size_t, C.POINTER(C.c_size_t)]),
    "grid_gpu_bdlop_commit_dev": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_size_t, _vp, _vp, _vp,
                                            C.c_size_t, _vp]),
    "grid_gpu_bdlop_commit": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_size_t, _vp, _vp]),
    "grid_gpu_garbage_h_workspace": (C.c_int, [_vp, C.c_size_t, C.c_size_t,
                                               C.POINTER(C.c_size_t)]),
    "grid_gpu_garbage_h_dev": (C.c_int, [_vp, _vp, _vp, C.c_size_t, C.c_size_t, _vp, _vp,
                                         C.c_size_t, _vp]),
    "grid_gpu_garbage_h": (C.c_int, [_vp, _vp, _vp, C.c_size_t, C.c_size_t, _vp]),
    "grid_gpu_amortize_workspace": (C.c_int, [_vp, C.c_size_t, C.c_size_t,
                                              C.POINTER(C.c_size_t)]),
    "grid_gpu_amortize_dev": (C.c_int, [_vp, _vp, _vp, C.c_size_t, C.c_size_t, _vp, _vp,
                                        C.c_size_t, _vp]),
    "grid_gpu_amortize": (C.c_int, [_vp, _vp, _vp, C.c_size_t, C.c_size_t, _vp]),
    "grid_gpu_jl_workspace": (C.c_int, [C.c_size_t, C.POINTER(C.c_size_t)]),
    "grid_gpu_jl_project_dev": (C.c_int, [_vp, _vp, C.c_size_t, _vp, C.c_size_t, C.c_size_t,
                                          C.c_size_t, _vp, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_jl_project": (C.c_int, [_vp, _vp, C.c_size_t, _vp, C.c_size_t, C.c_size_t,
                                      C.c_size_t, _vp, _vp]),
    "grid_gpu_decompose_balanced_dev": (C.c_int, [_vp, _vp, C.c_size_t, C.c_uint64, C.c_size_t,
                                                  _vp, _vp]),
    "grid_gpu_decompose_balanced": (C.c_int, [_vp, _vp, C.c_size_t, C.c_uint64, C.c_size_t, _vp]),
    "grid_gpu_gadget_digits": (C.c_int, [C.c_uint64, C.c_uint64, C.POINTER(C.c_size_t)]),
    "grid_gpu_gadget_decompose_dev": (C.c_int, [_vp, _vp, C.c_size_t, C.c_uint64, C.c_int, _vp,
                                                _vp]),
    "grid_gpu_gadget_decompose": (C.c_int, [_vp, _vp, C.c_size_t, C.c_uint64, C.c_int, _vp]),
    "grid_gpu_prover_round_workspace": (C.c_int, [_vp, C.c_size_t, C.c_size_t,
                                                  C.POINTER(C.c_size_t)]),
    "grid_gpu_prover_round_dev": (C.c_int, [_vp, _vp, C.c_size_t, C.c_uint64, C.c_size_t,
                                            C.c_uint64, C.c_size_t, _vp, C.c_size_t, _vp, _vp,
                                            _vp, _vp, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_batch_create": (C.c_int, [_vp, _vp, C.c_size_t, _vp, C.c_size_t, C.POINTER(_vp)]),
    "grid_gpu_batch_destroy": (C.c_int, [_vp]),
    "grid_gpu_batch_set_config": (C.c_int, [_vp, _vp]),
    "grid_gpu_batch_get_config": (C.c_int, [_vp, _vp]),
    "grid_gpu_batch_shape": (C.c_int, [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "grid_gpu_batch_workspace": (C.c_int, [_vp, C.POINTER(C.c_size_t)]),
    "grid_gpu_batch_commit_dev": (C.c_int, [_vp, _vp, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_batch_commit_graph": (C.c_int, [_vp, _vp, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_batch_oneshot_workspace": (C.c_int, [_vp, _vp, C.c_size_t, _vp, C.c_size_t,
                                                   C.c_uint32, C.POINTER(C.c_size_t)]),
    "grid_gpu_batch_commit_oneshot_dev": (C.c_int, [_vp, _vp, C.c_size_t, _vp, C.c_size_t,
                                                    C.c_uint32, _vp, _vp, _vp, C.c_size_t, _vp]),
    "grid_gpu_batch_gram_workspace": (C.c_int, [_vp, _vp, C.c_size_t, C.c_uint32,
                                                C.POINTER(C.c_size_t)]),
    "grid_gpu_batch_gram_dev": (C.c_int, [_vp, _vp, _vp, C.c_size_t, C.c_uint32, _vp, _vp,
                                          C.c_size_t, _vp]),
    "grid_gpu_noalloc_scratch_bytes": (C.c_size_t, []),
    "grid_gpu_gram_noalloc_dev": (C.c_int, [_vp, _vp, C.c_size_t, C.c_size_t, _vp, _vp]),
    "grid_gpu_host_register": (C.c_int, [_vp, C.c_size_t]),
    "grid_gpu_host_unregister": (C.c_int, [_vp]),
}

_lib = None
_lock = threading.Lock()


class GridGpuError(RuntimeError):
    """A non-OK grid_status returned by the C ABI."""

    def __init__(self, code: int, where: str = ""):
        self.code = code
        self.name = STATUS_NAMES.get(code, f"status{code}")
        super().__init__(f"{where}: {self.name} ({code})" if where else f"{self.name} ({code})")


def load():
    """Load libgridgpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `python -m lattica_b200.build` "
                    "(there is no CPU fallback)")
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(code: int, where: str = "") -> None:
    if code != GRID_OK:
        raise GridGpuError(code, where)
