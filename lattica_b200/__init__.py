"""B200-native (sm_100a) ring-arithmetic hot path for Gridland (mrain/lattica).

Host-side mirror of the reference's operator surface for R_q = Z_q[X]/(X^d+1):
twisted NTT plans, Ajtai/linear commitments, the LaBRADOR prover's Gram
matrix, JL projection and balanced/gadget decompositions. Every call runs the
CUDA kernels in libgridgpu.so through the C ABI of include/grid_gpu.h.
"""
from ._lib import GridGpuError, load as load_library
from .ntt import CommitmentError, NttError, TwistedNttPlan, poly_mul_ntt, twisted_ntt_plan

__all__ = [
    "GridGpuError", "load_library", "NttError", "CommitmentError", "TwistedNttPlan",
    "twisted_ntt_plan", "poly_mul_ntt",
]
