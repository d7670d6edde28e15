"""The Gram entry point that allocates nothing (grid_gpu_gram_noalloc_dev).

It serves callers that cannot allocate device memory — a latency-bound prover
loop where cudaMalloc would synchronise the device, or a plugin whose host
owns the memory pool — by taking its scratch from a fixed buffer compiled into
the library. This file is collected last so a stop-at-first-failure run has
already run every other test; it also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

Q = 4294966657


def _gram_with_workspace(lib, plan, S, r, n, torch, dev):
    nb = C.c_size_t()
    assert lib.grid_gpu_gram_workspace(plan.handle, r, n, C.byref(nb)) == 0
    ws = torch.empty(max(16, nb.value), dtype=torch.uint8, device=dev)
    G = torch.empty((r * (r + 1) // 2, 64), dtype=torch.int32, device=dev)
    st = lib.grid_gpu_gram_dev(plan.handle, S.data_ptr(), r, n, G.data_ptr(), ws.data_ptr(),
                               ws.numel(), torch.cuda.current_stream(dev).cuda_stream)
    assert st == 0
    return G


def test_noalloc_gram_matches_allocating_entry_point_on_two_calls(cuda):
    import torch
    from lattica_b200 import TwistedNttPlan, _lib
    lib = _lib.load()
    plan = TwistedNttPlan(Q, 64)
    assert lib.grid_gpu_noalloc_scratch_bytes() == 48 << 20
    stream = torch.cuda.current_stream(cuda).cuda_stream
    g = torch.Generator(device=cuda).manual_seed(99)
    # two calls in a row, different shapes (the second one splits K)
    for r, n in ((5, 130), (64, 2048)):
        S = torch.randint(0, Q, (r, n, 64), dtype=torch.int64, device=cuda,
                          generator=g).to(torch.int32)
        want = _gram_with_workspace(lib, plan, S, r, n, torch, cuda)
        got = torch.empty_like(want)
        st = lib.grid_gpu_gram_noalloc_dev(plan.handle, S.data_ptr(), r, n, got.data_ptr(), stream)
        assert st == 0
        torch.cuda.synchronize()
        assert torch.equal(got, want), (r, n)
    plan.check_device()


def test_noalloc_gram_rejects_problems_beyond_its_buffer(cuda):
    import torch
    from lattica_b200 import TwistedNttPlan, _lib
    lib = _lib.load()
    plan = TwistedNttPlan(Q, 64)
    r, n = 64, 8192  # 128 MiB of evaluations alone
    nb = C.c_size_t()
    assert lib.grid_gpu_gram_workspace(plan.handle, r, n, C.byref(nb)) == 0
    assert nb.value > lib.grid_gpu_noalloc_scratch_bytes()
    S = torch.zeros((1,), dtype=torch.int32, device=cuda)  # never read: rejected up front
    G = torch.zeros((1,), dtype=torch.int32, device=cuda)
    st = lib.grid_gpu_gram_noalloc_dev(plan.handle, S.data_ptr(), r, n, G.data_ptr(), None)
    assert st == 15  # GRID_ERR_SCRATCH_LIMIT
    assert b"scratch" in lib.grid_gpu_status_string(st)
