"""The failure path of the bounded device waits, run without a fault.

A kernel whose mbarrier wait runs out records a timeout in the plan's device
error word and finishes; the host sees GRID_ERR_TIMEOUT through
grid_gpu_plan_check, which clears the word, and the plan keeps working. The
stalled wait is made with grid_gpu_selftest_wait_timeout_dev: one warp waits on
a barrier nothing arrives at, with a small poll budget (no trap, no bad
address, no endless loop)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

Q = 4294966657


def _product(plan, oracle_plan, rng, cuda):
    import torch
    a = rng.integers(0, Q, (300, 64), dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, Q, (300, 64), dtype=np.uint64).astype(np.uint32)
    out = plan.ntt_mul_inverse(torch.from_numpy(a.view(np.int32)).to(cuda),
                               torch.from_numpy(b.view(np.int32)).to(cuda))
    got = out.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, oracle_plan.ntt_mul_inverse(a, b).reshape(300, 64))


def test_timed_out_wait_is_reported_and_plan_stays_usable(oracle, cuda):
    import torch
    from lattica_b200 import TwistedNttPlan, _lib
    from lattica_b200._lib import GridGpuError
    lib = _lib.load()
    plan = TwistedNttPlan(Q, 64)
    P = oracle.Plan(Q, 64)
    rng = np.random.default_rng(5)
    _product(plan, P, rng, cuda)
    plan.check_device()
    stream = torch.cuda.current_stream(cuda).cuda_stream
    assert lib.grid_gpu_selftest_wait_timeout_dev(plan.handle, 1000, stream) == 0
    with pytest.raises(GridGpuError) as ei:
        plan.check_device(stream)
    assert ei.value.code == 11 and ei.value.name == "Timeout"
    plan.check_device(stream)  # the word was cleared by the check
    _product(plan, P, rng, cuda)  # the same plan, bit-exact after the timeout
    plan.check_device()


def test_wait_budget_is_validated(cuda):
    from lattica_b200 import TwistedNttPlan, _lib
    lib = _lib.load()
    plan = TwistedNttPlan(Q, 64)
    assert lib.grid_gpu_selftest_wait_timeout_dev(plan.handle, 0, None) == 5
    assert lib.grid_gpu_selftest_wait_timeout_dev(plan.handle, (1 << 22) + 1, None) == 5
    assert lib.grid_gpu_selftest_wait_timeout_dev(None, 10, None) == 8
