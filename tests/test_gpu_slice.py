"""GPU parity of the Ring slice hooks for PrimeField (algebra/src/arith/prime.rs:433-491):
pointwise_mul_assign_slice, add_assign_slice, sub_assign_slice, scalar_mul_slice,
add_assign_scaled_slice and dot_product, word for word against the oracle,
including unaligned starts (the kernels' scalar path) and edge words."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

Q = 4294966657
LABRADOR_Q = 4294967291


def _dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).to(cuda)


def _host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("q,d", [(Q, 64), (12289, 64), (17, 8)])
@pytest.mark.parametrize("n,off", [(1, 0), (4099, 0), (4099, 1), (1 << 20, 3)])
def test_slice_hooks_match_oracle(oracle, cuda, q, d, n, off):
    from lattica_b200 import TwistedNttPlan
    plan = TwistedNttPlan(q, d)
    F = oracle.Field(q)
    rng = np.random.default_rng(n + off)
    a = rng.integers(0, q, n + off, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, q, n + off, dtype=np.uint64).astype(np.uint32)
    a[off:off + 3] = [q - 1, 0, 1][: min(3, n)]
    b[off:off + 3] = [q - 1, q - 1, q - 1][: min(3, n)]
    sc = int(rng.integers(1, q))
    ha, hb = a[off:], b[off:]
    for op, want in (
        ("pointwise_mul_assign_slice", F.pointwise_mul_slice(ha, hb)),
        ("add_assign_slice", F.add_slice(ha, hb)),
        ("sub_assign_slice", F.sub_slice(ha, hb)),
    ):
        ta, tb = _dev(a, cuda), _dev(b, cuda)
        getattr(plan, op)(ta[off:], tb[off:])
        assert np.array_equal(_host(ta)[off:], want), op
        assert np.array_equal(_host(ta)[:off], a[:off])
    ta = _dev(a, cuda)
    plan.scalar_mul_slice(ta[off:], sc)
    assert np.array_equal(_host(ta)[off:], F.scalar_mul_slice(ha, sc))
    ta, tb = _dev(a, cuda), _dev(b, cuda)
    plan.add_assign_scaled_slice(ta[off:], tb[off:], sc)
    assert np.array_equal(_host(ta)[off:], F.add_scaled_slice(ha, hb, sc))
    ta, tb = _dev(a, cuda), _dev(b, cuda)
    assert plan.dot_product(ta[off:], tb[off:]) == F.dot_product(ha, hb)
    plan.check_device()


def test_slice_hooks_reject_bad_arguments(cuda):
    import torch
    from lattica_b200 import TwistedNttPlan, _lib
    from lattica_b200.ntt import NttError
    plan = TwistedNttPlan(Q, 64)
    lib = _lib.load()
    x = torch.zeros(64, dtype=torch.int32, device=cuda)
    assert lib.grid_gpu_scalar_mul_dev(plan.handle, x.data_ptr(), Q, 64, None) == 5
    assert lib.grid_gpu_add_assign_scaled_dev(plan.handle, x.data_ptr(), x.data_ptr(), Q + 1,
                                              64, None) == 5
    assert lib.grid_gpu_add_assign_dev(plan.handle, None, x.data_ptr(), 64, None) == 8
    assert lib.grid_gpu_dot_product_dev(plan.handle, x.data_ptr(), x.data_ptr(), 64, None,
                                        None) == 8
    with pytest.raises(NttError):
        plan.add_assign_slice(x, x[:32])
