"""The d = 64 tensor-core transforms (byte-plane u8 MMAs with exact int32
accumulation) against the oracle and against the CUDA-core kernels, at tile
edges (128 polys per tile) and across the persistent grid's wrap."""
import os

import numpy as np
import pytest

Q = 4294966657

pytestmark = pytest.mark.gpu


def _plan(q, engine):
    """Plan whose d = 64 transforms use the tensor cores ("tc") or the
    CUDA-core kernels ("cuda_core"); the choice is made at plan creation."""
    from lattica_b200 import TwistedNttPlan
    old = os.environ.get("GRID_GPU_NTT_ENGINE")
    if engine == "cuda_core":
        os.environ["GRID_GPU_NTT_ENGINE"] = "cuda_core"
    else:
        os.environ.pop("GRID_GPU_NTT_ENGINE", None)
    try:
        return TwistedNttPlan(q, 64)
    finally:
        if old is None:
            os.environ.pop("GRID_GPU_NTT_ENGINE", None)
        else:
            os.environ["GRID_GPU_NTT_ENGINE"] = old


def _words(q, n, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, q, (n, 64), dtype=np.uint64).astype(np.uint32)
    edges = np.array([0, 1, q - 1, q - 2, q // 2], dtype=np.uint64).astype(np.uint32)
    a.reshape(-1)[: edges.size] = edges
    if n > 2:
        a[1, :] = q - 1      # all-maximal row: largest tensor-core partial sums
        a[2, :] = 0
    return a


@pytest.mark.parametrize("q", [Q, 12289, 4294962689])
@pytest.mark.parametrize("npolys", [1, 127, 128, 129, 148 * 128 + 77, 2 * 148 * 128 + 1])
def test_tensor_core_transforms_match_oracle_and_cuda_cores(cuda, oracle, q, npolys):
    import torch
    tcp, ccp = _plan(q, "tc"), _plan(q, "cuda_core")
    P = oracle.Plan(q, 64)
    a, b = _words(q, npolys, npolys), _words(q, npolys, npolys + 1)
    ta = torch.from_numpy(a.view(np.int32)).to(cuda)
    tb = torch.from_numpy(b.view(np.int32)).to(cuda)
    outs = {}
    for name, plan in (("tc", tcp), ("cc", ccp)):
        f = ta.clone()
        plan.forward_in_place(f)
        i = tb.clone()
        plan.inverse_in_place(i)
        m = plan.ntt_mul_inverse(ta, tb)
        torch.cuda.synchronize()
        outs[name] = [x.cpu().numpy().view(np.uint32) for x in (f, i, m)]
    for x, y in zip(outs["tc"], outs["cc"]):
        assert np.array_equal(x, y)
    idx = np.unique(np.r_[0, npolys - 1, np.linspace(0, npolys - 1, 40).astype(int)])
    assert np.array_equal(outs["tc"][0][idx], P.forward(a[idx]).reshape(-1, 64))
    assert np.array_equal(outs["tc"][1][idx], P.inverse(b[idx]).reshape(-1, 64))
    assert np.array_equal(outs["tc"][2][idx], P.ntt_mul_inverse(a[idx], b[idx]).reshape(-1, 64))
    tcp.check_device()
    ccp.check_device()


def test_tensor_core_round_trip_at_scale(cuda):
    """2^20 polys: INTT(NTT(a)) == a, and multiplying by the evaluations of
    the constant 1 is the identity."""
    import torch
    plan = _plan(Q, "tc")
    n = 1 << 20
    g = torch.Generator(device=cuda).manual_seed(3)
    a = torch.randint(0, Q, (n, 64), dtype=torch.int64, device=cuda, generator=g).to(torch.int32)
    x = a.clone()
    plan.forward_in_place(x)
    plan.inverse_in_place(x)
    assert torch.equal(x, a)
    # the Montgomery product with R mod q (the Montgomery word of 1) is the identity
    one = torch.full((n, 64), (1 << 32) % Q, dtype=torch.int64, device=cuda).to(torch.int32)
    y = plan.ntt_mul_inverse(a, one)
    assert torch.equal(y, a)
    plan.check_device()
