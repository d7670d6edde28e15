"""The tensor-core transforms (byte-plane u8 MMAs with exact int32
accumulation) against the oracle and against the CUDA-core kernels: d = 64
transforms at tile edges (128 polys per tile) and d = 256 products (4-point
steps on CUDA cores around 64-point tensor-core transforms, 32 polys per
tile), both across the persistent grid's wrap."""
import os

import numpy as np
import pytest

Q = 4294966657

pytestmark = pytest.mark.gpu


Q256 = 4294962689  # q' = 1 mod 512 for the d = 256 sweep


def _plan(q, engine, d=64):
    """Plan whose transforms use the tensor cores ("tc") where a tensor-core
    kernel exists or the CUDA-core kernels ("cuda_core"); the choice is made at
    plan creation."""
    from lattica_b200 import TwistedNttPlan
    old = os.environ.get("GRID_GPU_NTT_ENGINE")
    if engine == "cuda_core":
        os.environ["GRID_GPU_NTT_ENGINE"] = "cuda_core"
    else:
        os.environ.pop("GRID_GPU_NTT_ENGINE", None)
    try:
        return TwistedNttPlan(q, d)
    finally:
        if old is None:
            os.environ.pop("GRID_GPU_NTT_ENGINE", None)
        else:
            os.environ["GRID_GPU_NTT_ENGINE"] = old


def _words(q, n, seed, d=64):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, q, (n, d), dtype=np.uint64).astype(np.uint32)
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


@pytest.mark.parametrize("q", [Q256, 12289])
@pytest.mark.parametrize("npolys", [1, 31, 32, 33, 148 * 32 + 5, 3 * 148 * 32 + 17])
def test_d256_tensor_core_products_match_oracle_and_cuda_cores(cuda, oracle, q, npolys):
    import torch
    tcp, ccp = _plan(q, "tc", 256), _plan(q, "cuda_core", 256)
    P = oracle.Plan(q, 256)
    a, b = _words(q, npolys, npolys, 256), _words(q, npolys, npolys + 1, 256)
    ta = torch.from_numpy(a.view(np.int32)).to(cuda)
    tb = torch.from_numpy(b.view(np.int32)).to(cuda)
    got = tcp.ntt_mul_inverse(ta, tb)
    ref = ccp.ntt_mul_inverse(ta, tb)
    torch.cuda.synchronize()
    got, ref = got.cpu().numpy().view(np.uint32), ref.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, ref)
    idx = np.unique(np.r_[0, npolys - 1, np.linspace(0, npolys - 1, 12).astype(int)])
    assert np.array_equal(got[idx], P.ntt_mul_inverse(a[idx], b[idx]).reshape(-1, 256))
    tcp.check_device()
    ccp.check_device()


def test_d256_tensor_core_identity_at_scale(cuda):
    """2^20 polys: the Montgomery product with the evaluations of 1 (R mod q'
    in every slot) returns a unchanged."""
    import torch
    plan = _plan(Q256, "tc", 256)
    n = 1 << 20
    g = torch.Generator(device=cuda).manual_seed(4)
    a = torch.randint(0, Q256, (n, 256), dtype=torch.int64, device=cuda, generator=g).to(torch.int32)
    one = torch.full((n, 256), (1 << 32) % Q256, dtype=torch.int64, device=cuda).to(torch.int32)
    y = plan.ntt_mul_inverse(a, one)
    assert torch.equal(y, a)
    plan.check_device()
