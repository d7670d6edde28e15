"""GPU parity of the batched twisted NTT kernels against the CPU oracle
(bit-exact on every coefficient)."""
import numpy as np
import pytest

Q = 4294966657
Q256 = 4294962689
CASES = [(17, 8), (12289, 16), (12289, 32), (12289, 64), (Q, 8), (Q, 64), (12289, 128),
         (Q256, 128), (12289, 256), (Q256, 256)]

pytestmark = pytest.mark.gpu


def _rand(q, shape, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, q, shape, dtype=np.uint64).astype(np.uint32)
    # pin edge words into the first polys
    flat = a.reshape(-1)
    edges = np.array([0, 1, q - 1, q - 2, q // 2, (q + 1) // 2], dtype=np.uint64).astype(np.uint32)
    flat[: min(len(edges), flat.size)] = edges[: min(len(edges), flat.size)]
    return a


def _dev(a, cuda):
    import torch
    return torch.from_numpy(a.view(np.int32).copy()).to(cuda)


def _host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("q,d", CASES)
@pytest.mark.parametrize("npolys", [1, 33, 257])
def test_forward_inverse_mulinv_match_oracle(cuda, oracle, q, d, npolys):
    from lattica_b200 import TwistedNttPlan
    plan = TwistedNttPlan(q, d)
    P = oracle.Plan(q, d)
    a = _rand(q, (npolys, d), 1000 * d + npolys)
    b = _rand(q, (npolys, d), 7 + d + npolys)
    fwd = P.forward(a).reshape(npolys, d)
    inv = P.inverse(b).reshape(npolys, d)
    mul = P.ntt_mul_inverse(a, b).reshape(npolys, d)

    # device path
    ta = _dev(a, cuda)
    plan.forward_in_place(ta)
    assert np.array_equal(_host(ta), fwd)
    tb = _dev(b, cuda)
    plan.inverse_in_place(tb)
    assert np.array_equal(_host(tb), inv)
    tout = plan.ntt_mul_inverse(_dev(a, cuda), _dev(b, cuda))
    assert np.array_equal(_host(tout), mul)

    # host-buffer path
    ha = a.copy()
    plan.forward_in_place(ha)
    assert np.array_equal(ha, fwd)
    hb = b.copy()
    plan.inverse_in_place(hb)
    assert np.array_equal(hb, inv)
    assert np.array_equal(plan.ntt_mul_inverse(a, b), mul)


@pytest.mark.parametrize("q,d", [(17, 8), (12289, 64), (Q, 64), (Q256, 256)])
def test_poly_mul_matches_naive(cuda, oracle, q, d):
    from lattica_b200 import TwistedNttPlan
    plan = TwistedNttPlan(q, d)
    P = oracle.Plan(q, d)
    n = 40
    a = _rand(q, (n, d), 11)
    b = _rand(q, (n, d), 12)
    expect = np.stack([P.naive_negacyclic(a[i], b[i]) for i in range(n)])
    h = a.copy()
    plan.multiply_in_place(h, b)
    assert np.array_equal(h, expect)
    t = _dev(a, cuda)
    plan.multiply_in_place(t, _dev(b, cuda))
    assert np.array_equal(_host(t), expect)


def test_poly_mul_small_kat(cuda, oracle, kats):
    from lattica_b200 import poly_mul_ntt
    k = kats["poly_mul_small_f17"]
    P = oracle.Plan(k["q"], 8)
    a = P.field.to_mont(k["a"]).reshape(1, 8)
    b = P.field.to_mont(k["b"]).reshape(1, 8)
    got = poly_mul_ntt(a, b, k["q"])
    assert np.array_equal(got[0], P.naive_negacyclic(a[0], b[0])), k["source"]


def test_reference_error_variants(cuda, kats):
    from lattica_b200 import NttError, TwistedNttPlan, poly_mul_ntt
    for c in kats["ntt_errors"]:
        if c["kind"] == "LengthMismatch":
            a = np.ones((1, c["lengths"][0]), np.uint32)
            b = np.ones((1, c["lengths"][1]), np.uint32)
            with pytest.raises(NttError) as ei:
                poly_mul_ntt(a, b, c["q"])
            assert ei.value == NttError("LengthMismatch", **c["fields"]), c["source"]
        else:
            with pytest.raises(NttError) as ei:
                TwistedNttPlan(c["q"], c["fields"]["len"])
            assert ei.value == NttError(c["kind"], **c["fields"]), c["source"]


def test_empty_and_misaligned(cuda):
    import ctypes as C
    import torch
    from lattica_b200 import TwistedNttPlan, _lib
    plan = TwistedNttPlan(Q, 64)
    lib = _lib.load()
    t = torch.zeros(4 * 64 + 1, dtype=torch.int32, device=cuda)
    assert lib.grid_gpu_ntt_forward_dev(plan.handle, t.data_ptr(), 0, None) == 0
    assert lib.grid_gpu_ntt_forward_dev(plan.handle, t.data_ptr() + 4, 4, None) == 13
    plan.forward_in_place(t[: 4 * 64].view(4, 64))
    torch.cuda.synchronize()
    plan.check_device()


def test_config_scale_round_trip_and_sampled_parity(cuda, oracle):
    """2^22 polys of d = 64: bit-exact on a sample against the oracle, and the
    full batch is checked through the inverse(forward(a)) == a identity."""
    import torch
    from lattica_b200 import TwistedNttPlan
    n, d = 1 << 22, 64
    plan = TwistedNttPlan(Q, d)
    g = torch.Generator(device=cuda).manual_seed(123)
    a = torch.randint(0, Q, (n, d), dtype=torch.int64, device=cuda, generator=g)
    b = torch.randint(0, Q, (n, d), dtype=torch.int64, device=cuda, generator=g)
    a32 = a.to(torch.int32)   # wraps to the same 32-bit words
    b32 = b.to(torch.int32)
    del a, b
    out = plan.ntt_mul_inverse(a32, b32)
    x = a32.clone()
    plan.forward_in_place(x)
    plan.inverse_in_place(x)
    assert torch.equal(x, a32)
    idx = torch.tensor([0, 1, 31, 32, 4095, n // 2 + 17, n - 33, n - 1], device=cuda)
    P = oracle.Plan(Q, d)
    sa, sb, so = _host(a32[idx]), _host(b32[idx]), _host(out[idx])
    assert np.array_equal(P.ntt_mul_inverse(sa, sb).reshape(-1, d), so)
    plan.check_device()


def test_d256_sweep_scale_sampled(cuda, oracle):
    import torch
    from lattica_b200 import TwistedNttPlan
    n, d = 1 << 20, 256
    plan = TwistedNttPlan(Q256, d)
    g = torch.Generator(device=cuda).manual_seed(7)
    a32 = torch.randint(0, Q256, (n, d), dtype=torch.int64, device=cuda, generator=g).to(torch.int32)
    b32 = torch.randint(0, Q256, (n, d), dtype=torch.int64, device=cuda, generator=g).to(torch.int32)
    out = plan.ntt_mul_inverse(a32, b32)
    idx = torch.tensor([0, 7, 8, 9, n // 3, n - 1], device=cuda)
    P = oracle.Plan(Q256, d)
    assert np.array_equal(P.ntt_mul_inverse(_host(a32[idx]), _host(b32[idx])).reshape(-1, d),
                          _host(out[idx]))
    plan.check_device()
