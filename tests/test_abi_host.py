"""C-ABI library checks that need no GPU: it loads, exports every symbol the
headers declare, and its host-side plan logic (validation order, roots and the
merged twiddle tables) matches the oracle."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT

Q = 4294966657
Q256 = 4294962689


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h, encoding="utf-8").read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(grid_gpu_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    from lattica_b200 import _lib
    lib = _lib.load()
    declared = _declared_symbols()
    assert len(declared) >= 15
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert declared <= set(_lib.SIGNATURES), sorted(declared - set(_lib.SIGNATURES))
    assert lib.grid_gpu_abi_version() >> 16 == 1
    assert lib.grid_gpu_max_degree() == 256
    for code in range(16):
        assert lib.grid_gpu_status_string(code) not in (None, b"unknown status")


def _describe(q, d):
    from lattica_b200 import _lib
    lib = _lib.load()
    info = _lib.PlanInfo()
    z = np.zeros(max(d, 1), np.uint32)
    iz = np.zeros(max(d, 1), np.uint32)
    st = lib.grid_gpu_plan_describe(q, d, C.byref(info), z.ctypes.data, iz.ctypes.data)
    return st, info, z, iz


def test_plan_validation_matches_reference_errors(kats):
    codes = {"LengthNotPowerOfTwo": 2, "UnsupportedSize": 3, "UnsupportedTwist": 4}
    for c in kats["ntt_errors"]:
        if c["kind"] in codes:
            assert _describe(c["q"], c["fields"]["len"])[0] == codes[c["kind"]], c["source"]
    assert _describe(16, 8)[0] == 7          # not prime
    assert _describe(1 << 32 | 1, 8)[0] == 7  # too wide for u32 words
    assert _describe(Q, 256)[0] == 3         # q = 1 mod 128 only
    assert _describe(4294967291, 64)[0] == 3 # the LaBRADOR profile prime has no 64th root
    assert _describe(12289, 512)[0] == 12    # valid, but no kernel for d = 512
    assert _describe(Q, 64)[0] == 0 and _describe(Q256, 256)[0] == 0


def _brv(x, bits):
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


@pytest.mark.parametrize("q,d", [(17, 8), (12289, 16), (12289, 64), (Q, 64), (Q, 8),
                                 (12289, 128), (Q256, 256)])
def test_merged_twiddles_reproduce_reference_transform(oracle, q, d):
    """Model the GPU's merged CT/GS schedule on the host with the library's
    own twiddle tables and compare with the oracle's twist + NTT chain."""
    st, info, z, iz = _describe(q, d)
    assert st == 0
    P = oracle.Plan(q, d)
    F = P.field
    t = P.tables()
    assert (info.generator, info.psi, info.omega, info.n_inv) == (
        t["generator"], t["psi"], t["omega"], t["inv_scale"])
    bits = d.bit_length() - 1
    rng = np.random.default_rng(d)
    a = rng.integers(0, q, d, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, q, d, dtype=np.uint64).astype(np.uint32)
    x = [int(v) for v in a]
    L = d // 2
    while L >= 1:
        for g in range(d // (2 * L)):
            k = d // (2 * L) + g
            for j in range(g * 2 * L, g * 2 * L + L):
                tt = F.mul(x[j + L], int(z[k]))
                x[j + L] = F.sub(x[j], tt)
                x[j] = F.add(x[j], tt)
        L //= 2
    ref = P.forward(a)
    assert all(x[j] == int(ref[_brv(j, bits)]) for j in range(d))
    y = [F.mul(x[j], int(b[_brv(j, bits)])) for j in range(d)]
    L = 1
    while L < d:
        for g in range(d // (2 * L)):
            k = d // (2 * L) + g
            for j in range(g * 2 * L, g * 2 * L + L):
                u, v = y[j], y[j + L]
                y[j], y[j + L] = F.add(u, v), F.mul(F.sub(u, v), int(iz[k]))
        L *= 2
    y = [F.mul(v, info.n_inv) for v in y]
    assert np.array_equal(np.array(y, np.uint32), P.ntt_mul_inverse(a, b))


def test_plan_create_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from lattica_b200 import GridGpuError, TwistedNttPlan
    with pytest.raises(GridGpuError) as ei:
        TwistedNttPlan(Q, 64)
    assert ei.value.name == "NoDevice"


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """Without the built library every entry point refuses: there is no CPU fallback."""
    import pytest
    from lattica_b200 import _lib as L
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", str(tmp_path / "libgridgpu.so"))
    with pytest.raises(ImportError, match="no CPU fallback"):
        L.load()
