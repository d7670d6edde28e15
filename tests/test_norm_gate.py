"""The JL norm gate on the host, as labrador/src/main_protocol/mod.rs:194-247
(centered squared L2 norm: a value above q/2 counts as q - v, summed exactly)
and labrador/src/jl.rs:533-547 (||p||^2 <= (verify_factor * beta)^2; false for a
non-finite or non-positive beta and for a length other than the profile's rows)."""
import math

import numpy as np

from lattica_b200.labrador import squared_l2_norm_u128, verify_norm

Q = 4294966657


def _mont(values):
    return np.array([(int(v) % Q) * (1 << 32) % Q for v in values], dtype=np.uint64).astype(np.uint32)


def test_centered_squared_norm_is_exact():
    h = Q // 2
    vals = [0, 1, Q - 1, h, h + 1, 5, Q - 5, 2 ** 31]
    want = 0 + 1 + 1 + h * h + (Q - h - 1) ** 2 + 25 + 25 + (Q - 2 ** 31) ** 2
    assert squared_l2_norm_u128(_mont(vals), Q) == want
    # exact beyond f64: the sum of 256 squares near (q/2)^2 keeps every bit
    big = _mont([h] * 256)
    assert squared_l2_norm_u128(big, Q) == 256 * h * h


def test_verify_norm_threshold_and_invalid_inputs():
    p = _mont([1] * 256)                     # ||p||^2 = 256
    beta = math.sqrt(2.0)                    # (sqrt(128) * beta)^2 = 256
    assert verify_norm(p, Q, beta)
    assert not verify_norm(p, Q, beta * (1 - 1e-9))
    assert verify_norm(_mont([Q - 1] * 256), Q, beta)   # -1 counts as 1
    for bad in (0.0, -1.0, math.inf, math.nan):
        assert not verify_norm(p, Q, bad)
    assert not verify_norm(p[:255], Q, 10.0)            # length must equal the rows
    assert verify_norm(p[:100], Q, 10.0, rows=100)
