"""Extract the known-answer tests the reference keeps for the hot path.

Reads the reference's Rust test modules as TEXT (the Rust toolchain is not
available, so the reference cannot be executed) and writes the literal
known-answer values to tests/golden/reference_kats.json, each with its source
file:line. The reference checkout's root directory is a required argument:

    python tests/golden/extract_reference_kats.py <path to the reference checkout>
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "reference_kats.json")


def _read(root, rel):
    with open(os.path.join(root, rel), encoding="utf-8") as fh:
        return fh.read().splitlines()


def _fn_body(lines, name):
    """Return (start_line_1based, body_lines) of `fn name(` up to its closing brace."""
    for i, line in enumerate(lines):
        if re.search(rf"\bfn {re.escape(name)}\s*\(", line):
            depth, body = 0, []
            for j in range(i, len(lines)):
                body.append(lines[j])
                depth += lines[j].count("{") - lines[j].count("}")
                if depth == 0 and "{" in "".join(body):
                    return i + 1, body
    raise KeyError(name)


def decompose_balanced_cases(root):
    rel = "labrador/src/main_protocol/mod.rs"
    start, body = _fn_body(_read(root, rel), "test_decompose_coeff_balanced")
    pat = re.compile(r"\((\d+),\s*(\d+),\s*(\d+),\s*(\d+),\s*vec!\[([^\]]*)\]\)")
    cases = []
    for off, line in enumerate(body):
        m = pat.search(line)
        if m:
            limbs = [int(x) for x in m.group(5).split(",") if x.strip()]
            cases.append({"value": int(m.group(1)), "base": int(m.group(2)),
                          "num_limbs": int(m.group(3)), "q": int(m.group(4)),
                          "limbs": limbs, "source": f"{rel}:{start + off}"})
    return cases


def centered_mod_cases(root):
    rel = "labrador/src/main_protocol/mod.rs"
    start, body = _fn_body(_read(root, rel), "test_centered_mod")
    pat = re.compile(r"centered_mod\((-?\d+),\s*(\d+)\),\s*(-?\d+)\)")
    return [{"v": int(m.group(1)), "base": int(m.group(2)), "expected": int(m.group(3)),
             "source": f"{rel}:{start + off}"}
            for off, line in enumerate(body) for m in [pat.search(line)] if m]


def garbage_index_cases(root):
    rel = "labrador/src/main_protocol/mod.rs"
    start, body = _fn_body(_read(root, rel), "test_garbage_index")
    pat = re.compile(r"^\s*\((\d+),\s*(\d+),\s*(\d+),\s*(\d+)\),")
    idx = [{"r": int(m.group(1)), "i": int(m.group(2)), "j": int(m.group(3)),
            "expected": int(m.group(4)), "source": f"{rel}:{start + off}"}
           for off, line in enumerate(body) for m in [pat.search(line)] if m]
    start2, body2 = _fn_body(_read(root, rel), "test_garbage_count")
    pat2 = re.compile(r"garbage_count\((\d+)\),\s*(\d+)\)")
    cnt = [{"r": int(m.group(1)), "expected": int(m.group(2)), "source": f"{rel}:{start2 + off}"}
           for off, line in enumerate(body2) for m in [pat2.search(line)] if m]
    return idx, cnt


def linear_commit_f17(root):
    rel = "commit/src/linear.rs"
    start, body = _fn_body(_read(root, rel), "test_recompute_linear_commitment")
    text = "\n".join(body)
    vals = [int(x) for x in re.findall(r"F17::from_u64\((\d+)\)", text)]
    exp = [int(x) for x in re.findall(r"\.to_u64\(\),\s*(\d+)\)", text)]
    shapes = [tuple(int(v) for v in m) for m in re.findall(r"RingMat::new\(\s*(\d+),\s*(\d+),", text)]
    (mr, mc), (orows, oc) = shapes[0], shapes[1]
    a_msg = vals[: mr * mc]
    a_open = vals[mr * mc: mr * mc + orows * oc]
    rest = vals[mr * mc + orows * oc:]
    return {"q": 17, "rows": mr, "msg_cols": mc, "open_cols": oc, "a_msg": a_msg,
            "a_open": a_open, "message": rest[:mc], "randomness": rest[mc:mc + oc],
            "expected": exp, "source": f"{rel}:{start}"}


def ntt_facts(root):
    rel = "algebra/src/arith/prime.rs"
    lines = _read(root, rel)
    out = []
    for name in ("test_ntt_ring", "test_ntt_ring_12289"):
        start, body = _fn_body(lines, name)
        for off, line in enumerate(body):
            m = re.search(r"assert_eq!\(F(\d+)::max_ntt_size\(\),\s*(\d+)\)", line)
            if m:
                out.append({"kind": "max_ntt_size", "q": int(m.group(1)),
                            "value": int(m.group(2)), "source": f"{rel}:{start + off}"})
            m = re.search(r"assert!\((!?)F(\d+)::supports_ntt\((\d+)\)\)", line)
            if m:
                out.append({"kind": "supports_ntt", "q": int(m.group(2)), "n": int(m.group(3)),
                            "value": m.group(1) != "!", "source": f"{rel}:{start + off}"})
    return out


def poly_mul_small(root):
    rel = "algebra/src/poly/ntt.rs"
    start, body = _fn_body(_read(root, rel), "test_poly_mul_ntt_matches_naive_small")
    vals = [int(x) for x in re.findall(r"F17::from_u64\((\d+)\)", "\n".join(body))]
    return {"q": 17, "a": vals[:8], "b": vals[8:16], "source": f"{rel}:{start}",
            "property": "poly_mul_ntt(a, b) == naive_negacyclic(a, b)"}


def ntt_error_cases(root):
    rel = "algebra/src/poly/ntt.rs"
    lines = _read(root, rel)
    cases = []
    for name, kind in (("test_poly_mul_ntt_rejects_length_mismatch", "LengthMismatch"),
                       ("test_ntt_forward_rejects_non_power_of_two_length", "LengthNotPowerOfTwo"),
                       ("test_ntt_forward_rejects_unsupported_size", "UnsupportedSize"),
                       ("test_poly_mul_ntt_rejects_unsupported_twist", "UnsupportedTwist")):
        start, body = _fn_body(lines, name)
        text = "\n".join(body)
        lens = [int(x) for x in re.findall(r"vec!\[F17::from_u64\(1\);\s*(\d+)\]", text)]
        fields = dict((k, int(v)) for k, v in re.findall(r"(left|right|len):\s*(\d+)", text))
        cases.append({"kind": kind, "q": 17, "lengths": lens, "fields": fields,
                      "source": f"{rel}:{start}"})
    return cases


def add_sub_f17(root):
    rel = "algebra/src/arith/prime.rs"
    start, body = _fn_body(_read(root, rel), "test_add_sub")
    text = "\n".join(body)
    a, b = [int(x) for x in re.findall(r"F17::from_u64\((\d+)\)", text)][:2]
    exp = [int(x) for x in re.findall(r"\.to_u64\(\),\s*(\d+)\)", text)]
    return {"q": 17, "a": a, "b": b, "a_plus_b": exp[0], "a_minus_b": exp[1],
            "b_minus_a": exp[2], "source": f"{rel}:{start}"}


def round_trip_3329(root):
    rel = "algebra/src/arith/prime.rs"
    start, body = _fn_body(_read(root, rel), "test_ntt_round_trip_3329")
    vals = [int(x) for x in re.findall(r"F3329::from_u64\((\d+)\)", "\n".join(body))]
    return {"q": 3329, "input": vals, "source": f"{rel}:{start}"}


def main(root):
    idx, cnt = garbage_index_cases(root)
    data = {
        "generated_by": "tests/golden/extract_reference_kats.py",
        "decompose_coeff_balanced": decompose_balanced_cases(root),
        "centered_mod": centered_mod_cases(root),
        "garbage_index": idx,
        "garbage_count": cnt,
        "linear_commit_f17": linear_commit_f17(root),
        "ntt_facts": ntt_facts(root),
        "poly_mul_small_f17": poly_mul_small(root),
        "ntt_errors": ntt_error_cases(root),
        "add_sub_f17": add_sub_f17(root),
        "ntt_round_trip_3329": round_trip_3329(root),
    }
    with open(OUT, "w", encoding="utf-8") as fh:
        json.dump(data, fh, indent=1)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: extract_reference_kats.py <path to the reference checkout>")
    main(sys.argv[1])
