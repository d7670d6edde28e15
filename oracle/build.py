"""Build recipe for the CPU oracle (test infrastructure).

Compiles oracle/oracle.c and oracle/oracle_avx2.c into oracle/_build/liboracle.so
with gcc. The
reference itself is Rust and cannot be compiled here (no cargo/rustc), so
there is no oracle/_ref build; the oracle is the C restatement only.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
SOURCES = [os.path.join(HERE, "oracle.c"), os.path.join(HERE, "oracle_avx2.c")]


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    newest_src = max(os.path.getmtime(s) for s in SOURCES + [os.path.join(HERE, "oracle.h")])
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest_src:
        return LIB
    cmd = [
        "gcc", "-O3", "-mavx2", "-mfma", "-fopenmp", "-fPIC", "-shared",
        "-Wall", "-Wno-unused-function", "-o", LIB, *SOURCES,
    ]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
