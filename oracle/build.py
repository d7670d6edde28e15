"""Build recipe for the CPU oracle (test infrastructure).

Compiles oracle/oracle.c (baseline x86-64) and oracle/oracle_avx2.c (-mavx2
-mfma) separately and links them into oracle/_build/liboracle.so with gcc. The
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


# Only the AVX2 restatement is built for AVX2; the scalar oracle keeps the
# baseline x86-64 instruction set so that the checker runs on any host.
ISA_FLAGS = {"oracle.c": [], "oracle_avx2.c": ["-mavx2", "-mfma"]}


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    newest_src = max(os.path.getmtime(s) for s in SOURCES + [os.path.join(HERE, "oracle.h")])
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest_src:
        return LIB
    objs = []
    for src in SOURCES:
        obj = os.path.join(OUT_DIR, os.path.basename(src) + ".o")
        subprocess.check_call([
            "gcc", "-O3", *ISA_FLAGS[os.path.basename(src)], "-fopenmp", "-fPIC",
            "-Wall", "-Wno-unused-function", "-c", src, "-o", obj,
        ])
        objs.append(obj)
    subprocess.check_call(["gcc", "-shared", "-fopenmp", "-o", LIB, *objs])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
