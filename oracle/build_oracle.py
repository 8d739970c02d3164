"""Build recipe for the CPU oracle (test infrastructure, never the product).

Compiles ``oracle/tchll_oracle.c`` with gcc into
``oracle/build/libtchll_oracle.so``.  The reference (pure Python) has no
compiled part, so there is no ``oracle/_ref`` build: the reference's own Python
is imported only in this container, by ``tests/golden/make_golden.py``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "tchll_oracle.c")
OUT_DIR = os.path.join(HERE, "build")
LIB = os.path.join(OUT_DIR, "libtchll_oracle.so")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= os.path.getmtime(SRC)):
        return LIB
    cmd = ["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared",
           "-fvisibility=hidden", "-std=c11", "-Wall", "-Wno-unknown-pragmas",
           SRC, "-o", LIB + ".tmp", "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
