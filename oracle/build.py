"""Build recipe of the CPU oracle (test infrastructure): ``liboracle.so`` from ``pocean_oracle.c``.

The restatement is compiled with FMA contraction off and without fast-math so that its FP64 arithmetic is the
IEEE evaluation of the reference's expressions in their written order (what Numba does for the reference).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "pocean_oracle.c")
LIB = os.path.join(HERE, "liboracle.so")
CFLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared", "-std=c11",
          "-Wall", "-Wextra"]


def build(force: bool = False) -> str:
    """Compile liboracle.so when it is missing or older than its source; return its path."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    tmp = LIB + f".tmp{os.getpid()}"
    subprocess.run(["gcc", *CFLAGS, "-o", tmp, SRC, "-lm"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
