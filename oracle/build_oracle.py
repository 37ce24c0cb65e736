"""Build recipe for the oracle library (test infrastructure).

    python oracle/build_oracle.py

Compiles ``parflex_oracle.c`` with gcc into ``oracle/_build/liboracle.so``.
``-ffp-contract=off`` keeps every FP64 multiply and add separately rounded,
as in the reference's non-fastmath Numba code; OpenMP spreads stage-1 tiles
over host threads (the reference's cpu_parflex.py spreads them over a
process pool).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose: bool = False) -> str:
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    src = os.path.join(HERE, "parflex_oracle.c")
    out = os.path.join(out_dir, "liboracle.so")
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    cmd = ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math",
           "-fopenmp", "-fPIC", "-shared", "-Wall", "-Wno-unused-result",
           "-o", out + ".tmp", src, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build(verbose=True))
    sys.exit(0)
