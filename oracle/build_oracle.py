"""Build the CPU oracle: oracle/_build/libysoracle.so (test infrastructure).

    python -m oracle.build_oracle

-O3 -ffp-contract=off keeps every float operation a single IEEE binary32
rounding in source order (no FMA), the arithmetic the CUDA path reproduces.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build", "libysoracle.so")
SRCS = [os.path.join(HERE, "ys_oracle.cpp"), os.path.join(HERE, "ys_adjoint_oracle.cpp")]


def build(force: bool = False) -> str:
    if not force and os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(s) for s in SRCS):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["g++", "-O3", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           "-o", OUT + ".tmp", *SRCS]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
