"""Build recipe of the oracle's C part (test infrastructure, never linked into the library).

    python -m oracle.build [--force]

Compiles ``oracle/twobody_f32.c`` (the bit-exact FP32 restatement of the plain network) into
``oracle/libhignn_oracle.so`` with gcc: -O3, OpenMP, and -ffp-contract=off so that only the
explicit fused multiply-adds fuse. The batch kernel is built twice (x86-64-v3 with hardware FMA,
and a baseline build whose fmaf is the correctly rounded library call) and chosen at load time;
both give the same bits.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "twobody_f32.c")
LIB = os.path.join(HERE, "libhignn_oracle.so")


def build(force=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O3", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-math-errno",
           "-fno-trapping-math", SRC, "-o", LIB, "-lm"]
    p = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if p.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + " ".join(cmd) + "\n" + p.stdout)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
