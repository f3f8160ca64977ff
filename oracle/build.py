"""Build recipe of the oracle's C part (test infrastructure, never linked into the library).

    python -m oracle.build [--force]

Compiles ``oracle/twobody_f32.c`` (the bit-exact FP32 restatement of the plain network) and
``oracle/hmatvec_cpu.cpp`` (the C++/OpenMP restatement of the H-matvec: CloseDot, ACA FarDot) into
``oracle/libhignn_oracle.so`` with gcc/g++: -O3, OpenMP, and -ffp-contract=off so that only the
explicit fused multiply-adds fuse. The batch kernel is built twice (x86-64-v3 with hardware FMA,
and a baseline build whose fmaf is the correctly rounded library call) and chosen at load time;
both give the same bits.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC_C = os.path.join(HERE, "twobody_f32.c")
SRC_CPP = os.path.join(HERE, "hmatvec_cpu.cpp")
LIB = os.path.join(HERE, "libhignn_oracle.so")
OBJ = os.path.join(os.path.dirname(HERE), "_build", "oracle")


def _run(cmd):
    p = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if p.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + " ".join(cmd) + "\n" + p.stdout)


def build(force=False):
    srcs = (SRC_C, SRC_CPP)
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(f) for f in srcs):
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    flags = ["-O3", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-math-errno", "-fno-trapping-math"]
    o1, o2 = os.path.join(OBJ, "twobody_f32.o"), os.path.join(OBJ, "hmatvec_cpu.o")
    _run(["gcc", *flags, "-c", SRC_C, "-o", o1])
    _run(["g++", "-std=c++17", *flags, "-c", SRC_CPP, "-o", o2])
    _run(["g++", "-shared", "-fopenmp", o1, o2, "-o", LIB, "-lm"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
