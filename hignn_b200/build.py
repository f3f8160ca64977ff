"""Build recipe of the native library (nvcc/g++ only, no CMake), in-tree.

Produces ``hignn_b200/libhignn_b200.so`` (the C ABI of ``include/hignn_b200.h``,
CUDA runtime linked statically) and ``hignn_b200/hignn.<ext>`` (the pybind11
module that mirrors the reference's ``hignn`` Python interface on top of the C
ABI). All CUDA code is compiled for sm_100a only.

    python -m hignn_b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(REPO, "_build", "obj")
LIB = os.path.join(HERE, "libhignn_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CXX = shutil.which("g++") or "g++"

CU_SOURCES = {
    # file: extra nvcc flags
    "near_simt.cu": [],
    "far_aca.cu": ["-fmad=false"],  # FP64 determinants / inverses round as written
    "misc.cu": [],
    "tc_kernels.cu": [],
    "noalloc.cu": [],
    "dense_f64.cu": [],
    "tree_dev.cu": ["-fmad=false"],  # the device tree rounds every operation as the host build does
    "student.cu": [],
    "step.cu": [],
    "neighbors.cu": [],
    "three_body.cu": [],
    "capi.cu": [],
}
CXX_SOURCES = {
    # exact float/double rounding: the tree must match the restated reference bit for bit
    "tree.cpp": ["-ffp-contract=off"],
}


def _run(cmd):
    p = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if p.returncode != 0:
        raise RuntimeError("command failed:\n" + " ".join(cmd) + "\n" + p.stdout)
    return p.stdout


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(REPO, "include", "hignn_b200.h"))
    return hs


def compile_objects(force=False, jobs=8, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers()
    cmds = []
    objs = []
    for f, extra in CU_SOURCES.items():
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            cmds.append([NVCC, "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fopenmp",
                         "-Xptxas", "-v" if verbose else "-O3", "--expt-relaxed-constexpr",
                         "-I", os.path.join(REPO, "include"), *extra, "-c", src, "-o", obj])
    for f, extra in CXX_SOURCES.items():
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            cmds.append([CXX, "-std=c++17", "-O2", "-fPIC", "-fopenmp", *extra, "-I", os.path.join(REPO, "include"),
                         "-c", src, "-o", obj])
    if cmds:
        with cf.ThreadPoolExecutor(max(1, jobs)) as ex:
            outs = list(ex.map(_run, cmds))
        if verbose:
            for o in outs:
                sys.stdout.write(o)
    return objs


def link_library(objs, force=False):
    if force or _stale(LIB, objs):
        _run([NVCC, "-shared", *ARCH, "-cudart", "static", "-o", LIB, *objs, "-Xcompiler", "-fopenmp", "-lgomp"])
    return LIB


def build_pybind(force=False):
    import pybind11

    ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    out = os.path.join(HERE, "hignn" + ext)
    src = os.path.join(CSRC, "hignn_pybind.cpp")
    if not os.path.exists(src):
        return None
    if force or _stale(out, [src, LIB, os.path.join(REPO, "include", "hignn_b200.h")]):
        inc = sysconfig.get_paths()["include"]
        _run([CXX, "-std=c++17", "-O2", "-shared", "-fPIC", "-fvisibility=hidden", "-I", pybind11.get_include(),
              "-I", inc, "-I", os.path.join(REPO, "include"), src, "-o", out, "-L", HERE, "-lhignn_b200",
              "-Wl,-rpath,$ORIGIN"])
    return out


def build(force=False, jobs=8, verbose=False):
    objs = compile_objects(force=force, jobs=jobs, verbose=verbose)
    link_library(objs, force=force)
    build_pybind(force=force)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("-v", action="store_true", help="print ptxas register/spill reports")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j, verbose=a.v))
