"""Build libpdhcg_b200.so in-tree with nvcc for sm_100a.

    python -m pdhcg_b200.build          # incremental
    python -m pdhcg_b200.build --force

The library is plain C ABI (include/pdhcg.h, include/pdhcg_b200.h); no
PyTorch types cross it.  CUDA runtime is linked statically so the library
does not depend on which libcudart another component of the process loaded.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpdhcg_b200.so")
SOURCES = ["solver.cu", "batch.cu", "mlp.cu", "api.cpp", "mps.cpp", "qcqp.cpp"]
HEADERS = ["device.cuh", "kernels.cuh", "residual.cuh", "setup.cuh", "bb.cuh", "section.cuh", "internal.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps += [os.path.join(ROOT, "include", f) for f in ("pdhcg.h", "pdhcg_types.h", "pdhcg_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objs, cmds = [], []
    nvcc = _nvcc()
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]
    for src in SOURCES:
        obj = os.path.join(CSRC, os.path.splitext(src)[0] + ".o")
        if src.endswith(".cu"):
            # (no --split-compile: it cut the build from 10 to 3.5 min but
            # changed the register allocation of the step kernels -- 80 -> 101
            # registers on the cone kernel, spills in the FP32 dual kernel --
            # and cost ~8 % of the step)
            cmd = [nvcc, *ARCH, "-lineinfo", "-Xptxas", "-warn-spills", *common, "-c", os.path.join(CSRC, src),
                   "-o", obj]
        else:
            cmd = [os.environ.get("CXX", "g++"), "-O3", "-std=c++17", "-fPIC", "-I" + os.path.join(ROOT, "include"),
                   "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        cmds.append(cmd)
        objs.append(obj)
    # the translation units compile side by side (solver.cu dominates)
    with ThreadPoolExecutor(max_workers=len(cmds)) as pool:
        for f in [pool.submit(subprocess.check_call, c) for c in cmds]:
            f.result()
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", *objs, "-o", tmp, "-Xlinker", "-Bsymbolic", "-lz"]  # zlib: gzip MPS files
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
