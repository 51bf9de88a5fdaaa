"""Build libpdhcg_b200.so in-tree with nvcc for sm_100a.

    python -m pdhcg_b200.build          # incremental
    python -m pdhcg_b200.build --force

Incremental: nothing is done while the library is newer than every source
and header.  Otherwise every translation unit keeps its object, the
compiler's dependency list and its command line under pdhcg_b200/_build/; a
unit is recompiled when a file it includes is newer than its object or its
command changed, and the library is relinked.

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
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


BUILD = os.path.join(HERE, "_build")


def _deps(depfile: str) -> list[str]:
    """Prerequisites listed in a make-style dependency file (-MD -MF)."""
    try:
        with open(depfile) as f:
            text = f.read().replace("\\\n", " ")
    except OSError:
        return []
    _, _, rest = text.partition(":")
    return rest.split()


def _stamp(cmd: list[str]) -> str:
    """The command line with this tree's location taken out (a copied tree
    keeps its objects)."""
    return " ".join(cmd).replace(ROOT, "<root>")


def _unit_stale(obj: str, cmd: list[str]) -> bool:
    stamp, dep = obj + ".cmd", obj + ".d"
    if not (os.path.exists(obj) and os.path.exists(stamp) and os.path.exists(dep)):
        return True
    with open(stamp) as f:
        if f.read() != _stamp(cmd):
            return True
    t = os.path.getmtime(obj)
    deps = _deps(dep)
    if not deps:
        return True
    return any(not os.path.exists(d) or os.path.getmtime(d) > t for d in deps)


def _compile(obj: str, cmd: list[str]) -> None:
    subprocess.check_call(cmd + ["-MD", "-MF", obj + ".d"])
    with open(obj + ".cmd", "w") as f:
        f.write(_stamp(cmd))


def _lib_fresh() -> bool:
    """The library is newer than every source and header (the rule for a
    tree that carries the library but not the objects)."""
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".cpp", ".h"))]
    inc = os.path.join(ROOT, "include")
    files += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return all(os.path.getmtime(f) <= t for f in files)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and _lib_fresh():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    objs, todo = [], []
    nvcc = _nvcc()
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]
    for src in SOURCES:
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
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
        objs.append(obj)
        if force or _unit_stale(obj, cmd):
            if verbose:
                print(" ".join(cmd))
            todo.append((obj, cmd))
    # the translation units compile side by side (solver.cu dominates)
    if todo:
        with ThreadPoolExecutor(max_workers=len(todo)) as pool:
            for f in [pool.submit(_compile, o, c) for o, c in todo]:
                f.result()
    if not todo and os.path.exists(LIB) and all(os.path.getmtime(o) <= os.path.getmtime(LIB) for o in objs):
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", *objs, "-o", tmp, "-Xlinker", "-Bsymbolic", "-lz"]  # zlib: gzip MPS files
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
