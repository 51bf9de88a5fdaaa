"""Shared fixtures.

- ``oracle``: the CPU restatement (oracle/liboracle.so), the checker.
- ``ref``: the reference solver built from its own sources (oracle/_ref/),
  used as a checker; tests that need it skip when it was not built.
- ``lib``: the product library libpdhcg_b200.so.
"""
import ctypes as C
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from pdhcg_b200 import capi  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    path = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(path):
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle")], stdout=subprocess.DEVNULL)
    lib = C.CDLL(path)
    lib.oracle_solve.restype = C.POINTER(capi.PdhcgResult)
    lib.oracle_solve.argtypes = [C.POINTER(capi.QpProblem), C.POINTER(capi.PdhgParameters)]
    dp = C.POINTER(C.c_double)
    lib.oracle_rescale.argtypes = [C.POINTER(capi.QpProblem), C.POINTER(capi.PdhgParameters), dp, dp, dp, dp]
    lib.oracle_sigma_max.restype = C.c_double
    lib.oracle_sigma_max.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), dp, C.c_int, C.c_double]
    lib.oracle_project_cone_block.argtypes = [C.c_int, C.c_int, C.c_double, dp, dp, dp, C.c_double]
    lib.oracle_cone_dual_residual_block.argtypes = [C.c_int, C.c_int, C.c_double, dp, dp, dp]
    lib.pdhcg_result_free = None
    return lib


@pytest.fixture(scope="session")
def ref():
    path = os.path.join(ROOT, "oracle", "_ref", "libpdhcg_ref.so")
    if not os.path.exists(path):
        pytest.skip("reference library oracle/_ref/libpdhcg_ref.so not built")
    return capi.bind_api(C.CDLL(path))


@pytest.fixture(scope="session")
def lib():
    from pdhcg_b200 import native
    return native.load()
