"""The device rescaling (Curtis-Reid, Ruiz, Pock-Chambolle, bound /
objective scaling and the cone-preserving adjustment, pdhcg_b200_rescaling)
against the reference's own rescale_problem through the committed golden
fixtures (tests/golden/scaling.npz, generated from the reference by
tests/golden/make_golden.py).  The device kernels restate the reference's
host loops operation for operation, but the device compiler contracts
multiply-adds into fused ones, so the factors agree to a few units in the
last place (4e-16 .. 7e-16 relative measured: tolerance 4e-15), and to
1e-13 where the device's pow / log / exp (Pock-Chambolle with
alpha != 1, Curtis-Reid) round differently from the host's."""
import ctypes as C
import os

import numpy as np
import pytest

from pdhcg_b200 import capi
from golden_problems import SCALING_CASES, scaling_problem

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scaling.npz")
TOL = {"curtis_reid": 1e-13, "pc_alpha_half": 1e-13}  # else 4e-15


@pytest.mark.parametrize("case", sorted(SCALING_CASES))
def test_device_rescaling_matches_reference_golden(lib, case):
    g = np.load(GOLDEN)
    spec = SCALING_CASES[case]
    p = scaling_problem(spec["seed"])
    prob, keep = capi.build(lib, p)
    assert prob
    prm = capi.default_params(lib, **spec["params"])
    m, n = len(p.con_lb), p.n
    cr, vr, bo = np.zeros(m), np.zeros(n), np.zeros(2)
    dp = C.POINTER(C.c_double)
    rc = lib.pdhcg_b200_rescaling(prob, C.byref(prm), cr.ctypes.data_as(dp), vr.ctypes.data_as(dp),
                                  bo.ctypes.data_as(dp))
    lib.qp_problem_free(prob)
    assert rc == 0
    want_cr, want_vr, want_s = g[f"{case}/con_rescale"], g[f"{case}/var_rescale"], g[f"{case}/scalars"]
    tol = TOL.get(case, 4e-15)
    for got, want in ((cr, want_cr), (vr, want_vr), (bo, want_s)):
        err = np.abs(got - want) / np.abs(want)
        assert err.max() <= tol, (case, err.max(), int(err.argmax()))


def test_rescaling_refuses_bad_arguments(lib):
    assert lib.pdhcg_b200_rescaling(None, None, None, None, None) == -1
