"""Generate golden fixtures from the reference itself.

Runs on a machine where the reference sources are present and
oracle/_ref/libpdhcg_ref.so has been built (``make -f oracle/ref.mk``).
Only host-side reference functions are called (create_qp_problem,
rescale_problem), so no GPU is needed.  Output: tests/golden/scaling.npz.

    python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from pdhcg_b200 import capi  # noqa: E402
from golden_problems import SCALING_CASES, scaling_problem  # noqa: E402


class RescaleInfo(C.Structure):
    """rescale_info_t, reference internal/internal_types.h:301-310."""
    _fields_ = [("scaled_problem", C.POINTER(capi.QpProblem)), ("processed", C.c_void_p),
                ("con_rescale", C.POINTER(C.c_double)), ("var_rescale", C.POINTER(C.c_double)),
                ("con_bound_rescale", C.c_double), ("obj_vec_rescale", C.c_double), ("time", C.c_double)]


def reference_rescale(ref, prob, prm, m, n):
    ref.rescale_problem.restype = C.POINTER(RescaleInfo)
    ref.rescale_problem.argtypes = [C.POINTER(capi.PdhgParameters), C.POINTER(capi.QpProblem)]
    info = ref.rescale_problem(C.byref(prm), prob).contents
    cr = np.ctypeslib.as_array(info.con_rescale, shape=(m,)).copy()
    vr = np.ctypeslib.as_array(info.var_rescale, shape=(n,)).copy()
    return cr, vr, info.con_bound_rescale, info.obj_vec_rescale


def main():
    ref = capi.bind_api(C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libpdhcg_ref.so")))
    out = {}
    for name, case in SCALING_CASES.items():
        p = scaling_problem(case["seed"])
        prob, keep = capi.build(ref, p)
        prm = capi.default_params(ref, **case["params"])
        cr, vr, sb, sc = reference_rescale(ref, prob, prm, len(p.con_lb), p.n)
        out[f"{name}/con_rescale"] = cr
        out[f"{name}/var_rescale"] = vr
        out[f"{name}/scalars"] = np.array([sb, sc])
        ref.qp_problem_free(prob)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "scaling.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
