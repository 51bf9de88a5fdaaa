"""The oracle pinned before it is trusted (CPU, no GPU needed).

1. Rescaling is bit-identical to the reference's own rescale_problem, through
   the committed golden fixtures (tests/golden/scaling.npz, produced by
   tests/golden/make_golden.py from the reference) and, when the reference
   library is built, directly.
2. Whole solves reproduce the answers the reference's end-to-end tests assert
   (tests/problems.py).
"""
import ctypes as C
import os

import numpy as np
import pytest

from pdhcg_b200 import capi
from golden_problems import SCALING_CASES, scaling_problem
from problems import INFEASIBLE, KNOWN_ANSWERS, check_known_answer

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scaling.npz")
_dp = C.POINTER(C.c_double)


def _builder(request):
    """Problems are built by the reference's create_qp_problem when it is
    available, else by the product library's host-only builder."""
    try:
        return request.getfixturevalue("ref")
    except pytest.skip.Exception:
        return request.getfixturevalue("lib")


def _oracle_rescale(oracle, prob, prm, m, n):
    cr, vr = np.zeros(m), np.zeros(n)
    sb, sc = C.c_double(), C.c_double()
    oracle.oracle_rescale(prob, C.byref(prm), cr.ctypes.data_as(_dp), vr.ctypes.data_as(_dp), C.byref(sb),
                          C.byref(sc))
    return cr, vr, sb.value, sc.value


@pytest.mark.parametrize("case", sorted(SCALING_CASES))
def test_rescale_matches_reference_golden(case, oracle, request):
    g = np.load(GOLDEN)
    builder = _builder(request)
    spec = SCALING_CASES[case]
    p = scaling_problem(spec["seed"])
    prob, keep = capi.build(builder, p)
    prm = capi.default_params(builder, **spec["params"])
    cr, vr, sb, sc = _oracle_rescale(oracle, prob, prm, len(p.con_lb), p.n)
    # bit-for-bit: same operations in the same order as the reference
    assert np.array_equal(cr, g[f"{case}/con_rescale"])
    assert np.array_equal(vr, g[f"{case}/var_rescale"])
    assert (sb, sc) == tuple(g[f"{case}/scalars"])


@pytest.mark.parametrize("name", sorted(KNOWN_ANSWERS))
def test_oracle_known_answers(name, oracle, request):
    builder = _builder(request)
    p, prm_over, expect = KNOWN_ANSWERS[name]()
    prob, keep = capi.build(builder, p)
    prm = capi.default_params(builder, **prm_over)
    r = oracle.oracle_solve(prob, C.byref(prm))
    assert r
    res = capi.result_dict(r, p.n, 0 if p.A is None else p.A.m)
    oracle.oracle_result_free(r)
    check_known_answer(res, expect)


def test_oracle_sigma_max_matches_svd(oracle):
    rng = np.random.default_rng(3)
    A = rng.standard_normal((40, 70)) * (rng.random((40, 70)) < 0.2)
    M = capi.CsrMatrix.from_dense(A)
    s = oracle.oracle_sigma_max(M.m, M.n, M.row_ptr.ctypes.data_as(C.POINTER(C.c_int)),
                                M.col_ind.ctypes.data_as(C.POINTER(C.c_int)), M.val.ctypes.data_as(_dp), 5000, 1e-10)
    assert abs(s - np.linalg.svd(A, compute_uv=False)[0]) <= 1e-6 * s


def _proj(oracle, typ, vdim, x, d, q=None, tau=0.0):
    x = np.array(x, dtype=np.float64)
    d = np.array(d, dtype=np.float64)
    qq = None if q is None else np.array(q, dtype=np.float64)
    oracle.oracle_project_cone_block(typ, vdim, 0.0, x.ctypes.data_as(_dp), d.ctypes.data_as(_dp),
                                     None if qq is None else qq.ctypes.data_as(_dp), tau)
    return x


@pytest.mark.parametrize("typ", [capi.CONE_STANDARD_SOC, capi.CONE_ROTATED_SOC])
def test_oracle_weighted_projection_is_optimal(oracle, typ):
    """Weighted projection = argmin over the cone, checked against a brute
    force: random feasible points never do better, KKT residual small."""
    rng = np.random.default_rng(5)
    k = 6
    for trial in range(50):
        r = rng.standard_normal(k + 2) * 3
        d = rng.uniform(0.5, 2.0, k + 2)
        q = rng.uniform(0.0, 3.0, k + 2)
        tau = 0.7
        x = _proj(oracle, typ, k, r, d, q, tau)
        w = 1 + tau * q
        u = x / d

        def in_cone(u, eps=1e-9):
            if typ == capi.CONE_STANDARD_SOC:
                return np.linalg.norm(u[:k + 1]) <= u[k + 1] + eps
            return u[k] >= -eps and u[k + 1] >= -eps and u[:k] @ u[:k] <= 2 * u[k] * u[k + 1] + eps

        assert in_cone(u, 1e-7)
        f0 = np.sum(w * (x - r) ** 2)
        # perturb along feasible points on the segment to x and beyond
        for _ in range(20):
            t = rng.uniform(0, 1)
            cand_u = u + t * rng.standard_normal(k + 2) * 0.01
            if in_cone(cand_u, 0.0):
                assert np.sum(w * (cand_u * d - r) ** 2) >= f0 - 1e-9


@pytest.mark.parametrize("name", sorted(INFEASIBLE))
def test_oracle_detects_infeasibility(lib, oracle, name):
    """The oracle's certificate logic (reference compute_infeasibility_information)
    reports the expected status on the constructed infeasible instances."""
    make, status = INFEASIBLE[name]
    p = make()
    prob, keep = capi.build(lib, p)
    prm = capi.default_params(lib, **{"termination_criteria.iteration_limit": 2000})
    r = oracle.oracle_solve(prob, C.byref(prm))
    d = capi.result_dict(r, p.n, p.A.m)
    oracle.oracle_result_free(r)
    lib.qp_problem_free(prob)
    assert d["status"] == status


def test_mpc_instances_have_the_batched_shape():
    """MPC generator: n = 12 T, m = 8 T, 13 nonzeros per dynamics row
    (5 in the first block row), inputs boxed, states free."""
    from pdhcg_b200 import instances
    for T in (10, 37, 100):
        p = instances.mpc_qp(3, T)
        assert p.n == 12 * T and p.A.m == 8 * T
        assert p.A.nnz == 8 * (1 + 4) + 8 * (T - 1) * 13
        assert np.all(p.var_lb[8 * T:] == -1.0) and np.all(np.isinf(p.var_lb[:8 * T]))


def test_mlp_oracle_gradient_matches_finite_differences():
    """The oracle's backward formulas (without BF16 rounding) against central
    differences of its own loss."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("mlp_oracle", os.path.join(os.path.dirname(
        os.path.dirname(os.path.abspath(__file__))), "oracle", "mlp_oracle.py"))
    mo = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mo)
    rng = np.random.default_rng(0)
    dims = (3, 6, 2, 5)
    npar = sum(int(np.prod(s)) for s in mo.shapes(*dims))
    w = rng.standard_normal(npar) * 0.5
    x, t, tl = rng.standard_normal((4, 3)), rng.standard_normal((4, 5)), rng.standard_normal(4)
    _, g, _, _ = mo.loss_grad(w, x, t, tl, *dims, quantize=False)
    h = 1e-6
    for k in rng.choice(npar, 25, replace=False):
        e = np.zeros(npar)
        e[k] = h
        lp = mo.loss_grad(w + e, x, t, tl, *dims, quantize=False)[0]
        lm = mo.loss_grad(w - e, x, t, tl, *dims, quantize=False)[0]
        assert abs((lp - lm) / (2 * h) - g[k]) <= 1e-6 * (1 + abs(g[k]))
