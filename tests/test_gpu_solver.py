"""Whole solves on the GPU through the C ABI, checked against the oracle and
against the answers of the reference's own end-to-end tests.

Tolerances: both sides run the same FP64 iteration, but the device sums
in a different order, so trajectories agree to rounding and drift apart
slowly.  The termination status must be identical; objectives must agree to
within the termination tolerance; iteration counts within 25 %.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from pdhcg_b200 import capi, instances, native
from pdhcg_b200.capi import CsrMatrix
from problems import INFEASIBLE, KNOWN_ANSWERS, check_known_answer

pytestmark = pytest.mark.gpu


def _solve_gpu(lib, p, params):
    prob, keep = capi.build(lib, p)
    assert prob
    prm = capi.default_params(lib, **params)
    r = lib.solve_qp_problem(prob, C.byref(prm))
    assert r, "solve_qp_problem returned NULL"
    m = p.A.m if p.A is not None else 0
    d = capi.result_dict(r, p.n, max(m, 1))
    lib.pdhcg_result_free(r)
    lib.qp_problem_free(prob)
    return d


def _solve_oracle(oracle, lib, p, params):
    prob, keep = capi.build(lib, p)
    prm = capi.default_params(lib, **params)
    r = oracle.oracle_solve(prob, C.byref(prm))
    assert r
    m = p.A.m if p.A is not None else 0
    d = capi.result_dict(r, p.n, max(m, 1))
    oracle.oracle_result_free(r)
    lib.qp_problem_free(prob)
    return d


@pytest.mark.parametrize("name", sorted(KNOWN_ANSWERS))
def test_known_answers_on_gpu(lib, name):
    p, prm, expect = KNOWN_ANSWERS[name]()
    res = _solve_gpu(lib, p, prm)
    check_known_answer(res, expect)


def _all_cones_sparse_q(seed=16):
    """SOC / RSOC blocks covering every variable, with a tridiagonal Q (the
    inner BB solve with an empty free-variable list)."""
    p = instances.conic_lp(seed=seed, nfree=0)
    n = p.n
    rows, cols, vals = [], [], []
    for i in range(n):
        for j, v in ((i - 1, 0.3), (i, 1.0), (i + 1, 0.3)):
            if 0 <= j < n:
                rows.append(i), cols.append(j), vals.append(v)
    p.Q = CsrMatrix.from_scipy(sp.csr_matrix((vals, (rows, cols)), shape=(n, n)))
    return p


CASES = {
    "box_lp": (lambda: instances.box_lp(), {}),
    "diag_qp": (lambda: instances.diag_qp(), {}),
    "conic_lp": (lambda: instances.conic_lp(), {}),
    "conic_qp": (lambda: instances.conic_lp(with_q=True), {}),
    "soc_qp_small": (lambda: instances.soc_qp(scale=0.001),
                     {"termination_criteria.eps_optimal_relative": 1e-6,
                      "termination_criteria.eps_feasible_relative": 1e-6}),
    "diag_qp_l2": (lambda: instances.diag_qp(seed=9), {"optimality_norm": capi.NORM_L2}),
    "box_lp_no_bound_obj": (lambda: instances.box_lp(seed=8), {"bound_objective_rescaling": False}),
    # inner BB solve: sparse Q, and low rank + diagonal Q with a rotated-SOC block
    "sparse_qp_small": (lambda: instances.sparse_qp(scale=0.05), {}),
    "sparse_qp_no_precond": (lambda: instances.sparse_qp(seed=7, scale=0.03), {"diag_jacobi_precond": False}),
    "portfolio_small": (lambda: instances.portfolio(scale=0.01), {}),
    # Curtis-Reid scaling before Ruiz (cone-preserving and not)
    "box_lp_curtis_reid": (lambda: instances.box_lp(seed=10), {"curtis_reid_iterations": 8}),
    "conic_qp_curtis_reid": (lambda: instances.conic_lp(seed=11, with_q=True), {"curtis_reid_iterations": 5}),
    "conic_lp_curtis_reid_np": (lambda: instances.conic_lp(seed=12), {"curtis_reid_iterations": 5,
                                                                       "use_cone_preserving_scaling": False}),
    # every cone kind in one problem: the SOC / RSOC launch and the 3-slot launch of the step
    "mixed_cones_lp": (lambda: instances.conic_lp(seed=13, nexp=12, npow=12), {}),
    "mixed_cones_qp": (lambda: instances.conic_lp(seed=14, with_q=True, nexp=10, npow=10), {}),
    "exp_pow_only_qp": (lambda: instances.conic_lp(seed=15, nsoc=0, nrsoc=0, with_q=True, nexp=15, npow=15), {}),
    # rows and columns longer than the long-row threshold (segment passes before every product)
    "dense_rows_lp": (lambda: instances.dense_rows_qp(), {}),
    "dense_rows_qp": (lambda: instances.dense_rows_qp(seed=22, with_q=True), {}),
    "portfolio_long_rows": (lambda: instances.portfolio(seed=4, scale=0.05), {}),
    # PSD blocks: the LP step (own launch) and, with a diagonal Q, the inner BB solve
    "psd_lp": (lambda: instances.psd_lp(), {}),
    "psd_lp_mixed_cones": (lambda: instances.psd_lp(seed=7, orders=(2, 4, 1, 3)), {"use_cone_preserving_scaling": False}),
    "psd_qp": (lambda: instances.psd_lp(seed=8, with_q=True), {}),
    "psd_large_lp": (lambda: instances.psd_lp(seed=12, orders=(24, 3, 30)), {}),
    "all_cones_sparse_q": (_all_cones_sparse_q, {}),
    # affine cones F x + g in K over rows: every cone type, with and without Q
    "affine_lp": (lambda: instances.affine_cone_qp(), {}),
    "affine_qp": (lambda: instances.affine_cone_qp(seed=10, with_q=True), {}),
    "affine_lp_l2_np": (lambda: instances.affine_cone_qp(seed=13), {"optimality_norm": capi.NORM_L2,
                                                                     "use_cone_preserving_scaling": False}),
    "affine_lp_curtis_reid": (lambda: instances.affine_cone_qp(seed=14), {"curtis_reid_iterations": 5}),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_oracle(lib, oracle, name):
    make, prm = CASES[name]
    p = make()
    prm = {"termination_criteria.iteration_limit": 100000, **prm}
    g = _solve_gpu(lib, p, prm)
    o = _solve_oracle(oracle, lib, p, prm)
    assert g["status"] == o["status"] == "OPTIMAL"
    eps = prm.get("termination_criteria.eps_optimal_relative", 1e-4)
    assert abs(g["primal_objective_value"] - o["primal_objective_value"]) <= 10 * eps * (
        1 + abs(o["primal_objective_value"]))
    assert abs(g["total_count"] - o["total_count"]) <= max(40, 0.25 * o["total_count"]), (
        g["total_count"], o["total_count"])
    assert g["rel_kkt"] < eps


def test_gpu_iteration_limit_and_result_fields(lib):
    p = instances.box_lp(seed=11)
    g = _solve_gpu(lib, p, {"termination_criteria.iteration_limit": 37})
    assert g["status"] == "ITERATION_LIMIT"
    assert g["total_count"] == 37
    assert np.all(np.isfinite(g["x"])) and np.all(np.isfinite(g["y"]))


def _solve_gpu_opts(lib, p, params, **opts):
    prob, keep = capi.build(lib, p)
    prm = capi.default_params(lib, **params)
    o = native.default_options(**opts)
    r = lib.pdhcg_b200_solve(prob, C.byref(prm), C.byref(o))
    assert r
    m = p.A.m if p.A is not None else 0
    d = capi.result_dict(r, p.n, max(m, 1))
    lib.pdhcg_result_free(r)
    lib.qp_problem_free(prob)
    return d, native.last_stats()


@pytest.mark.parametrize("name", ["diag_qp", "conic_qp", "soc_qp_small", "box_lp", "dense_rows_qp", "affine_qp",
                                  "sparse_qp_small", "portfolio_small", "psd_qp"])
def test_mixed_precision_reaches_fp64_answer(lib, name):
    """FP32 bulk phase + FP64 polish: same status as plain FP64, objective
    within the termination tolerance of the FP64 answer, and the FP32 phase
    actually ran (fp32_iterations > 0).  The last three take the inner BB
    solve, whose bulk phase reads FP32 values of Q, R and R^T."""
    make, prm = CASES[name]
    p = make()
    prm = {"termination_criteria.iteration_limit": 100000,
           "termination_criteria.eps_optimal_relative": 1e-6,
           "termination_criteria.eps_feasible_relative": 1e-6}
    ref, _ = _solve_gpu_opts(lib, p, prm, precision=0)
    mix, st = _solve_gpu_opts(lib, p, prm, precision=1)
    assert ref["status"] == mix["status"] == "OPTIMAL"
    assert st["fp32_iterations"] > 0
    assert mix["rel_kkt"] < 1e-6
    assert abs(mix["primal_objective_value"] - ref["primal_objective_value"]) <= 1e-5 * (
        1 + abs(ref["primal_objective_value"]))


def test_device_resident_handle_matches_host_path(lib):
    """pdhcg_b200_upload + pdhcg_b200_solve_device give the same answer as the
    host-buffer call, the handle can be solved repeatedly, and the solution
    can stay on the device."""
    import torch
    p = instances.conic_lp(seed=31, with_q=True)
    prm_over = {"termination_criteria.iteration_limit": 50000}
    host = _solve_gpu(lib, p, prm_over)
    prob, keep = capi.build(lib, p)
    prm = capi.default_params(lib, **prm_over)
    h = lib.pdhcg_b200_upload(prob)
    assert h
    for _ in range(2):
        r = lib.pdhcg_b200_solve_device(h, C.byref(prm), None)
        assert r
        d = capi.result_dict(r, p.n, p.A.m)
        lib.pdhcg_result_free(r)
        assert d["status"] == host["status"]
        assert d["total_count"] == host["total_count"]
        np.testing.assert_allclose(d["x"], host["x"], rtol=1e-12, atol=1e-12)
    o = native.default_options(solution_on_device=1)
    r = lib.pdhcg_b200_solve_device(h, C.byref(prm), C.byref(o))
    assert r and not r.contents.primal_solution
    lib.pdhcg_result_free(r)
    xp, yp, rp = C.c_void_p(), C.c_void_p(), C.c_void_p()
    assert lib.pdhcg_b200_device_solution(h, C.byref(xp), C.byref(yp), C.byref(rp)) == 0
    torch.cuda.synchronize()

    class _DeviceArray:  # wraps the library's device pointer for torch
        def __init__(self, ptr, n):
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 2}

    xt = torch.as_tensor(_DeviceArray(xp.value, p.n), device="cuda")
    np.testing.assert_allclose(xt.cpu().numpy(), host["x"], rtol=1e-12, atol=1e-12)
    lib.pdhcg_b200_device_problem_free(h)
    lib.qp_problem_free(prob)


@pytest.mark.parametrize("name", sorted(INFEASIBLE))
def test_infeasibility_certificates_match_oracle(lib, oracle, name):
    """Infeasibility detection (reference compute_infeasibility_information,
    src/pdhg_core_op.cu:1296-1429): same status and iteration count as the
    oracle, certificate scalars to 1e-6 relative."""
    make, status = INFEASIBLE[name]
    p = make()
    prm = {"termination_criteria.iteration_limit": 2000}
    g = _solve_gpu(lib, p, prm)
    o = _solve_oracle(oracle, lib, p, prm)
    assert g["status"] == o["status"] == status
    assert g["total_count"] == o["total_count"]
    for f in ("max_primal_ray_infeasibility", "max_dual_ray_infeasibility", "primal_ray_linear_objective",
              "dual_ray_objective"):
        assert abs(g[f] - o[f]) <= 1e-6 * (1.0 + abs(o[f])), (f, g[f], o[f])
