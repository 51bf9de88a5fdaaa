"""The benchmark workloads at their full sizes against the reference's own
build (oracle/_ref, the same GPU, through its C API): the same status,
iteration count, objective, relative residuals and solution (see
test_gpu_reference.check_same_solution for what is compared).

- sparse QP (n = 1e4, m = 5e3, sparse Q = B'B + 0.1 I, inner BB solve) at
  eps 1e-4 and 1e-6: iterates within 1e-4 relative (the BB stopping test
  sees the rounding differences of the two builds; ~8e-7 measured);
- SOC-constrained QP (n = 1e6, 20000 SOC blocks of 50, m = 5e5) at 1e-6,
  the plain FP64 form (iterates ~5e-10 apart) and the mixed form (FP32
  bulk, FP64 polish below 1e-5): the mixed form's answer against the FP64
  reference solve is within 1e-6 in x, y and the reduced cost (~5e-7
  measured), 1e-7 in the objective (~4e-9 measured) and 0.5 eps in each
  relative residual;
- low-rank portfolio QP (n = 2e5, dense R 100 x 2e5, RSOC tracking error)
  at 1e-6;
- 32 of the batched MPC instances (T in [10, 100], eps 1e-5) solved by one
  pdhcg_b200_solve_batch call (FP32 storage, FP64 accumulation and
  residuals) against one reference solve each: the same status,
  iterations within 2 % + 10, objective within 10 eps, x, y within 1e-4
  relative;
- 5 held-out instances of the parametric family of the learned warm start
  (n = 5e4), cold, at 1e-6.

Skipped when the reference build is absent."""
import ctypes as C
import os

import pytest

from pdhcg_b200 import capi, instances, native
from test_gpu_reference import check_same_solution, _solve

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libpdhcg_ref.so")


def _eps(e):
    return {"termination_criteria.eps_optimal_relative": e, "termination_criteria.eps_feasible_relative": e}


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF):
        pytest.skip("the reference build (oracle/_ref) is not present")
    return capi.bind_api(C.CDLL(REF))


@pytest.mark.parametrize("eps", [1e-4, 1e-6])
def test_sparse_qp_full_size(lib, ref, eps):
    p = instances.sparse_qp(seed=1)
    g, r = _solve(lib, p, _eps(eps)), _solve(ref, p, _eps(eps))
    assert g["total_count"] == r["total_count"], (g["total_count"], r["total_count"])
    check_same_solution(g, r, eps, sol_tol=1e-4, res_tol=0.2)


def test_soc_qp_full_size_fp64_and_mixed(lib, ref):
    p = instances.soc_qp(seed=2)
    r = _solve(ref, p, _eps(1e-6))
    g = _solve(lib, p, _eps(1e-6))
    assert g["total_count"] == r["total_count"], (g["total_count"], r["total_count"])
    check_same_solution(g, r, 1e-6)
    mixed = _solve(lib, p, _eps(1e-6), native.default_options(precision=1))
    assert abs(mixed["total_count"] - r["total_count"]) <= 0.1 * r["total_count"], (mixed["total_count"],
                                                                                   r["total_count"])
    check_same_solution(mixed, r, 1e-6, obj_tol=1e-7, sol_tol=1e-6, res_tol=0.5)


def test_portfolio_full_size(lib, ref):
    p = instances.portfolio(seed=3)
    g, r = _solve(lib, p, _eps(1e-6)), _solve(ref, p, _eps(1e-6))
    assert g["total_count"] == r["total_count"], (g["total_count"], r["total_count"])
    check_same_solution(g, r, 1e-6, sol_tol=1e-6)
    # mixed: FP32 values of R and of A's long rows in the bulk phase, FP64 polish
    mixed = _solve(lib, p, _eps(1e-6), native.default_options(precision=1))
    assert abs(mixed["total_count"] - r["total_count"]) <= 0.1 * r["total_count"], (mixed["total_count"],
                                                                                   r["total_count"])
    check_same_solution(mixed, r, 1e-6, obj_tol=1e-7, sol_tol=1e-6, res_tol=0.5)


def test_mpc_batch_sample_against_reference(lib, ref):
    eps = 1e-5
    over = {**_eps(eps), "termination_criteria.iteration_limit": 200000}
    probs = instances.mpc_batch(seed=4, count=32)
    got = native.solve_batch(probs, over)
    for p, g in zip(probs, got):
        r = _solve(ref, p, over)
        assert abs(g["total_count"] - r["total_count"]) <= 0.02 * r["total_count"] + 10, (g["total_count"],
                                                                                        r["total_count"])
        check_same_solution(g, r, eps, obj_tol=10 * eps, sol_tol=1e-4, res_tol=1.0)


def test_parametric_family_against_reference(lib, ref):
    from pdhcg_b200.warmstart import ParametricQP
    fam = ParametricQP(seed=5)
    for th in fam.thetas(5, seed=777):
        p = fam.problem(th)
        g, r = _solve(lib, p, _eps(1e-6)), _solve(ref, p, _eps(1e-6))
        assert g["total_count"] == r["total_count"], (g["total_count"], r["total_count"])
        check_same_solution(g, r, 1e-6)
