"""Known-answer problems from the reference's own end-to-end tests.

Each entry restates the problem data and the expected answer of one test
in the reference's test/ directory (cited per entry), so the oracle and the
CUDA solver are both checked against the answers the reference asserts.
"""
import numpy as np

from pdhcg_b200.capi import (CONE_ROTATED_SOC, CONE_STANDARD_SOC, Cone, CsrMatrix, Problem)

BIG = 1e30


def lp_small():
    """test/test_c_api_working.c:72-277: min x + 2y s.t. x + y = 1, x, y >= 0.
    Expected x ~ (1, 0), y ~ 1, objective ~ 1."""
    p = Problem(c=np.array([1.0, 2.0]), A=CsrMatrix.from_dense([[1.0, 1.0]]), con_lb=np.array([1.0]),
                con_ub=np.array([1.0]), var_lb=np.array([0.0, 0.0]), var_ub=np.array([BIG, BIG]))
    return p, {}, {"x": [1.0, 0.0], "y": [1.0], "obj": 1.0, "tol": 1e-3}


def sparse_q_soc():
    """test/test_sparse_q_cones.c:19-90: sparse Q couples (a, b); (v, w, z) in SOC.
    Expected a=3, b=4, v=3, w=4, z=5, objective -1.5 (tol 1e-4)."""
    A = CsrMatrix(4, 5, np.array([0, 1, 2, 4, 6]), np.array([0, 1, 0, 2, 1, 3]),
                  np.array([1.0, 1.0, 1.0, -1.0, 1.0, -1.0]))
    Q = CsrMatrix(5, 5, np.array([0, 2, 4, 4, 4, 4]), np.array([0, 1, 0, 1]), np.array([1.0, 0.5, 0.5, 1.0]))
    p = Problem(c=np.array([-3.0, -4.0, 0.0, 0.0, 1.0]), A=A, Q=Q, con_lb=np.array([3.0, 4.0, 0.0, 0.0]),
                con_ub=np.array([3.0, 4.0, 0.0, 0.0]), var_lb=np.full(5, -BIG), var_ub=np.full(5, BIG),
                cones=[Cone(CONE_STANDARD_SOC, 2, 1)])
    prm = {"termination_criteria.eps_optimal_relative": 1e-7, "termination_criteria.eps_feasible_relative": 1e-7,
           "termination_criteria.iteration_limit": 100000}
    return p, prm, {"x": [3.0, 4.0, 3.0, 4.0, 5.0], "obj": -1.5, "tol": 1e-4}


def soc_diag_q():
    """test/test_diag_q_cones.c:20-102: min 1/2 v^2 + 1/2 z^2 - 3v - 4z s.t. w = 4,
    (v, w, z) in SOC.  KKT: w = 4, v^2 + w^2 = z^2, (3/v - 1)/2 = (1 - 4/z)/2."""
    A = CsrMatrix(1, 3, np.array([0, 1]), np.array([1]), np.array([1.0]))
    Q = CsrMatrix(3, 3, np.array([0, 1, 1, 2]), np.array([0, 2]), np.array([1.0, 1.0]))
    p = Problem(c=np.array([-3.0, 0.0, -4.0]), A=A, Q=Q, con_lb=np.array([4.0]), con_ub=np.array([4.0]),
                var_lb=np.full(3, -BIG), var_ub=np.full(3, BIG), cones=[Cone(CONE_STANDARD_SOC, 0, 1)])
    prm = {"termination_criteria.eps_optimal_relative": 1e-8, "termination_criteria.eps_feasible_relative": 1e-8,
           "termination_criteria.iteration_limit": 100000}
    return p, prm, {"soc_kkt": True, "tol": 1e-5}


def rsoc_diag_q_sym():
    """test/test_diag_q_cones.c:105-170: no rows, (v, s, t) in RSOC.
    Expected v = 1, s = t = 3, objective -9.5."""
    A = CsrMatrix(0, 3, np.array([0]), np.zeros(0, np.int32), np.zeros(0))
    Q = CsrMatrix(3, 3, np.array([0, 1, 2, 3]), np.array([0, 1, 2]), np.array([1.0, 1.0, 1.0]))
    p = Problem(c=np.array([-1.0, -3.0, -3.0]), A=A, Q=Q, var_lb=np.full(3, -BIG), var_ub=np.full(3, BIG),
                cones=[Cone(CONE_ROTATED_SOC, 0, 1)])
    prm = {"termination_criteria.eps_optimal_relative": 1e-8, "termination_criteria.eps_feasible_relative": 1e-8,
           "termination_criteria.iteration_limit": 100000}
    return p, prm, {"x": [1.0, 3.0, 3.0], "obj": -9.5, "tol": 1e-4}


def rsoc_diag_q_asym():
    """test/test_diag_q_cones.c:173-275: RSOC with Q_s != Q_t, boundary active.
    Reference solution (v, s, t) = (3.26153501744331, 4.28128575585834,
    1.24233831570958), objective -17.57031817800 (tol 1e-3)."""
    A = CsrMatrix(0, 3, np.array([0]), np.zeros(0, np.int32), np.zeros(0))
    Q = CsrMatrix(3, 3, np.array([0, 1, 2, 3]), np.array([0, 1, 2]), np.array([1.0, 1.0, 4.0]))
    p = Problem(c=np.array([-4.0, -4.0, -4.0]), A=A, Q=Q, var_lb=np.full(3, -BIG), var_ub=np.full(3, BIG),
                cones=[Cone(CONE_ROTATED_SOC, 0, 1)])
    prm = {"termination_criteria.eps_optimal_relative": 1e-8, "termination_criteria.eps_feasible_relative": 1e-8,
           "termination_criteria.iteration_limit": 200000}
    return p, prm, {"x": [3.26153501744331, 4.28128575585834, 1.24233831570958], "obj": -17.57031817800,
                    "tol": 1e-3}


KNOWN_ANSWERS = {
    "lp_small": lp_small,
    "sparse_q_soc": sparse_q_soc,
    "soc_diag_q": soc_diag_q,
    "rsoc_diag_q_sym": rsoc_diag_q_sym,
    "rsoc_diag_q_asym": rsoc_diag_q_asym,
}


def check_known_answer(res: dict, expect: dict):
    """Assert a solve result against a known answer (the reference's own checks)."""
    assert res["status"] == "OPTIMAL", res["status"]
    tol = expect["tol"]
    x = res["x"]
    if "x" in expect:
        np.testing.assert_allclose(x, expect["x"], atol=tol * (1 + np.abs(expect["x"])).max())
    if "y" in expect:
        np.testing.assert_allclose(res["y"], expect["y"], atol=tol * 10)
    if "obj" in expect:
        assert abs(res["primal_objective_value"] - expect["obj"]) <= 10 * tol * (1 + abs(expect["obj"]))
    if expect.get("soc_kkt"):
        v, w, z = x
        assert abs(w - 4.0) <= tol * 5
        assert abs(v * v + w * w - z * z) <= tol
        assert abs((3.0 / v - 1.0) / 2.0 - (1.0 - 4.0 / z) / 2.0) <= 1e-4
