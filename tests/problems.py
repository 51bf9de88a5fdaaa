"""Known-answer problems from the reference's own end-to-end tests.

Each entry restates the problem data and the expected answer of one test
in the reference's test/ directory (cited per entry), so the oracle and the
CUDA solver are both checked against the answers the reference asserts.
"""
import numpy as np

from pdhcg_b200.capi import (CONE_EXPONENTIAL, CONE_POWER, CONE_PSD, CONE_ROTATED_SOC, CONE_STANDARD_SOC, NORM_L2, Cone,
                             CsrMatrix, Problem)

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


def exp_cone_linear():
    """test/test_conic_e2e.c:148-215: min -x s.t. y = 1, z = 2, (x, y, z) in
    K_exp.  Expected x = log 2, y = 1, z = 2 (tol 5e-3)."""
    A = CsrMatrix(2, 3, np.array([0, 1, 2]), np.array([1, 2]), np.array([1.0, 1.0]))
    p = Problem(c=np.array([-1.0, 0.0, 0.0]), A=A, con_lb=np.array([1.0, 2.0]), con_ub=np.array([1.0, 2.0]),
                var_lb=np.full(3, -BIG), var_ub=np.full(3, BIG), cones=[Cone(CONE_EXPONENTIAL, 0, 1)])
    prm = {"termination_criteria.eps_optimal_relative": 1e-6, "termination_criteria.eps_feasible_relative": 1e-6,
           "termination_criteria.iteration_limit": 1000000}
    return p, prm, {"x": [np.log(2.0), 1.0, 2.0], "tol": 5e-3}


_POW_PRM = {"termination_evaluation_frequency": 10, "termination_criteria.eps_optimal_relative": 1e-8,
            "termination_criteria.eps_feasible_relative": 1e-8, "termination_criteria.iteration_limit": 1000000}


def pow_full_cone(alpha, l2=False):
    """test/test_power_cone.c:109-152: max z s.t. x + y = 2, (x, y, z) in
    K_alpha, started from (1, 1, 0).  Expected (2a, 2(1-a), (2a)^a (2(1-a))^(1-a))
    (tol 2e-5)."""
    A = CsrMatrix(1, 3, np.array([0, 2]), np.array([0, 1]), np.array([1.0, 1.0]))
    p = Problem(c=np.array([0.0, 0.0, -1.0]), A=A, con_lb=np.array([2.0]), con_ub=np.array([2.0]),
                var_lb=np.full(3, -np.inf), var_ub=np.full(3, np.inf), cones=[Cone(CONE_POWER, 0, 1, alpha=alpha)],
                primal_start=np.array([1.0, 1.0, 0.0]), dual_start=np.array([0.0]))
    om = 1.0 - alpha
    prm = dict(_POW_PRM)
    if l2:
        prm["optimality_norm"] = NORM_L2
    return p, prm, {"x": [2 * alpha, 2 * om, (2 * alpha) ** alpha * (2 * om) ** om], "tol": 2e-5, "nonzero_iters": True}


def pow_diag_q():
    """test/test_power_cone.c:196-209: min sum w_i (x_i - c_i)^2 / 2 over the
    power cone (a = 0.7, no rows), center (1.5, -0.4, -2.2), weights
    (0.3, 2, 5).  Expected (3.427365210244501, 0.4816579589566281,
    -1.902365192823554) (tol 2e-4)."""
    center, w = np.array([1.5, -0.4, -2.2]), np.array([0.3, 2.0, 5.0])
    A = CsrMatrix(0, 3, np.array([0]), np.zeros(0, np.int32), np.zeros(0))
    Q = CsrMatrix(3, 3, np.array([0, 1, 2, 3]), np.array([0, 1, 2]), w)
    p = Problem(c=-w * center, A=A, Q=Q, var_lb=np.full(3, -np.inf), var_ub=np.full(3, np.inf),
                cones=[Cone(CONE_POWER, 0, 1, alpha=0.7)])
    return p, dict(_POW_PRM), {"x": [3.427365210244501, 0.4816579589566281, -1.902365192823554], "tol": 2e-4}


_PSD_PRM = {"use_cone_preserving_scaling": False, "termination_evaluation_frequency": 10,
            "termination_criteria.eps_optimal_relative": 1e-7, "termination_criteria.eps_feasible_relative": 1e-7,
            "termination_criteria.iteration_limit": 1000000, "termination_criteria.time_sec_limit": 30.0}


def variable_psd():
    """test/test_psd_cones.c:24-68: min X_22 over svec(X) in PSD (order 2)
    with 100 X_11 = 100 and 0.01 svec_21 = 0.02 sqrt 2, i.e. X_21 = 2.
    Expected svec = (1, 2 sqrt 2, 4) (tol 2e-4, 2e-4, 3e-4), relative
    primal and dual residuals below 2e-6."""
    r2 = np.sqrt(2.0)
    A = CsrMatrix(2, 3, np.array([0, 1, 2]), np.array([0, 1]), np.array([100.0, 0.01]))
    b = np.array([100.0, 0.02 * r2])
    p = Problem(c=np.array([0.0, 0.0, 1.0]), A=A, con_lb=b, con_ub=b.copy(), var_lb=np.full(3, -np.inf),
                var_ub=np.full(3, np.inf), cones=[Cone(CONE_PSD, 0, 2)])
    return p, dict(_PSD_PRM), {"x": [1.0, 2.0 * r2, 4.0], "x_tol": [2e-4, 2e-4, 3e-4], "tol": 3e-4, "res": 2e-6}


def diagonal_q_psd():
    """test/test_psd_cones.c:120-180: min X_22^2 / 2 - 3 X_22 over svec(X) in
    PSD (order 2) with X_11 = 1, svec_21 = 2 sqrt 2 (diagonal Q: the inner
    BB solve).  Expected X_22 = 4 (tol 5e-4), relative residuals below
    3e-6."""
    r2 = np.sqrt(2.0)
    A = CsrMatrix(2, 3, np.array([0, 1, 2]), np.array([0, 1]), np.array([1.0, 1.0]))
    b = np.array([1.0, 2.0 * r2])
    Q = CsrMatrix(3, 3, np.array([0, 0, 0, 1]), np.array([2]), np.array([1.0]))
    p = Problem(c=np.array([0.0, 0.0, -3.0]), A=A, con_lb=b, con_ub=b.copy(), var_lb=np.full(3, -np.inf),
                var_ub=np.full(3, np.inf), Q=Q, cones=[Cone(CONE_PSD, 0, 2)])
    return p, dict(_PSD_PRM), {"xi": [(2, 4.0)], "tol": 5e-4, "res": 3e-6}


_AFF_PRM = {"termination_evaluation_frequency": 10, "termination_criteria.eps_optimal_relative": 1e-7,
            "termination_criteria.eps_feasible_relative": 1e-7, "termination_criteria.iteration_limit": 1000000,
            "termination_criteria.time_sec_limit": 30.0}


def _affine_one_variable(c, q, F_rows, g, cone, norm, preserving):
    """One variable x, F x + g in one affine cone (test/test_affine_cones.c:
    make_one_variable_problem / make_one_variable_quadratic_problem)."""
    m = len(F_rows)
    rp = np.cumsum([0] + [len(r) for r in F_rows])
    F = CsrMatrix(m, 1, rp, np.zeros(int(rp[-1]), np.int32), np.array([v for r in F_rows for v in r], float))
    Q = CsrMatrix(1, 1, np.array([0, 1]), np.array([0]), np.array([q])) if q else \
        CsrMatrix(1, 1, np.array([0, 0]), np.zeros(0, np.int32), np.zeros(0))
    p = Problem(c=np.array([c]), Q=Q, F=F, g=np.array(g, float), affine_cones=[cone])
    prm = dict(_AFF_PRM, optimality_norm=norm, use_cone_preserving_scaling=preserving)
    return p, prm


def affine_soc():
    """test/test_affine_cones.c:113-137: min x^2/2 - 2x s.t. (10x, 0, x + 9) in
    the SOC, i.e. 10 |x| <= x + 9.  Expected x = 1 (tol 2e-4), relative
    residuals below 2e-6 (L-inf norm, no cone-preserving scaling)."""
    p, prm = _affine_one_variable(-2.0, 1.0, [[10.0], [], [1.0]], [0.0, 0.0, 9.0], Cone(CONE_STANDARD_SOC, 0, 1),
                                  1, False)
    return p, prm, {"x": [1.0], "tol": 2e-4, "res": 2e-6}


def affine_rsoc():
    """test/test_affine_cones.c:191-215: max x s.t. (x, 1, 1) in the rotated
    SOC (x^2 <= 2).  Expected x = sqrt 2 (L2 norm)."""
    p, prm = _affine_one_variable(-1.0, 0.0, [[1.0], [], []], [0.0, 1.0, 1.0], Cone(CONE_ROTATED_SOC, 0, 1), 0, True)
    return p, prm, {"x": [np.sqrt(2.0)], "tol": 2e-4, "res": 2e-6}


def affine_exp():
    """test/test_affine_cones.c:139-163: max x s.t. (x, 1, 2) in K_exp
    (exp(x) <= 2).  Expected x = log 2 (L-inf norm)."""
    p, prm = _affine_one_variable(-1.0, 0.0, [[1.0], [], []], [0.0, 1.0, 2.0], Cone(CONE_EXPONENTIAL, 0, 1), 1, True)
    return p, prm, {"x": [np.log(2.0)], "tol": 2e-4, "res": 2e-6}


def affine_pow():
    """test/test_affine_cones.c:165-189: max x s.t. (1, 1, x) in K_0.3
    (|x| <= 1).  Expected x = 1 (L2 norm)."""
    p, prm = _affine_one_variable(-1.0, 0.0, [[], [], [1.0]], [1.0, 1.0, 0.0], Cone(CONE_POWER, 0, 1, alpha=0.3),
                                  0, True)
    return p, prm, {"x": [1.0], "tol": 2e-4, "res": 2e-6}


def affine_psd():
    """test/test_psd_cones.c:70-118: min x s.t. svec [[x, 1], [1, 1]] =
    (x, sqrt 2, 1) in PSD (x >= 1).  Expected x = 1 (tol 3e-4), relative
    residuals below 2e-6."""
    r2 = np.sqrt(2.0)
    F = CsrMatrix(3, 1, np.array([0, 1, 1, 1]), np.array([0]), np.array([1.0]))
    p = Problem(c=np.array([1.0]), F=F, g=np.array([0.0, r2, 1.0]), affine_cones=[Cone(CONE_PSD, 0, 2)])
    return p, dict(_PSD_PRM), {"x": [1.0], "tol": 3e-4, "res": 2e-6}


KNOWN_ANSWERS = {
    "affine_soc": affine_soc,
    "affine_rsoc": affine_rsoc,
    "affine_exp": affine_exp,
    "affine_pow": affine_pow,
    "affine_psd": affine_psd,
    "variable_psd": variable_psd,
    "diagonal_q_psd": diagonal_q_psd,
    "exp_cone_linear": exp_cone_linear,
    "pow_full_cone_0.2": lambda: pow_full_cone(0.2),
    "pow_full_cone_0.5": lambda: pow_full_cone(0.5),
    "pow_full_cone_0.8": lambda: pow_full_cone(0.8),
    "pow_full_cone_0.5_l2": lambda: pow_full_cone(0.5, l2=True),
    "pow_diag_q": pow_diag_q,
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
        e = np.asarray(expect["x"], dtype=float)
        t = np.asarray(expect.get("x_tol", [tol] * len(e)), dtype=float)
        assert np.all(np.abs(np.asarray(x) - e) <= t * (1 + np.abs(e))), (x, e)
    for i, v in expect.get("xi", []):
        assert abs(x[i] - v) <= tol * (1 + abs(v)), (i, x[i], v)
    if "res" in expect:
        assert res["relative_primal_residual"] < expect["res"], res["relative_primal_residual"]
        assert res["relative_dual_residual"] < expect["res"], res["relative_dual_residual"]
    if "y" in expect:
        np.testing.assert_allclose(res["y"], expect["y"], atol=tol * 10)
    if "obj" in expect:
        assert abs(res["primal_objective_value"] - expect["obj"]) <= 10 * tol * (1 + abs(expect["obj"]))
    if expect.get("nonzero_iters"):
        assert res["total_count"] > 0  # a feasible non-optimal start must not pass at iteration 0
    if expect.get("soc_kkt"):
        v, w, z = x
        assert abs(w - 4.0) <= tol * 5
        assert abs(v * v + w * w - z * z) <= tol
        assert abs((3.0 / v - 1.0) / 2.0 - (1.0 - 4.0 / z) / 2.0) <= 1e-4


# ---- infeasible instances (no reference test pins these; the GPU solver is
# checked against the oracle's restatement of the certificate logic,
# reference src/pdhg_core_op.cu:1296-1429 and src/utils.cu:230-280) ----------

def primal_infeasible_lp(seed=41, n=60, m=30):
    """A feasible box LP plus the row sum(x) >= 2 n + 5, which the box
    [-2, 2]^n cannot meet."""
    import scipy.sparse as sp
    from pdhcg_b200 import instances
    p = instances.box_lp(seed=seed, n=n, m=m)
    A = sp.vstack([p.A.to_scipy(), sp.csr_matrix(np.ones((1, n)))]).tocsr()
    return Problem(c=p.c, A=CsrMatrix.from_scipy(A), con_lb=np.concatenate([p.con_lb, [2.0 * n + 5]]),
                   con_ub=np.concatenate([p.con_ub, [np.inf]]), var_lb=p.var_lb, var_ub=p.var_ub)


def dual_infeasible(seed=42, n=60, m=30, diag_q=False):
    """A feasible box LP (or diagonal QP) whose first variable is free, in no
    row, has cost -1 and (QP) zero curvature: the objective is unbounded."""
    from pdhcg_b200 import instances
    p = instances.box_lp(seed=seed, n=n, m=m)
    A = p.A.to_scipy().tolil()
    A[:, 0] = 0.0
    A = A.tocsr()
    A.eliminate_zeros()
    lb, ub, c = p.var_lb.copy(), p.var_ub.copy(), p.c.copy()
    lb[0], ub[0], c[0] = -np.inf, np.inf, -1.0
    q = None
    if diag_q:
        qd = np.random.default_rng(seed).uniform(0.1, 1.0, n)
        qd[0] = 0.0
        q = CsrMatrix(n, n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), qd)
    return Problem(c=c, A=CsrMatrix.from_scipy(A), con_lb=p.con_lb, con_ub=p.con_ub, var_lb=lb, var_ub=ub, Q=q)


# expected status with an iteration limit of 2000.  The QP is unbounded too,
# but its certificate carries max |Q dx|, which the not yet converged
# curvature directions keep above eps_infeasible * |c . dx| while certificates
# are computed (k < 3 * termination_evaluation_frequency), so the reference's
# logic runs it to the limit.
INFEASIBLE = {
    "primal_infeasible_lp": (primal_infeasible_lp, "PRIMAL_INFEASIBLE"),
    "dual_infeasible_lp": (dual_infeasible, "DUAL_INFEASIBLE"),
    "dual_infeasible_qp": (lambda: dual_infeasible(diag_q=True), "ITERATION_LIMIT"),
}
