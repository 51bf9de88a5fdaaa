"""Seeded problem generators shared by the golden-fixture script and the tests."""
import numpy as np
import scipy.sparse as sp

from pdhcg_b200.capi import CONE_ROTATED_SOC, CONE_STANDARD_SOC, Cone, CsrMatrix, Problem

SCALING_CASES = {
    "default": {"seed": 11, "params": {}},
    "curtis_reid": {"seed": 12, "params": {"curtis_reid_iterations": 5}},
    "no_cone_preserving": {"seed": 13, "params": {"use_cone_preserving_scaling": False}},
    "no_pock_chambolle": {"seed": 14, "params": {"has_pock_chambolle_alpha": False}},
    "pc_alpha_half": {"seed": 15, "params": {"pock_chambolle_alpha": 0.5}},
    "no_bound_obj": {"seed": 16, "params": {"bound_objective_rescaling": False, "l_inf_ruiz_iterations": 3}},
}


def scaling_problem(seed: int, n: int = 300, m: int = 120) -> Problem:
    """Random conic QP with SOC / RSOC blocks, boxes on free slots, diag Q."""
    rng = np.random.default_rng(seed)
    A = sp.random(m, n, density=0.05, random_state=np.random.RandomState(seed), format="csr")
    A.data = rng.standard_normal(A.nnz) * rng.choice([1e-2, 1.0, 1e2], size=A.nnz)
    cones = [Cone(CONE_STANDARD_SOC, 0, 10), Cone(CONE_ROTATED_SOC, 12, 3), Cone(CONE_STANDARD_SOC, 20, 60)]
    lb = rng.uniform(-1, 0, n)
    ub = rng.uniform(0, 1, n)
    for k in cones:
        lb[k.start:k.start + k.v_dim + 2] = -np.inf
        ub[k.start:k.start + k.v_dim + 2] = np.inf
    clb = rng.uniform(-2, -1, m)
    cub = rng.uniform(1, 2, m)
    eq = rng.random(m) < 0.3
    cub[eq] = clb[eq]
    return Problem(c=rng.standard_normal(n), A=CsrMatrix.from_scipy(A), con_lb=clb, con_ub=cub, var_lb=lb,
                   var_ub=ub, cones=cones, Q=CsrMatrix.from_scipy(sp.diags(rng.uniform(0.1, 1, n)).tocsr()))
