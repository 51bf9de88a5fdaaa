"""Batched solver (pdhcg_b200_solve_batch) against one solve_qp_problem per
instance on uneven MPC-style QPs (the batched workload at reduced count).

The batch runs in FP32 with FP64 accumulation and residuals, the single
solves in FP64, so both must reach the same status at the same tolerance;
objectives agree to 10 eps relative and the batch's own relative residuals
are below eps."""
import numpy as np
import pytest

from pdhcg_b200 import instances, native

pytestmark = pytest.mark.gpu

EPS = 1e-5
PRM = {"termination_criteria.eps_optimal_relative": EPS, "termination_criteria.eps_feasible_relative": EPS,
       "termination_criteria.iteration_limit": 200000, "termination_criteria.time_sec_limit": 60.0}


@pytest.mark.parametrize("shape", [-1, 0, 2, 4])
def test_batch_matches_single_solves(lib, shape):
    probs = instances.mpc_batch(seed=5, count=24, tmin=10, tmax=100)
    got = native.solve_batch(probs, PRM, shape=shape)
    for p, g in zip(probs, got):
        ref = native.solve(p, PRM)
        assert g["status"] == ref["status"] == "OPTIMAL"
        assert abs(g["primal_objective_value"] - ref["primal_objective_value"]) <= 10 * EPS * (
            1 + abs(ref["primal_objective_value"]))
        assert g["relative_primal_residual"] < EPS and g["relative_dual_residual"] < EPS
        assert g["relative_objective_gap"] < EPS
        # FP32 storage against FP64: ~5e-6 relative measured against the reference build
        np.testing.assert_allclose(g["x"], ref["x"], rtol=0, atol=1e-4 * (1 + np.abs(ref["x"]).max()))
        np.testing.assert_allclose(g["y"], ref["y"], rtol=0, atol=1e-4 * (1 + np.abs(ref["y"]).max()))


def test_batch_mixed_sizes_and_fallback(lib):
    """LP and QP instances together, plus one with a cone, which the batch
    hands to the single-instance solver."""
    probs = instances.mpc_batch(seed=6, count=6, tmin=5, tmax=30)
    probs.append(instances.box_lp(seed=31))
    probs.append(instances.conic_lp(seed=32))
    got = native.solve_batch(probs, PRM)
    for p, g in zip(probs, got):
        ref = native.solve(p, PRM)
        assert g["status"] == ref["status"] == "OPTIMAL"
        assert abs(g["primal_objective_value"] - ref["primal_objective_value"]) <= 10 * EPS * (
            1 + abs(ref["primal_objective_value"]))


def test_batch_autotune_picks_a_shape(lib):
    import ctypes as C
    from pdhcg_b200 import capi
    probs = instances.mpc_batch(seed=7, count=32, tmin=10, tmax=60)
    built = [capi.build(lib, p) for p in probs]
    arr = (C.POINTER(capi.QpProblem) * len(built))(*[b[0] for b in built])
    prm = capi.default_params(lib, **PRM)
    opts = native.BatchOptions()
    lib.pdhcg_b200_default_batch_options(C.byref(opts))
    ms = (C.c_double * native.BATCH_SHAPES)()
    assert lib.pdhcg_b200_batch_autotune(len(built), arr, C.byref(prm), C.byref(opts), ms) == 0
    assert 0 <= opts.shape < native.BATCH_SHAPES
    assert all(v > 0 for v in ms)
    for b in built:
        lib.qp_problem_free(b[0])
