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


@pytest.mark.parametrize("shape", [-1, 0, 2, 4, 5, 6])
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
    # horizons 10..60 span several size bands, each tuned on its own
    tuned = [b for b in opts.band_shape if b != 0]
    assert len(tuned) >= 2 and all(1 <= b <= native.BATCH_SHAPES for b in tuned)
    res = (C.POINTER(capi.PdhcgResult) * len(built))()
    assert lib.pdhcg_b200_solve_batch(len(built), arr, C.byref(prm), C.byref(opts), res) == 0
    for p, r in zip(probs, res):
        assert capi.TERMINATION_REASONS[r.contents.termination_reason] == "OPTIMAL"
        lib.pdhcg_result_free(r)
    for b in built:
        lib.qp_problem_free(b[0])


def _solve_raw(lib, built, prm, shape):
    import ctypes as C
    from pdhcg_b200 import capi
    arr = (C.POINTER(capi.QpProblem) * len(built))(*[b[0] for b in built])
    opts = native.BatchOptions()
    lib.pdhcg_b200_default_batch_options(C.byref(opts))
    opts.shape = shape
    res = (C.POINTER(capi.PdhcgResult) * len(built))()
    rc = lib.pdhcg_b200_solve_batch(len(built), arr, C.byref(prm), C.byref(opts), res)
    out = []
    if rc == 0:
        for b, r in zip(built, res):
            n, m = r.contents.num_variables, r.contents.num_constraints
            out.append((np.ctypeslib.as_array(r.contents.primal_solution, (n,)).copy(),
                        np.ctypeslib.as_array(r.contents.dual_solution, (m,)).copy(),
                        np.ctypeslib.as_array(r.contents.reduced_cost, (n,)).copy(), r.contents.total_count))
            lib.pdhcg_result_free(r)
    st = native.BatchStats()
    lib.pdhcg_b200_last_batch_stats(C.byref(st))
    return rc, out, st


def test_batch_buffers_kept_between_calls(lib):
    """The staging and device buffers outlive a call and grow on demand: an
    instance gives bit-identical x, y, reduced cost and iteration count
    alone, in a small batch, in a larger one (the buffers grow), after
    pdhcg_b200_batch_release, and the transposes built on the device give
    the same iterates as the host-side counting sort did (checked through
    the single solves in test_batch_matches_single_solves)."""
    import ctypes as C
    from pdhcg_b200 import capi
    probs = instances.mpc_batch(seed=8, count=40, tmin=5, tmax=80)
    built = [capi.build(lib, p) for p in probs]
    prm = capi.default_params(lib, **PRM)
    try:
        rc, alone, st = _solve_raw(lib, built[:1], prm, 0)
        assert rc == 0 and st.batched == 1 and st.launches == 2  # A^T build + one class
        assert st.h2d_bytes > 0 and st.d2h_bytes >= 8 * (probs[0].n + probs[0].A.m)
        rc, small, _ = _solve_raw(lib, built[:8], prm, 0)
        assert rc == 0
        rc, large, st = _solve_raw(lib, built, prm, 0)
        assert rc == 0 and st.batched == 40
        lib.pdhcg_b200_batch_release()
        rc, again, _ = _solve_raw(lib, built[:8], prm, 0)
        assert rc == 0
        for got in (small[0], large[0], again[0]):
            for a, b in zip(alone[0][:3], got[:3]):
                assert np.array_equal(a, b)
            assert alone[0][3] == got[3]
        for i in range(8):
            for a, b in zip(small[i][:3], large[i][:3]):
                assert np.array_equal(a, b)
            for a, b in zip(small[i][:3], again[i][:3]):
                assert np.array_equal(a, b)
    finally:
        for b in built:
            lib.qp_problem_free(b[0])


def test_batch_rejects_bad_column_index_on_host(lib):
    """A column index outside [0, n) written into a built problem is caught
    while packing, before anything reaches the device."""
    import ctypes as C
    from pdhcg_b200 import capi
    probs = instances.mpc_batch(seed=9, count=3, tmin=5, tmax=10)
    built = [capi.build(lib, p) for p in probs]
    prm = capi.default_params(lib, **PRM)
    try:
        A = built[1][0].contents.constraint_matrix.contents
        saved = A.col_ind[2]
        A.col_ind[2] = probs[1].n + 7
        rc, out, _ = _solve_raw(lib, built, prm, -1)
        A.col_ind[2] = saved
        assert rc == -1 and out == []
        rc, out, _ = _solve_raw(lib, built, prm, -1)  # the same problems, repaired
        assert rc == 0 and len(out) == 3
    finally:
        for b in built:
            lib.qp_problem_free(b[0])
