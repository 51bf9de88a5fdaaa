"""Host-side failure paths of a running solve, made on the host (no GPU
fault, trap or hang is involved):

- the time limit (reference check_termination_criteria, src/utils.cu:279-288)
  stops a solve that cannot reach its tolerance, with TIME_LIMIT;
- the reference's cancel flag g_pdhcg_cancel_request (src/pdhcg.c:31, read
  at every evaluation, src/utils.cu:252-256) set by another host thread
  while a solve runs stops it with USER_INTERRUPT;
- NaN in the objective, the bounds or a matrix, or an infinite objective
  or matrix entry, gives NULL (with a message) instead of a run that
  would iterate on NaN until a limit;
- the warm start is projected onto the variable box before the first
  iteration, and a start that is already optimal terminates at iteration
  0 (a port of the reference's test/test_initial_box_projection.c:21-82).
"""
import ctypes as C
import threading
import time

import numpy as np
import pytest

from pdhcg_b200 import capi, instances
from pdhcg_b200.capi import CsrMatrix, Problem

pytestmark = pytest.mark.gpu

NEVER = {"termination_criteria.eps_optimal_relative": 0.0, "termination_criteria.eps_feasible_relative": 0.0,
         "termination_criteria.iteration_limit": 2_000_000_000}


def _solve(lib, p, over):
    prob, keep = capi.build(lib, p)
    assert prob
    prm = capi.default_params(lib, **over)
    r = lib.solve_qp_problem(prob, C.byref(prm))
    try:
        if not r:
            return None
        m = p.A.m if p.A is not None else 0
        d = capi.result_dict(r, p.n, max(m, 1))
        lib.pdhcg_result_free(r)
        return d
    finally:
        lib.qp_problem_free(prob)


def test_time_limit_stops_a_solve_that_cannot_converge(lib):
    p = instances.soc_qp(seed=2, scale=0.05)  # n = 5e4 in 1000 SOC blocks
    t0 = time.perf_counter()
    d = _solve(lib, p, {**NEVER, "termination_criteria.time_sec_limit": 0.3})
    wall = time.perf_counter() - t0
    assert d["status"] == "TIME_LIMIT"
    assert d["cumulative_time_sec"] >= 0.3
    assert wall < 10.0  # checked at every evaluation, so it stops within a few evaluations
    assert d["total_count"] > 0
    assert np.all(np.isfinite(d["x"])) and np.all(np.isfinite(d["y"]))


def test_cancel_flag_set_by_another_thread_stops_a_running_solve(lib):
    flag = C.c_int.in_dll(lib, "g_pdhcg_cancel_request")  # the reference's exported sig_atomic_t
    flag.value = 0
    p = instances.soc_qp(seed=2, scale=0.05)
    out = {}

    def run():  # ctypes releases the GIL for the call
        out["d"] = _solve(lib, p, {**NEVER, "termination_criteria.time_sec_limit": 60.0})

    th = threading.Thread(target=run)
    t0 = time.perf_counter()
    th.start()
    try:
        time.sleep(1.0)
        assert th.is_alive(), "the solve ended before the flag was set"
        flag.value = 1
        th.join(timeout=30.0)
        assert not th.is_alive(), "the solve did not stop after the flag was set"
    finally:
        flag.value = 0
        th.join()
    wall = time.perf_counter() - t0
    d = out["d"]
    assert d["status"] == "USER_INTERRUPT"
    assert wall < 30.0
    assert d["total_count"] > 0
    # the flag is cleared by the caller: the next solve runs normally
    d2 = _solve(lib, instances.box_lp(seed=4), {"termination_criteria.iteration_limit": 100000})
    assert d2["status"] == "OPTIMAL"


def _with(p, field, index, value):
    a = getattr(p, field).copy()
    a[index] = value
    setattr(p, field, a)
    return p


def _with_matrix_value(p, name, index, value):
    M = getattr(p, name)
    val = M.val.copy()
    val[index] = value
    setattr(p, name, CsrMatrix(M.m, M.n, M.row_ptr, M.col_ind, val))
    return p


@pytest.mark.parametrize("case", ["c_nan", "c_inf", "con_lb_nan", "var_ub_nan", "A_nan", "A_inf", "Q_nan"])
def test_nan_or_infinite_input_gives_null(lib, case):
    p = instances.diag_qp(seed=6)
    if case == "c_nan":
        _with(p, "c", 3, np.nan)
    elif case == "c_inf":
        _with(p, "c", 3, np.inf)
    elif case == "con_lb_nan":
        _with(p, "con_lb", 2, np.nan)
    elif case == "var_ub_nan":
        _with(p, "var_ub", 5, np.nan)
    elif case == "A_nan":
        _with_matrix_value(p, "A", 7, np.nan)
    elif case == "A_inf":
        _with_matrix_value(p, "A", 7, -np.inf)
    else:
        _with_matrix_value(p, "Q", 1, np.nan)
    prob, keep = capi.build(lib, p)
    if prob:  # the builder copies the values as given; the solve refuses them
        prm = capi.default_params(lib, **{"termination_criteria.iteration_limit": 1000})
        assert not lib.solve_qp_problem(prob, C.byref(prm))
        lib.qp_problem_free(prob)
    # an infinite bound is "no bound", not an error
    q = instances.diag_qp(seed=6)
    _with(q, "var_ub", 5, np.inf)
    assert _solve(lib, q, {"termination_criteria.iteration_limit": 100000})["status"] == "OPTIMAL"


def _one_variable(start):
    """min 0 x  s.t.  0 <= x <= 10 (one row), 1 <= x <= 2 (reference
    test/test_initial_box_projection.c:23-43)."""
    A = CsrMatrix(1, 1, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([1.0]))
    return Problem(c=np.zeros(1), A=A, con_lb=np.zeros(1), con_ub=np.full(1, 10.0), var_lb=np.ones(1),
                   var_ub=np.full(1, 2.0), primal_start=None if start is None else np.array([start]))


@pytest.mark.parametrize("start,expected", [(None, 1.0), (3.0, 2.0)])
def test_initial_box_projection(lib, oracle, start, expected):
    """No start: x = 0 projected onto [1, 2] is 1; start 3 (above the box)
    projects to 2.  Either point is optimal (c = 0, the row holds), so the
    solve stops at its first evaluation with total_count == 0 and x equal
    to the projection to 1e-12.  The oracle does the same."""
    p = _one_variable(start)
    d = _solve(lib, p, {})
    assert d["status"] == "OPTIMAL" and d["total_count"] == 0, (d["status"], d["total_count"])
    assert abs(d["x"][0] - expected) <= 1e-12, d["x"][0]
    prob, keep = capi.build(lib, p)
    r = oracle.oracle_solve(prob, C.byref(capi.default_params(lib)))
    o = capi.result_dict(r, 1, 1)
    oracle.oracle_result_free(r)
    lib.qp_problem_free(prob)
    assert o["status"] == "OPTIMAL" and o["total_count"] == 0
    assert abs(o["x"][0] - expected) <= 1e-12
