"""The command-line front end (pdhcg_b200.cli): the reference CLI's flags
map to the same pdhg_parameters_t fields (reference src/cli.c:212-350), and
a solve of an MPS file writes the reference CLI's three files (:79-154)."""
import os

import numpy as np
import pytest

from pdhcg_b200 import capi, cli

LP = """NAME LPSMALL
ROWS
 N  OBJ
 E  C1
COLUMNS
    X  OBJ  1.0  C1  1.0
    Y  OBJ  2.0  C1  1.0
RHS
    RHS  C1  1.0
ENDATA
"""


@pytest.fixture(scope="module")
def lib():
    from pdhcg_b200 import native
    return native.load()


def test_cli_flags_map_to_parameters(lib):
    args = cli.parser().parse_args([
        "p.mps", "out", "--time_limit", "12.5", "--iter_limit", "777", "--eps_opt", "1e-7", "--eps_feas", "2e-7",
        "--eps_infeas_detect", "3e-9", "--l_inf_ruiz_iter", "4", "--pock_chambolle_alpha", "0.5", "--sv_max_iter", "99",
        "--sv_tol", "1e-5", "--eval_freq", "50", "--opt_norm", "l2", "--inner_iter_limit", "12",
        "--inner_init_tol", "1e-2", "--inner_min_tol", "1e-8", "--no_bound_obj_rescaling", "--no_diag_precond",
        "--no_cone_preserving_scaling", "--artificial_restart_threshold", "0.4",
        "--sufficient_reduction_for_restart", "0.1", "--necessary_reduction_for_restart", "0.7",
        "--curtis_reid_iter", "3", "-v", "0"])
    p = cli.params_from_args(lib, args)
    tc = p.termination_criteria
    assert (tc.time_sec_limit, tc.iteration_limit, tc.eps_optimal_relative, tc.eps_feasible_relative,
            tc.eps_infeasible) == (12.5, 777, 1e-7, 2e-7, 3e-9)
    assert (p.l_inf_ruiz_iterations, p.pock_chambolle_alpha, p.sv_max_iter, p.sv_tol,
            p.termination_evaluation_frequency) == (4, 0.5, 99, 1e-5, 50)
    assert p.optimality_norm == capi.NORM_L2
    ip = p.inner_solver_parameters
    assert (ip.iteration_limit, ip.initial_tolerance, ip.min_tolerance) == (12, 1e-2, 1e-8)
    assert not p.bound_objective_rescaling and not p.diag_jacobi_precond and not p.use_cone_preserving_scaling
    assert p.has_pock_chambolle_alpha  # only --no_pock_chambolle clears it
    rp = p.restart_params
    assert (rp.artificial_restart_threshold, rp.sufficient_reduction_for_restart,
            rp.necessary_reduction_for_restart) == (0.4, 0.1, 0.7)
    assert p.curtis_reid_iterations == 3 and p.verbose == 0
    q = cli.params_from_args(lib, cli.parser().parse_args(["p.mps", "out", "--no_pock_chambolle"]))
    assert not q.has_pock_chambolle_alpha


def test_cli_instance_name():
    assert cli.instance_name("/data/afiro.mps.gz") == "afiro"
    assert cli.instance_name("qp.v2.qps") == "qp"


@pytest.mark.gpu
def test_cli_solves_an_mps_file(tmp_path):
    """test/test_c_api_working.c's LP (min x + 2y, x + y = 1, x, y >= 0) as an
    MPS file: OPTIMAL, x = (1, 0), y = 1, objective 1."""
    path = tmp_path / "lpsmall.mps"
    path.write_text(LP)
    out = tmp_path / "out"
    assert cli.main([str(path), str(out), "--eps_opt", "1e-6", "--eps_feas", "1e-6", "-v", "0"]) == 0
    summary = (out / "lpsmall_summary.txt").read_text().splitlines()
    assert summary[0] == "Termination Reason: OPTIMAL"
    fields = dict(line.split(": ", 1) for line in summary)
    assert abs(float(fields["Primal Objective Value"]) - 1.0) < 1e-4
    assert (fields["Rows"], fields["Columns"]) == ("1", "2")
    x = np.loadtxt(out / "lpsmall_primal_solution.txt")
    y = np.loadtxt(out / "lpsmall_dual_solution.txt", ndmin=1)
    np.testing.assert_allclose(x, [1.0, 0.0], atol=1e-4)
    np.testing.assert_allclose(y, [1.0], atol=1e-3)
    assert os.path.getsize(out / "lpsmall_primal_solution.txt") > 0
