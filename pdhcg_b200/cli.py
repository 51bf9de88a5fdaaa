"""Command-line solve of a problem file, with the reference CLI's flags and
output files (reference src/cli.c:79-154 for the files, :212-350 for the
flags).

    python -m pdhcg_b200.cli [OPTIONS] <problem_file> <output_dir>

The problem file is MPS / QPS, plain or gzip (read by read_mps_file).  The
solve is solve_qp_problem of this library on the current GPU.  Three files
are written to output_dir, named after the file's base name up to its
first dot: <name>_summary.txt (termination reason, runtime, iteration
counts, objectives, residuals, sizes), <name>_primal_solution.txt and
<name>_dual_solution.txt (one value per line, printf "%.10g").

Flags map to pdhg_parameters_t as in the reference CLI.  Presolve and
feasibility polishing are accepted and have no effect (neither is part of
this library's solve); CBF files are refused.
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import sys

from . import capi, native

_FLOAT_FLAGS = {
    "time_limit": "termination_criteria.time_sec_limit",
    "eps_opt": "termination_criteria.eps_optimal_relative",
    "eps_feas": "termination_criteria.eps_feasible_relative",
    "eps_infeas_detect": "termination_criteria.eps_infeasible",
    "eps_feas_polish": "termination_criteria.eps_feas_polish_relative",
    "pock_chambolle_alpha": "pock_chambolle_alpha",
    "sv_tol": "sv_tol",
    "inner_init_tol": "inner_solver_parameters.initial_tolerance",
    "inner_min_tol": "inner_solver_parameters.min_tolerance",
    "artificial_restart_threshold": "restart_params.artificial_restart_threshold",
    "sufficient_reduction_for_restart": "restart_params.sufficient_reduction_for_restart",
    "necessary_reduction_for_restart": "restart_params.necessary_reduction_for_restart",
}
_INT_FLAGS = {
    "iter_limit": "termination_criteria.iteration_limit",
    "l_inf_ruiz_iter": "l_inf_ruiz_iterations",
    "sv_max_iter": "sv_max_iter",
    "eval_freq": "termination_evaluation_frequency",
    "inner_iter_limit": "inner_solver_parameters.iteration_limit",
    "curtis_reid_iter": "curtis_reid_iterations",
}
_OFF_FLAGS = {
    "no_pock_chambolle": "has_pock_chambolle_alpha",
    "no_bound_obj_rescaling": "bound_objective_rescaling",
    "no_diag_precond": "diag_jacobi_precond",
    "no_cone_preserving_scaling": "use_cone_preserving_scaling",
}


def parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="python -m pdhcg_b200.cli",
                                 description="Solve an MPS / QPS problem file on the GPU.")
    ap.add_argument("problem_file")
    ap.add_argument("output_dir")
    ap.add_argument("-v", "--verbose", type=int, default=None)
    for f in _FLOAT_FLAGS:
        ap.add_argument("--" + f, type=float, default=None)
    for f in _INT_FLAGS:
        ap.add_argument("--" + f, type=int, default=None)
    for f in _OFF_FLAGS:
        ap.add_argument("--" + f, action="store_true")
    ap.add_argument("-f", "--feasibility_polishing", action="store_true")
    ap.add_argument("--opt_norm", choices=["l2", "linf"], default=None)
    ap.add_argument("--presolve", type=int, default=None)
    ap.add_argument("--soc_form", choices=["rotated", "standard"], default=None)
    return ap


def params_from_args(lib, args) -> capi.PdhgParameters:
    """pdhg_parameters_t: defaults, then the flags given."""
    over = {}
    if args.verbose is not None:
        over["verbose"] = args.verbose
    for f, path in {**_FLOAT_FLAGS, **_INT_FLAGS}.items():
        v = getattr(args, f)
        if v is not None:
            over[path] = v
    for f, path in _OFF_FLAGS.items():
        if getattr(args, f):
            over[path] = False
    if args.feasibility_polishing:
        over["feasibility_polishing"] = True
    if args.opt_norm is not None:
        over["optimality_norm"] = capi.NORM_L2 if args.opt_norm == "l2" else capi.NORM_LINF
    if args.presolve is not None:
        over["presolve"] = args.presolve != 0
    if args.soc_form is not None:
        over["default_cone_type"] = capi.CONE_ROTATED_SOC if args.soc_form == "rotated" else capi.CONE_STANDARD_SOC
    prm = capi.default_params(lib, **over)
    if args.verbose is None:  # default_params silences the solve; the CLI keeps the library default
        d = capi.PdhgParameters()
        lib.set_default_parameters(C.byref(d))
        prm.verbose = d.verbose
    return prm


def instance_name(path: str) -> str:
    """Base name up to its first dot (reference extract_instance_name)."""
    return os.path.basename(path).split(".", 1)[0]


def write_outputs(r, n: int, m: int, output_dir: str, name: str) -> None:
    """The reference CLI's three files (save_solver_summary, save_solution)."""
    res = r.contents
    lines = [
        f"Termination Reason: {capi.TERMINATION_REASONS[res.termination_reason]}",
        f"Runtime (sec): {res.cumulative_time_sec:e}",
        f"Iterations Count: {res.total_count}",
    ]
    if res.total_inner_count > 0:
        lines.append(f"Inner Iterations Count: {res.total_inner_count}")
    lines += [
        f"Primal Objective Value: {res.primal_objective_value:e}",
        f"Dual Objective Value: {res.dual_objective_value:e}",
        f"Absolute Primal Residual: {res.absolute_primal_residual:e}",
        f"Absolute Dual Residual: {res.absolute_dual_residual:e}",
        f"Relative Primal Residual: {res.relative_primal_residual:e}",
        f"Relative Dual Residual: {res.relative_dual_residual:e}",
        f"Absolute Objective Gap: {res.objective_gap:e}",
        f"Relative Objective Gap: {res.relative_objective_gap:e}",
        f"Rows: {res.num_constraints}",
        f"Columns: {res.num_variables}",
        f"Nonzeros: {res.num_nonzeros}",
    ]
    with open(os.path.join(output_dir, name + "_summary.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    for suffix, ptr, k in (("_primal_solution.txt", res.primal_solution, n),
                           ("_dual_solution.txt", res.dual_solution, m)):
        with open(os.path.join(output_dir, name + suffix), "w") as f:
            f.write("".join("%.10g\n" % ptr[i] for i in range(k)))


def main(argv=None) -> int:
    args = parser().parse_args(argv)
    name = instance_name(args.problem_file)
    stem = args.problem_file[:-3] if args.problem_file.endswith(".gz") else args.problem_file
    if stem.endswith(".cbf"):
        print("CBF files are not supported by this library (MPS / QPS only).", file=sys.stderr)
        return 1
    lib = native.load()
    prob = lib.read_mps_file(args.problem_file.encode())
    if not prob:
        print("Failed to read or parse the file.", file=sys.stderr)
        return 1
    n, m = prob.contents.num_variables, prob.contents.num_constraints
    prm = params_from_args(lib, args)
    r = lib.solve_qp_problem(prob, C.byref(prm))
    if not r:
        print("Solver failed.", file=sys.stderr)
    else:
        os.makedirs(args.output_dir, exist_ok=True)
        write_outputs(r, n, m, args.output_dir, name)
        lib.pdhcg_result_free(r)
    lib.qp_problem_free(prob)
    return 0


if __name__ == "__main__":
    sys.exit(main())
