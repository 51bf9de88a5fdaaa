"""ctypes mirror of the PDHCG C interface (include/pdhcg_types.h, include/pdhcg.h).

The same struct definitions bind any library that exports the reference's
C API: libpdhcg_b200.so (this package) and, in the tests, the reference
itself.  Problems are built from numpy / scipy.sparse data through the
library's own ``create_qp_problem`` (reference src/pdhcg.c:365-508), so the
host-side semantics (format conversion, validation, ownership) are exercised
exactly as a C caller would.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

# ---- enums (reference include/pdhcg_types.h:28-71, 250-257) -------------
TERMINATION_REASONS = [
    "UNSPECIFIED", "OPTIMAL", "PRIMAL_INFEASIBLE", "DUAL_INFEASIBLE",
    "INFEASIBLE_OR_UNBOUNDED", "TIME_LIMIT", "ITERATION_LIMIT",
    "USER_INTERRUPT", "FEAS_POLISH_SUCCESS",
]
OPTIMAL = 1
NORM_L2, NORM_LINF = 0, 1
CONE_ROTATED_SOC, CONE_STANDARD_SOC, CONE_EXPONENTIAL, CONE_POWER, CONE_PSD = 0, 1, 2, 3, 4
MATRIX_DENSE, MATRIX_CSR, MATRIX_CSC, MATRIX_COO = 0, 1, 2, 3

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class CsrComponent(C.Structure):
    _fields_ = [("row_ptr", _ip), ("col_ind", _ip), ("val", _dp)]


class ConeBlocks(C.Structure):
    _fields_ = [("num_cones", C.c_int), ("start_idx", _ip), ("v_dim", _ip), ("type", _ip),
                ("power_alpha", _dp), ("fixed_mask_size", C.c_int), ("is_fixed", C.POINTER(C.c_byte))]


class ConeSpec(C.Structure):
    _fields_ = [("type", C.c_int), ("start_idx", C.c_int), ("v_dim", C.c_int),
                ("power_alpha", C.c_double), ("is_fixed", C.c_void_p)]


class QpProblem(C.Structure):
    _fields_ = [
        ("num_variables", C.c_int), ("num_constraints", C.c_int), ("num_rank_lowrank_obj", C.c_int),
        ("variable_lower_bound", _dp), ("variable_upper_bound", _dp), ("objective_vector", _dp),
        ("objective_constant", C.c_double),
        ("constraint_matrix", C.POINTER(CsrComponent)), ("constraint_matrix_num_nonzeros", C.c_int),
        ("objective_sparse_matrix", C.POINTER(CsrComponent)), ("objective_sparse_matrix_num_nonzeros", C.c_int),
        ("objective_lowrank_matrix", C.POINTER(CsrComponent)), ("objective_lowrank_matrix_num_nonzeros", C.c_int),
        ("objective_lowrank_middle_matrix", C.POINTER(CsrComponent)),
        ("objective_lowrank_middle_matrix_num_nonzeros", C.c_int),
        ("constraint_lower_bound", _dp), ("constraint_upper_bound", _dp),
        ("affine_cone_offset", _dp), ("affine_cones", ConeBlocks),
        ("num_quadratic_constraints", C.c_int), ("quadratic_constraint_row_indices", _ip),
        ("quadratic_constraint_matrices", C.c_void_p), ("quadratic_constraint_matrix_num_nonzeros", _ip),
        ("cones", ConeBlocks), ("num_original_variables", C.c_int),
        ("primal_start", _dp), ("dual_start", _dp),
    ]


class RestartParameters(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "artificial_restart_threshold", "sufficient_reduction_for_restart",
        "necessary_reduction_for_restart", "k_p", "k_i", "k_d", "i_smooth")]


class TerminationCriteria(C.Structure):
    _fields_ = [("eps_optimal_relative", C.c_double), ("eps_feasible_relative", C.c_double),
                ("eps_feas_polish_relative", C.c_double), ("eps_infeasible", C.c_double),
                ("time_sec_limit", C.c_double), ("iteration_limit", C.c_int)]


class InnerSolverParameters(C.Structure):
    _fields_ = [("iteration_limit", C.c_int), ("initial_tolerance", C.c_double), ("min_tolerance", C.c_double)]


class GridSize(C.Structure):
    _fields_ = [("row_dims", C.c_int), ("col_dims", C.c_int), ("decided", C.c_bool)]


class PdhgParameters(C.Structure):
    _fields_ = [
        ("curtis_reid_iterations", C.c_int), ("l_inf_ruiz_iterations", C.c_int),
        ("has_pock_chambolle_alpha", C.c_bool), ("pock_chambolle_alpha", C.c_double),
        ("bound_objective_rescaling", C.c_bool), ("use_cone_preserving_scaling", C.c_bool),
        ("verbose", C.c_int), ("termination_evaluation_frequency", C.c_int),
        ("sv_max_iter", C.c_int), ("sv_tol", C.c_double),
        ("termination_criteria", TerminationCriteria), ("restart_params", RestartParameters),
        ("reflection_coefficient", C.c_double), ("feasibility_polishing", C.c_bool),
        ("optimality_norm", C.c_int), ("inner_solver_parameters", InnerSolverParameters),
        ("presolve", C.c_bool), ("diag_jacobi_precond", C.c_bool), ("default_cone_type", C.c_int),
        ("partition_method", C.c_int), ("permute_method", C.c_int), ("grid_size", GridSize),
        ("permute_block_size", C.c_int),
    ]


class PdhcgResult(C.Structure):
    _fields_ = [
        ("num_variables", C.c_int), ("num_constraints", C.c_int), ("num_nonzeros", C.c_int),
        ("num_reduced_variables", C.c_int), ("num_reduced_constraints", C.c_int),
        ("num_reduced_nonzeros", C.c_int),
        ("primal_solution", _dp), ("dual_solution", _dp), ("reduced_cost", _dp),
        ("total_count", C.c_int), ("total_inner_count", C.c_int),
        ("rescaling_time_sec", C.c_double), ("cumulative_time_sec", C.c_double),
        ("absolute_primal_residual", C.c_double), ("relative_primal_residual", C.c_double),
        ("absolute_dual_residual", C.c_double), ("relative_dual_residual", C.c_double),
        ("primal_objective_value", C.c_double), ("dual_objective_value", C.c_double),
        ("objective_gap", C.c_double), ("relative_objective_gap", C.c_double),
        ("max_primal_ray_infeasibility", C.c_double), ("max_dual_ray_infeasibility", C.c_double),
        ("primal_ray_linear_objective", C.c_double), ("dual_ray_objective", C.c_double),
        ("termination_reason", C.c_int), ("feasibility_polishing_time", C.c_double),
        ("feasibility_iteration", C.c_int), ("presolve_time", C.c_double), ("presolve_status", C.c_int),
    ]


class _MatDense(C.Structure):
    _fields_ = [("A", _dp)]


class _MatCSR(C.Structure):
    _fields_ = [("nnz", C.c_int), ("row_ptr", _ip), ("col_ind", _ip), ("vals", _dp)]


class _MatData(C.Union):
    _fields_ = [("dense", _MatDense), ("csr", _MatCSR), ("csc", _MatCSR), ("coo", _MatCSR)]


class MatrixDesc(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("fmt", C.c_int), ("zero_tolerance", C.c_double),
                ("data", _MatData)]


def bind_api(lib: C.CDLL) -> C.CDLL:
    """Declare argument / return types of the nine pdhcg.h functions on ``lib``."""
    P = C.POINTER
    lib.create_qp_problem.restype = P(QpProblem)
    lib.create_qp_problem.argtypes = [_dp, P(MatrixDesc), P(MatrixDesc), P(MatrixDesc), P(MatrixDesc),
                                      _dp, _dp, _dp, _dp, _dp, C.c_int, P(ConeSpec), P(MatrixDesc), _dp,
                                      C.c_int, P(ConeSpec)]
    lib.set_start_values.restype = None
    lib.set_start_values.argtypes = [P(QpProblem), _dp, _dp]
    lib.set_cone_fixed.restype = C.c_int
    lib.set_cone_fixed.argtypes = [P(QpProblem), C.c_int, C.c_int, C.c_double]
    lib.qcqp_to_socp_qp.restype = P(QpProblem)
    lib.qcqp_to_socp_qp.argtypes = [P(QpProblem), C.c_int]
    lib.solve_qp_problem.restype = P(PdhcgResult)
    lib.solve_qp_problem.argtypes = [P(QpProblem), P(PdhgParameters)]
    lib.solve_qp_problem_distributed.restype = P(PdhcgResult)
    lib.solve_qp_problem_distributed.argtypes = [P(PdhgParameters), P(QpProblem)]
    lib.set_default_parameters.restype = None
    lib.set_default_parameters.argtypes = [P(PdhgParameters)]
    lib.pdhcg_result_free.restype = None
    lib.pdhcg_result_free.argtypes = [P(PdhcgResult)]
    lib.qp_problem_free.restype = None
    lib.qp_problem_free.argtypes = [P(QpProblem)]
    if hasattr(lib, "read_mps_file"):
        lib.read_mps_file.restype = P(QpProblem)
        lib.read_mps_file.argtypes = [C.c_char_p]
    if hasattr(lib, "pdhcg_b200_validate_fixed_sections"):
        lib.pdhcg_b200_validate_fixed_sections.restype = C.c_int
        lib.pdhcg_b200_validate_fixed_sections.argtypes = [P(QpProblem)]
    return lib


def problem_arrays(prob) -> dict:
    """Copy the arrays of a qp_problem_t (e.g. from read_mps_file) into numpy:
    sizes, c, bounds, objective constant, A and Q as (row_ptr, col_ind, val)
    and the quadratic constraints as (row, (row_ptr, col_ind, val))."""
    p = prob.contents
    n, m = p.num_variables, p.num_constraints

    def vec(ptr, k):
        return np.ctypeslib.as_array(ptr, shape=(k,)).copy() if (ptr and k > 0) else np.zeros(0)

    def csr(M, rows, nnz):
        if not M:
            return None
        M = M.contents
        rp = np.ctypeslib.as_array(M.row_ptr, shape=(rows + 1,)).copy() if M.row_ptr else None
        ci = np.ctypeslib.as_array(M.col_ind, shape=(nnz,)).copy() if (M.col_ind and nnz > 0) else np.zeros(0, int)
        v = np.ctypeslib.as_array(M.val, shape=(nnz,)).copy() if (M.val and nnz > 0) else np.zeros(0)
        return rp, ci, v

    qcs = []
    mats = C.cast(p.quadratic_constraint_matrices, C.POINTER(C.POINTER(CsrComponent)))
    for k in range(p.num_quadratic_constraints):
        nnz = p.quadratic_constraint_matrix_num_nonzeros[k]
        qcs.append((p.quadratic_constraint_row_indices[k], csr(mats[k], n, nnz)))
    nc = p.cones.num_cones
    cones = {"start": [p.cones.start_idx[i] for i in range(nc)], "v_dim": [p.cones.v_dim[i] for i in range(nc)],
             "type": [p.cones.type[i] for i in range(nc)]}
    fixed = bytes(C.string_at(p.cones.is_fixed, p.cones.fixed_mask_size)) if p.cones.is_fixed else b""
    return {"n": n, "m": m, "cones": cones, "fixed": fixed, "primal_start": vec(p.primal_start, n),
            "c": vec(p.objective_vector, n), "obj_const": p.objective_constant,
            "var_lb": vec(p.variable_lower_bound, n), "var_ub": vec(p.variable_upper_bound, n),
            "con_lb": vec(p.constraint_lower_bound, m), "con_ub": vec(p.constraint_upper_bound, m),
            "A": csr(p.constraint_matrix, m, p.constraint_matrix_num_nonzeros),
            "Q": csr(p.objective_sparse_matrix, n, p.objective_sparse_matrix_num_nonzeros), "qc": qcs}


# ---- numpy-side problem description -----------------------------------

def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a, t=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


@dataclass
class CsrMatrix:
    """CSR triple with shape; ``from_scipy`` accepts any scipy.sparse matrix."""
    m: int
    n: int
    row_ptr: np.ndarray
    col_ind: np.ndarray
    val: np.ndarray

    @staticmethod
    def from_scipy(M) -> "CsrMatrix":
        M = M.tocsr()
        M.sort_indices()
        return CsrMatrix(M.shape[0], M.shape[1], _i32(M.indptr), _i32(M.indices), _f64(M.data))

    @staticmethod
    def from_dense(D) -> "CsrMatrix":
        import scipy.sparse as sp
        return CsrMatrix.from_scipy(sp.csr_matrix(np.asarray(D, dtype=np.float64)))

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col_ind, self.row_ptr), shape=(self.m, self.n))

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])


@dataclass
class Cone:
    type: int
    start: int
    v_dim: int
    alpha: float = 0.0


@dataclass
class Problem:
    """A QP in the reference's canonical form, held as numpy arrays."""
    c: np.ndarray
    A: Optional[CsrMatrix] = None
    con_lb: Optional[np.ndarray] = None
    con_ub: Optional[np.ndarray] = None
    var_lb: Optional[np.ndarray] = None
    var_ub: Optional[np.ndarray] = None
    Q: Optional[CsrMatrix] = None
    R: Optional[CsrMatrix] = None
    D: Optional[CsrMatrix] = None
    cones: Sequence[Cone] = field(default_factory=list)
    obj_const: float = 0.0
    primal_start: Optional[np.ndarray] = None
    dual_start: Optional[np.ndarray] = None
    R_dense: Optional[np.ndarray] = None  # optional dense R (k x n), passed as matrix_dense
    F: Optional[CsrMatrix] = None  # affine cone rows: F x + g in the affine cones
    g: Optional[np.ndarray] = None
    affine_cones: Sequence[Cone] = field(default_factory=list)  # blocks over the rows of F
    fixed: Sequence[tuple] = field(default_factory=list)  # (cone index, slot, value) for set_cone_fixed

    @property
    def n(self) -> int:
        return int(len(self.c))


def _desc(M: Optional[CsrMatrix], keep: list):
    if M is None:
        return None
    d = MatrixDesc()
    d.m, d.n, d.fmt, d.zero_tolerance = M.m, M.n, MATRIX_CSR, 0.0
    rp, ci, v = _i32(M.row_ptr), _i32(M.col_ind), _f64(M.val)
    keep += [rp, ci, v]
    d.data.csr.nnz = int(rp[-1])
    d.data.csr.row_ptr = _ptr(rp, C.c_int)
    d.data.csr.col_ind = _ptr(ci, C.c_int)
    d.data.csr.vals = _ptr(v)
    keep.append(d)
    return C.pointer(d)


def _dense_desc(D: np.ndarray, keep: list):
    d = MatrixDesc()
    arr = _f64(D)
    d.m, d.n, d.fmt, d.zero_tolerance = arr.shape[0], arr.shape[1], MATRIX_DENSE, 0.0
    d.data.dense.A = _ptr(arr)
    keep += [arr, d]
    return C.pointer(d)


def build(lib: C.CDLL, p: Problem):
    """Call ``lib.create_qp_problem`` on ``p``; returns (qp_problem_t*, keepalive)."""
    keep: list = []
    c = _f64(p.c)
    keep.append(c)
    arrs = [_f64(a) for a in (p.con_lb, p.con_ub, p.var_lb, p.var_ub)]
    keep += arrs
    oc = C.c_double(p.obj_const)
    cones = (ConeSpec * max(1, len(p.cones)))()
    for i, k in enumerate(p.cones):
        cones[i].type, cones[i].start_idx, cones[i].v_dim = k.type, k.start, k.v_dim
        cones[i].power_alpha, cones[i].is_fixed = k.alpha, None
    keep.append(cones)
    acones = (ConeSpec * max(1, len(p.affine_cones)))()
    for i, k in enumerate(p.affine_cones):
        acones[i].type, acones[i].start_idx, acones[i].v_dim = k.type, k.start, k.v_dim
        acones[i].power_alpha, acones[i].is_fixed = k.alpha, None
    keep.append(acones)
    g = _f64(p.g) if p.g is not None else None
    keep.append(g)
    Rd = _dense_desc(p.R_dense, keep) if p.R_dense is not None else _desc(p.R, keep)
    prob = lib.create_qp_problem(_ptr(c), _desc(p.Q, keep), Rd, _desc(p.D, keep), _desc(p.A, keep),
                                 _ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]), _ptr(arrs[3]), C.byref(oc),
                                 len(p.cones), cones if p.cones else None, _desc(p.F, keep),
                                 _ptr(g) if g is not None else None, len(p.affine_cones),
                                 acones if p.affine_cones else None)
    if prob and (p.primal_start is not None or p.dual_start is not None):
        ps, ds = _f64(p.primal_start), _f64(p.dual_start)
        keep += [ps, ds]
        lib.set_start_values(prob, _ptr(ps), _ptr(ds))
    for cone, slot, value in (p.fixed if prob else []):
        if lib.set_cone_fixed(prob, int(cone), int(slot), float(value)) != 0:
            lib.qp_problem_free(prob)
            return None, keep
    return prob, keep


def default_params(lib: C.CDLL, **overrides) -> PdhgParameters:
    """Parameters from ``lib.set_default_parameters`` with dotted overrides,
    e.g. ``default_params(lib, **{"termination_criteria.eps_optimal_relative": 1e-6})``."""
    prm = PdhgParameters()
    lib.set_default_parameters(C.byref(prm))
    prm.verbose = 0
    for k, v in overrides.items():
        obj = prm
        parts = k.split(".")
        for part in parts[:-1]:
            obj = getattr(obj, part)
        setattr(obj, parts[-1], v)
    return prm


def result_dict(res_ptr, n: int, m: int) -> dict:
    """Copy a pdhcg_result_t into a dict (arrays copied out of C memory)."""
    r = res_ptr.contents
    out = {f: getattr(r, f) for f, _ in PdhcgResult._fields_ if f not in ("primal_solution", "dual_solution", "reduced_cost")}
    out["status"] = TERMINATION_REASONS[r.termination_reason] if 0 <= r.termination_reason < len(TERMINATION_REASONS) else str(r.termination_reason)
    out["x"] = np.ctypeslib.as_array(r.primal_solution, shape=(n,)).copy() if n > 0 else np.zeros(0)
    out["y"] = np.ctypeslib.as_array(r.dual_solution, shape=(max(m, 1),)).copy()[:m] if m >= 0 else np.zeros(0)
    out["rc"] = np.ctypeslib.as_array(r.reduced_cost, shape=(n,)).copy() if n > 0 else np.zeros(0)
    out["rel_kkt"] = max(r.relative_primal_residual, r.relative_dual_residual, r.relative_objective_gap)
    return out
