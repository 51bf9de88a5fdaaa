"""Loader for libpdhcg_b200.so (built in-tree by pdhcg_b200.build).

``load()`` builds the library when it is missing or stale and binds the
argument types of every C entry point.  There is no fallback: if the
library cannot be built or loaded, ``load()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import capi

_LIB = None
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Options(C.Structure):
    """pdhcg_b200_options_t (include/pdhcg_b200.h)."""
    _fields_ = [("precision", C.c_int), ("polish_threshold", C.c_double),
                ("has_initial_primal_weight", C.c_int), ("initial_primal_weight", C.c_double),
                ("use_graphs", C.c_int), ("time_steps", C.c_int), ("solution_on_device", C.c_int),
                ("has_initial_step_size", C.c_int), ("initial_step_size", C.c_double), ("reserved", C.c_int * 4)]


class Stats(C.Structure):
    """pdhcg_b200_stats_t (include/pdhcg_b200.h)."""
    _fields_ = [("setup_ms", C.c_double), ("loop_ms", C.c_double), ("step_kernel_ms", C.c_double),
                ("step_kernel_launches", C.c_longlong), ("kernel_launches", C.c_longlong),
                ("iterations", C.c_int), ("fp32_iterations", C.c_int), ("restarts", C.c_int),
                ("evaluations", C.c_int), ("step_bytes", C.c_double), ("spmv_bytes", C.c_double),
                ("host_copy_ms", C.c_double), ("upload_ms", C.c_double), ("result_ms", C.c_double),
                ("total_ms", C.c_double), ("primal_weight", C.c_double), ("step_size", C.c_double)]


class BatchOptions(C.Structure):
    """pdhcg_b200_batch_options_t (include/pdhcg_b200.h)."""
    _fields_ = [("shape", C.c_int), ("band_shape", C.c_int * 7)]


BATCH_SHAPES = 7


class BatchStats(C.Structure):
    """pdhcg_b200_batch_stats_t (include/pdhcg_b200.h)."""
    _fields_ = [("kernel_ms", C.c_double), ("total_ms", C.c_double), ("pack_ms", C.c_double),
                ("h2d_bytes", C.c_double), ("d2h_bytes", C.c_double), ("launches", C.c_int), ("batched", C.c_int),
                ("fallback", C.c_int), ("reserved", C.c_int * 5)]


class StepArgs(C.Structure):
    """pdhcg_b200_step_t (include/pdhcg_b200.h); every pointer is a device address."""
    _fields_ = [("n", C.c_int), ("m", C.c_int),
                ("A_row_ptr", C.c_void_p), ("A_col_ind", C.c_void_p), ("A_val", C.c_void_p),
                ("At_row_ptr", C.c_void_p), ("At_col_ind", C.c_void_p), ("At_val", C.c_void_p),
                ("c", C.c_void_p), ("var_lb", C.c_void_p), ("var_ub", C.c_void_p), ("q_diag", C.c_void_p),
                ("con_lb", C.c_void_p), ("con_ub", C.c_void_p), ("affine_offset", C.c_void_p),
                ("var_rescale", C.c_void_p), ("num_cones", C.c_int),
                ("cone_start", C.c_void_p), ("cone_vdim", C.c_void_p), ("cone_type", C.c_void_p),
                ("cone_alpha", C.c_void_p),
                ("tau", C.c_double), ("sigma", C.c_double), ("halpern_weight", C.c_double),
                ("reflection", C.c_double),
                ("x_init", C.c_void_p), ("x_cur", C.c_void_p), ("y_init", C.c_void_p), ("y_cur", C.c_void_p),
                ("x_pdhg", C.c_void_p), ("x_refl", C.c_void_p), ("y_pdhg", C.c_void_p), ("y_refl", C.c_void_p),
                ("Aty", C.c_void_p), ("Ax", C.c_void_p)]


EXPORTS = [
    # reference interface (include/pdhcg.h)
    "create_qp_problem", "set_start_values", "set_cone_fixed", "qcqp_to_socp_qp", "solve_qp_problem",
    "solve_qp_problem_distributed", "set_default_parameters", "pdhcg_result_free", "qp_problem_free",
    # additive entry points (include/pdhcg_b200.h)
    "pdhcg_b200_default_options", "pdhcg_b200_solve", "pdhcg_b200_last_stats", "pdhcg_b200_rescaling",
    "pdhcg_b200_csr_spmv",
    "pdhcg_b200_project_cones", "pdhcg_b200_pdhg_step", "pdhcg_b200_upload", "pdhcg_b200_solve_device",
    "pdhcg_b200_device_solution", "pdhcg_b200_device_problem_free", "pdhcg_b200_request_cancel",
    "cone_block_length", "pdhcg_b200_project_cones_noalloc", "pdhcg_b200_project_cone_sections",
    "pdhcg_b200_validate_fixed_sections", "pdhcg_b200_default_batch_options",
    "pdhcg_b200_solve_batch", "pdhcg_b200_batch_autotune", "pdhcg_b200_last_batch_stats", "pdhcg_b200_batch_release",
    "pdhcg_b200_mlp_create", "pdhcg_b200_mlp_free", "pdhcg_b200_mlp_num_params", "pdhcg_b200_mlp_get_params",
    "pdhcg_b200_mlp_set_params", "pdhcg_b200_mlp_predict", "pdhcg_b200_mlp_loss_grad", "pdhcg_b200_mlp_train",
    "read_mps_file",
]


def library_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "libpdhcg_b200.so")


def load(build: bool = True) -> C.CDLL:
    global _LIB
    if _LIB is not None:
        return _LIB
    if build:
        from .build import build as _build
        _build()
    path = library_path()
    if not os.path.exists(path):
        raise RuntimeError(f"libpdhcg_b200.so is missing at {path}; run python -m pdhcg_b200.build")
    lib = capi.bind_api(C.CDLL(path))
    P = C.POINTER
    lib.pdhcg_b200_default_options.restype = None
    lib.pdhcg_b200_default_options.argtypes = [P(Options)]
    lib.pdhcg_b200_solve.restype = P(capi.PdhcgResult)
    lib.pdhcg_b200_solve.argtypes = [P(capi.QpProblem), P(capi.PdhgParameters), P(Options)]
    lib.pdhcg_b200_last_stats.restype = C.c_int
    lib.pdhcg_b200_last_stats.argtypes = [P(Stats)]
    dp = P(C.c_double)
    lib.pdhcg_b200_rescaling.restype = C.c_int
    lib.pdhcg_b200_rescaling.argtypes = [P(capi.QpProblem), P(capi.PdhgParameters), dp, dp, dp]
    lib.pdhcg_b200_csr_spmv.restype = C.c_int
    lib.pdhcg_b200_csr_spmv.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]
    lib.pdhcg_b200_project_cones.restype = C.c_int
    lib.pdhcg_b200_project_cones.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
    lib.pdhcg_b200_project_cones_noalloc.restype = C.c_int
    lib.pdhcg_b200_project_cones_noalloc.argtypes = lib.pdhcg_b200_project_cones.argtypes
    lib.pdhcg_b200_pdhg_step.restype = C.c_int
    lib.pdhcg_b200_pdhg_step.argtypes = [P(StepArgs), C.c_void_p]
    lib.pdhcg_b200_upload.restype = C.c_void_p
    lib.pdhcg_b200_upload.argtypes = [P(capi.QpProblem)]
    lib.pdhcg_b200_solve_device.restype = P(capi.PdhcgResult)
    lib.pdhcg_b200_solve_device.argtypes = [C.c_void_p, P(capi.PdhgParameters), P(Options)]
    lib.pdhcg_b200_device_solution.restype = C.c_int
    lib.pdhcg_b200_device_solution.argtypes = [C.c_void_p, P(C.c_void_p), P(C.c_void_p), P(C.c_void_p)]
    lib.pdhcg_b200_device_problem_free.restype = None
    lib.pdhcg_b200_device_problem_free.argtypes = [C.c_void_p]
    lib.pdhcg_b200_default_batch_options.restype = None
    lib.pdhcg_b200_default_batch_options.argtypes = [P(BatchOptions)]
    lib.pdhcg_b200_solve_batch.restype = C.c_int
    lib.pdhcg_b200_solve_batch.argtypes = [C.c_int, P(P(capi.QpProblem)), P(capi.PdhgParameters), P(BatchOptions),
                                           P(P(capi.PdhcgResult))]
    lib.pdhcg_b200_batch_autotune.restype = C.c_int
    lib.pdhcg_b200_batch_autotune.argtypes = [C.c_int, P(P(capi.QpProblem)), P(capi.PdhgParameters),
                                              P(BatchOptions), P(C.c_double)]
    lib.pdhcg_b200_last_batch_stats.restype = C.c_int
    lib.pdhcg_b200_last_batch_stats.argtypes = [P(BatchStats)]
    lib.pdhcg_b200_batch_release.restype = None
    lib.pdhcg_b200_batch_release.argtypes = []
    fp = P(C.c_float)
    lib.pdhcg_b200_mlp_create.restype = C.c_void_p
    lib.pdhcg_b200_mlp_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong]
    lib.pdhcg_b200_mlp_free.restype = None
    lib.pdhcg_b200_mlp_free.argtypes = [C.c_void_p]
    lib.pdhcg_b200_mlp_num_params.restype = C.c_longlong
    lib.pdhcg_b200_mlp_num_params.argtypes = [C.c_void_p]
    lib.pdhcg_b200_mlp_get_params.restype = C.c_int
    lib.pdhcg_b200_mlp_get_params.argtypes = [C.c_void_p, fp]
    lib.pdhcg_b200_mlp_set_params.restype = C.c_int
    lib.pdhcg_b200_mlp_set_params.argtypes = [C.c_void_p, fp]
    lib.pdhcg_b200_mlp_predict.restype = C.c_int
    lib.pdhcg_b200_mlp_predict.argtypes = [C.c_void_p, C.c_int, fp, fp, fp]
    lib.pdhcg_b200_mlp_loss_grad.restype = C.c_int
    lib.pdhcg_b200_mlp_loss_grad.argtypes = [C.c_void_p, C.c_int, fp, fp, fp, P(C.c_double), fp]
    lib.pdhcg_b200_mlp_train.restype = C.c_int
    lib.pdhcg_b200_mlp_train.argtypes = [C.c_void_p, C.c_int, fp, fp, fp, C.c_int, C.c_int, C.c_float,
                                         P(C.c_double)]
    lib.pdhcg_b200_request_cancel.restype = None
    lib.pdhcg_b200_request_cancel.argtypes = [C.c_int]
    _LIB = lib
    return lib


def default_options(**kw) -> Options:
    lib = load()
    o = Options()
    lib.pdhcg_b200_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def last_stats() -> dict:
    lib = load()
    s = Stats()
    lib.pdhcg_b200_last_stats(C.byref(s))
    return {f: getattr(s, f) for f, _ in Stats._fields_ if f != "reserved"}


def solve(p: capi.Problem, params: dict | None = None, options: Options | None = None) -> dict:
    """Build ``p`` with create_qp_problem and solve it on the current device."""
    lib = load()
    prob, keep = capi.build(lib, p)
    if not prob:
        raise ValueError("create_qp_problem rejected the problem")
    prm = capi.default_params(lib, **(params or {}))
    try:
        r = lib.pdhcg_b200_solve(prob, C.byref(prm), C.byref(options) if options is not None else None)
        if not r:
            raise RuntimeError("solve failed (see stderr)")
        m = 0 if p.A is None else p.A.m
        out = capi.result_dict(r, p.n, max(m, 1) if m == 0 else m)
        lib.pdhcg_result_free(r)
    finally:
        lib.qp_problem_free(prob)
    return out


def solve_batch(problems, params: dict | None = None, shape: int = -1) -> list:
    """Build every problem with create_qp_problem and solve them together with
    pdhcg_b200_solve_batch; returns one result dict per problem."""
    lib = load()
    built = [capi.build(lib, p) for p in problems]
    if any(not b[0] for b in built):
        raise ValueError("create_qp_problem rejected a problem")
    arr = (C.POINTER(capi.QpProblem) * len(built))(*[b[0] for b in built])
    prm = capi.default_params(lib, **(params or {}))
    opts = BatchOptions()
    lib.pdhcg_b200_default_batch_options(C.byref(opts))
    opts.shape = shape
    res = (C.POINTER(capi.PdhcgResult) * len(built))()
    try:
        rc = lib.pdhcg_b200_solve_batch(len(built), arr, C.byref(prm), C.byref(opts), res)
        if rc != 0:
            raise RuntimeError("pdhcg_b200_solve_batch failed (see stderr)")
        out = []
        for p, r in zip(problems, res):
            out.append(capi.result_dict(r, p.n, p.A.m))
            lib.pdhcg_result_free(r)
    finally:
        for b in built:
            lib.qp_problem_free(b[0])
    return out
