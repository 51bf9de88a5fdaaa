"""Host side of the C boundary (CPU, no GPU): the library loads, exports every
symbol its headers declare, and builds problems exactly as the reference
does (reference src/pdhcg.c:35-666)."""
import ctypes as C
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp

from pdhcg_b200 import capi, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = []
    for h in ("pdhcg.h", "pdhcg_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b([a-z_0-9]+)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if not n.startswith("sizeof")))


def test_library_exports_every_declared_symbol(lib):
    declared = _declared_functions()
    assert "create_qp_problem" in declared and "pdhcg_b200_pdhg_step" in declared
    for name in declared:
        assert hasattr(lib, name), name
    for name in native.EXPORTS:
        assert name in declared, name


def test_cancel_flag_is_the_reference_symbol(lib):
    """The reference's Python binding declares g_pdhcg_cancel_request extern
    (reference python_bindings/_core_bindings.cpp:41) and writes it; the
    library must export that data symbol, and pdhcg_b200_request_cancel
    writes the same word."""
    flag = C.c_int.in_dll(lib, "g_pdhcg_cancel_request")
    assert flag.value == 0
    lib.pdhcg_b200_request_cancel(1)
    assert flag.value == 1
    lib.pdhcg_b200_request_cancel(0)
    assert flag.value == 0


def test_cone_block_length_matches_reference_rule(lib):
    """cone_block_length (reference src/cone_utils.c:26-45): 3 for EXP/POW,
    v_dim + 2 for (R)SOC, the triangle of v_dim for PSD, -1 when invalid."""
    types = np.array([capi.CONE_EXPONENTIAL, capi.CONE_POWER, capi.CONE_STANDARD_SOC,
                      capi.CONE_ROTATED_SOC, capi.CONE_PSD, capi.CONE_PSD, capi.CONE_STANDARD_SOC], dtype=np.int32)
    vdim = np.array([1, 1, 5, 0, 4, 0, -1], dtype=np.int32)
    blk = capi.ConeBlocks()
    blk.num_cones = len(types)
    blk.type = types.ctypes.data_as(C.POINTER(C.c_int))
    blk.v_dim = vdim.ctypes.data_as(C.POINTER(C.c_int))
    fn = lib.cone_block_length
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(capi.ConeBlocks), C.c_int]
    got = [fn(C.byref(blk), i) for i in range(len(types))]
    assert got == [3, 3, 7, 2, 10, -1, -1]
    assert fn(C.byref(blk), -1) == -1 and fn(C.byref(blk), len(types)) == -1
    assert fn(None, 0) == -1


def _problem_fields(P):
    p = P.contents
    n, m = p.num_variables, p.num_constraints
    out = {"n": n, "m": m, "rank": p.num_rank_lowrank_obj, "const": p.objective_constant,
           "nnzA": p.constraint_matrix_num_nonzeros, "nnzQ": p.objective_sparse_matrix_num_nonzeros,
           "nnzR": p.objective_lowrank_matrix_num_nonzeros,
           "nnzD": p.objective_lowrank_middle_matrix_num_nonzeros,
           "n_orig": p.num_original_variables}
    arr = lambda ptr, k: np.ctypeslib.as_array(ptr, shape=(k,)).copy() if (ptr and k > 0) else np.zeros(0)
    out["c"] = arr(p.objective_vector, n)
    out["l"] = arr(p.variable_lower_bound, n)
    out["u"] = arr(p.variable_upper_bound, n)
    out["lc"] = arr(p.constraint_lower_bound, m)
    out["uc"] = arr(p.constraint_upper_bound, m)
    out["g"] = arr(p.affine_cone_offset, m)
    A = p.constraint_matrix.contents
    out["A_rp"] = arr(A.row_ptr, m + 1)
    out["A_ci"] = arr(A.col_ind, out["nnzA"])
    out["A_v"] = arr(A.val, out["nnzA"])
    if p.objective_sparse_matrix:
        Q = p.objective_sparse_matrix.contents
        out["Q_rp"] = arr(Q.row_ptr, n + 1)
        out["Q_v"] = arr(Q.val, out["nnzQ"])
    if p.objective_lowrank_matrix and out["rank"] > 0:
        R = p.objective_lowrank_matrix.contents
        out["R_rp"] = arr(R.row_ptr, out["rank"] + 1)
        out["R_v"] = arr(R.val, out["nnzR"])
    k = p.cones.num_cones
    out["cones"] = [(p.cones.start_idx[i], p.cones.v_dim[i], p.cones.type[i]) for i in range(k)]
    return out


def _random_problem(seed, fmt_dense_R=False):
    rng = np.random.default_rng(seed)
    n, m = 40, 15
    A = sp.random(m, n, density=0.2, random_state=np.random.RandomState(seed), format="csr")
    A.data = rng.standard_normal(A.nnz)
    Q = sp.random(n, n, density=0.05, random_state=np.random.RandomState(seed + 1))
    Q = (Q + Q.T).tocsr()
    R = rng.standard_normal((3, n))
    D = np.diag(rng.uniform(0.5, 2.0, 3))
    lb = rng.uniform(-1, 0, n)
    ub = rng.uniform(0, 1, n)
    cones = [capi.Cone(capi.CONE_STANDARD_SOC, 30, 4), capi.Cone(capi.CONE_ROTATED_SOC, 36, 2)]
    for kk in cones:
        lb[kk.start:kk.start + kk.v_dim + 2] = -np.inf
        ub[kk.start:kk.start + kk.v_dim + 2] = np.inf
    return capi.Problem(c=rng.standard_normal(n), A=capi.CsrMatrix.from_scipy(A), con_lb=rng.uniform(-2, -1, m),
                        con_ub=rng.uniform(1, 2, m), var_lb=lb, var_ub=ub, Q=capi.CsrMatrix.from_scipy(Q),
                        R_dense=R if fmt_dense_R else None,
                        R=None if fmt_dense_R else capi.CsrMatrix.from_dense(R), D=capi.CsrMatrix.from_dense(D),
                        cones=cones, obj_const=1.5)


@pytest.mark.parametrize("seed,dense_R", [(1, False), (2, True)])
def test_create_qp_problem_matches_reference(lib, ref, seed, dense_R):
    p = _random_problem(seed, dense_R)
    mine, k1 = capi.build(lib, p)
    theirs, k2 = capi.build(ref, p)
    assert mine and theirs
    a, b = _problem_fields(mine), _problem_fields(theirs)
    assert a.keys() == b.keys()
    for key in a:
        if isinstance(a[key], np.ndarray):
            np.testing.assert_array_equal(a[key], b[key], err_msg=key)
        else:
            assert a[key] == b[key], key
    lib.qp_problem_free(mine)
    ref.qp_problem_free(theirs)


def test_default_parameters_match_reference(lib, ref):
    pa, pb = capi.PdhgParameters(), capi.PdhgParameters()
    lib.set_default_parameters(C.byref(pa))
    ref.set_default_parameters(C.byref(pb))
    for f, _ in capi.PdhgParameters._fields_:
        va, vb = getattr(pa, f), getattr(pb, f)
        if isinstance(va, C.Structure):
            for g, _ in va._fields_:
                if (f, g) in (("grid_size", "row_dims"), ("grid_size", "col_dims")):
                    continue  # left uninitialised by the reference
                assert getattr(va, g) == getattr(vb, g), (f, g)
        elif f != "permute_block_size":
            assert va == vb, f


def _csr_desc(rp, ci, v, m, n):
    keep = [np.asarray(rp, np.int32), np.asarray(ci, np.int32), np.asarray(v, np.float64)]
    d = capi.MatrixDesc()
    d.m, d.n, d.fmt = m, n, capi.MATRIX_CSR
    d.data.csr.nnz = len(keep[2])
    d.data.csr.row_ptr = keep[0].ctypes.data_as(C.POINTER(C.c_int))
    d.data.csr.col_ind = keep[1].ctypes.data_as(C.POINTER(C.c_int))
    d.data.csr.vals = keep[2].ctypes.data_as(C.POINTER(C.c_double))
    return d, keep


@pytest.mark.parametrize("case", ["bad_col", "bad_rowptr", "cone_box", "overlap"])
def test_invalid_inputs_return_null(lib, case):
    c = np.zeros(3)
    if case == "bad_col":
        d, keep = _csr_desc([0, 1], [5], [1.0], 1, 3)
        r = lib.create_qp_problem(c.ctypes.data_as(C.POINTER(C.c_double)), None, None, None, C.byref(d),
                                  None, None, None, None, None, 0, None, None, None, 0, None)
    elif case == "bad_rowptr":
        d, keep = _csr_desc([0, 2], [0], [1.0], 1, 3)
        r = lib.create_qp_problem(c.ctypes.data_as(C.POINTER(C.c_double)), None, None, None, C.byref(d),
                                  None, None, None, None, None, 0, None, None, None, 0, None)
    else:
        d, keep = _csr_desc([0, 1], [0], [1.0], 1, 3)
        cones = (capi.ConeSpec * 2)()
        cones[0].type, cones[0].start_idx, cones[0].v_dim = capi.CONE_STANDARD_SOC, 0, 1
        cones[1].type, cones[1].start_idx, cones[1].v_dim = capi.CONE_STANDARD_SOC, 0, 1
        lb = np.array([0.0, -np.inf, -np.inf]) if case == "cone_box" else np.full(3, -np.inf)
        r = lib.create_qp_problem(c.ctypes.data_as(C.POINTER(C.c_double)), None, None, None, C.byref(d),
                                  None, None, lb.ctypes.data_as(C.POINTER(C.c_double)), None, None,
                                  1 if case == "cone_box" else 2, cones, None, None, 0, None)
    assert not r


def test_set_cone_fixed_and_start_values(lib, ref):
    p = _random_problem(3)
    for L in (lib, ref):
        prob, keep = capi.build(L, p)
        assert L.set_cone_fixed(prob, 0, 1, 0.25) == 0
        assert L.set_cone_fixed(prob, 5, 0, 0.0) == -1
        assert L.set_cone_fixed(prob, 0, 99, 0.0) == -1
        assert L.set_cone_fixed(prob, 0, 0, float("inf")) == -1
        pp = prob.contents
        assert pp.primal_start[31] == 0.25 and pp.cones.is_fixed[31] == 1
        L.qp_problem_free(prob)


def test_distributed_entry_returns_null(lib):
    prm = capi.default_params(lib)
    assert not lib.solve_qp_problem_distributed(C.byref(prm), None)
