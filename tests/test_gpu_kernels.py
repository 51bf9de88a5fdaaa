"""Kernel-level parity through the C ABI (device pointers from torch):
SpMV against scipy, cone projections and one fused PDHG step against the
oracle.  FP64 throughout; tolerance 1e-12 relative (different summation
order only) except projections found by root finding (1e-9)."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from pdhcg_b200 import capi, instances, native

pytestmark = pytest.mark.gpu
_dp = C.POINTER(C.c_double)


def _dev(a, dtype=None):
    import torch
    t = torch.as_tensor(np.ascontiguousarray(a, dtype=dtype)).cuda()
    return t


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def test_csr_spmv_matches_scipy(lib):
    import torch
    rng = np.random.default_rng(0)
    for rows, cols, per in [(1000, 700, 8), (37, 5000, 300), (5000, 10, 3)]:
        M = instances.random_csr(rng, rows, cols, per)
        x = rng.standard_normal(cols)
        rp, ci, v, xd = _dev(M.row_ptr, np.int32), _dev(M.col_ind, np.int32), _dev(M.val), _dev(x)
        y = torch.zeros(rows, dtype=torch.float64, device="cuda")
        assert lib.pdhcg_b200_csr_spmv(rows, _ptr(rp), _ptr(ci), _ptr(v), _ptr(xd), _ptr(y), None) == 0
        torch.cuda.synchronize()
        np.testing.assert_allclose(y.cpu().numpy(), M.to_scipy() @ x, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("uniform_d", [False, True])
def test_cone_projection_matches_oracle(lib, oracle, weighted, uniform_d):
    import torch
    rng = np.random.default_rng(1 + 2 * weighted + uniform_d)
    blocks = []
    st = 0
    for L, t in [(3, 1), (5, 0), (50, 1), (33, 1), (102, 0), (4, 0), (250, 1), (64, 0)] * 3:
        blocks.append((st, L, t))
        st += L
    n = st
    x = rng.standard_normal(n) * 2
    d = np.ones(n) * 1.7 if uniform_d else rng.uniform(0.5, 2.0, n)
    if uniform_d:
        for s0, L, t in blocks:  # uniform within each block, varying across
            d[s0:s0 + L] = rng.uniform(0.5, 2.0)
    q = rng.uniform(0.0, 2.0, n) if weighted else None
    tau = 0.37
    expect = x.copy()
    for s0, L, t in blocks:
        blk = expect[s0:s0 + L].copy()
        dd = d[s0:s0 + L].copy()
        qq = q[s0:s0 + L].copy() if weighted else None
        oracle.oracle_project_cone_block(t, L - 2, 0.0, blk.ctypes.data_as(_dp), dd.ctypes.data_as(_dp),
                                         qq.ctypes.data_as(_dp) if weighted else None, tau)
        expect[s0:s0 + L] = blk
    starts = _dev([b[0] for b in blocks], np.int32)
    vdims = _dev([b[1] - 2 for b in blocks], np.int32)
    types = _dev([b[2] for b in blocks], np.int32)
    xd, dd_, qd = _dev(x), _dev(d), (_dev(q) if weighted else None)
    rc = lib.pdhcg_b200_project_cones(len(blocks), _ptr(starts), _ptr(vdims), _ptr(types), None, _ptr(xd),
                                      _ptr(dd_), _ptr(qd), tau, None)
    assert rc == 0
    torch.cuda.synchronize()
    got = xd.cpu().numpy()
    tol = 1e-12 if (uniform_d and not weighted) else 1e-9
    np.testing.assert_allclose(got, expect, rtol=tol, atol=tol * np.abs(expect).max())


@pytest.mark.parametrize("weighted", [False, True])
def test_exp_pow_projection_matches_oracle(lib, oracle, weighted):
    """Exponential and power blocks (one thread per block on the device)
    against the oracle's restatement of the reference's point projections:
    points inside, in the polar / opposite cone and in general position,
    power exponents across (0, 1).  Tolerance 1e-9 (math-library round-off
    through the Newton / bisection steps)."""
    import torch
    rng = np.random.default_rng(11 + weighted)
    nb = 600
    types = rng.choice([capi.CONE_EXPONENTIAL, capi.CONE_POWER], nb)
    alpha = rng.uniform(0.1, 0.9, nb)
    x = rng.standard_normal(3 * nb) * rng.choice([0.1, 1.0, 10.0], 3 * nb)
    x[0:30:3] = -np.abs(x[0:30:3])  # some x <= 0, y <= 0 points
    x[1:30:3] = -np.abs(x[1:30:3])
    d = np.repeat(rng.uniform(0.5, 2.0, nb), 3) * rng.uniform(0.8, 1.25, 3 * nb)
    q = rng.uniform(0.0, 2.0, 3 * nb) if weighted else None
    tau = 0.37
    expect = x.copy()
    for b in range(nb):
        blk = expect[3 * b:3 * b + 3].copy()
        dd = d[3 * b:3 * b + 3].copy()
        qq = q[3 * b:3 * b + 3].copy() if weighted else None
        oracle.oracle_project_cone_block(int(types[b]), 1, float(alpha[b]), blk.ctypes.data_as(_dp),
                                         dd.ctypes.data_as(_dp), qq.ctypes.data_as(_dp) if weighted else None, tau)
        expect[3 * b:3 * b + 3] = blk
    starts = _dev(np.arange(nb) * 3, np.int32)
    vdims = _dev(np.ones(nb), np.int32)
    tp = _dev(types, np.int32)
    al = _dev(alpha)
    xd, dd_, qd = _dev(x), _dev(d), (_dev(q) if weighted else None)
    rc = lib.pdhcg_b200_project_cones(nb, _ptr(starts), _ptr(vdims), _ptr(tp), _ptr(al), _ptr(xd), _ptr(dd_),
                                      _ptr(qd), tau, None)
    torch.cuda.synchronize()
    assert rc == 0
    got = xd.cpu().numpy()
    np.testing.assert_allclose(got, expect, rtol=1e-9, atol=1e-9 * np.abs(expect).max())


def _svec(X):
    n = X.shape[0]
    return np.array([X[r, c] if r == c else X[r, c] * np.sqrt(2.0) for c in range(n) for r in range(c, n)])


def test_psd_projection_matches_oracle(lib, oracle):
    """PSD blocks of orders 1..22 (svec packing) among SOC blocks, with
    spectra of mixed signs, all negative (projection 0) and all positive
    (projection = input), against the oracle's Jacobi restatement and numpy's
    eigh.  PSD blocks take no metric (d and q do not enter), as in the
    reference.  Tolerance 1e-10 relative to the block scale."""
    import torch
    rng = np.random.default_rng(31)
    blocks, parts, st = [], [], 0
    for k, order in enumerate([1, 2, 3, 4, 5, 7, 9, 12, 16, 22, 1, 2, 6]):
        M = rng.standard_normal((order, order))
        M = (M + M.T) / 2
        if k == 3:
            M = -M @ M.T - 0.1 * np.eye(order)  # negative definite: projects to 0
        if k == 4:
            M = M @ M.T + 0.1 * np.eye(order)  # positive definite: unchanged
        v = _svec(M)
        blocks.append((st, order, capi.CONE_PSD, M))
        parts.append(v)
        st += len(v)
        L = int(rng.integers(3, 40))  # an SOC block between PSD blocks
        blocks.append((st, L - 2, capi.CONE_STANDARD_SOC, None))
        parts.append(rng.standard_normal(L))
        st += L
    x = np.concatenate(parts)
    d = rng.uniform(0.5, 2.0, st)
    expect = x.copy()
    for s0, vd, t, M in blocks:
        L = vd * (vd + 1) // 2 if t == capi.CONE_PSD else vd + 2
        blk = expect[s0:s0 + L].copy()
        dd = d[s0:s0 + L].copy()
        oracle.oracle_project_cone_block(t, vd, 0.0, blk.ctypes.data_as(_dp), dd.ctypes.data_as(_dp), None, 0.0)
        expect[s0:s0 + L] = blk
        if M is not None:  # the oracle itself against eigh
            w, V = np.linalg.eigh(M)
            np.testing.assert_allclose(blk, _svec((V * np.maximum(w, 0)) @ V.T), atol=1e-11 * (1 + np.abs(M).max()))
    starts = _dev([b[0] for b in blocks], np.int32)
    vdims = _dev([b[1] for b in blocks], np.int32)
    types = _dev([b[2] for b in blocks], np.int32)
    xd, dd_ = _dev(x), _dev(d)
    rc = lib.pdhcg_b200_project_cones(len(blocks), _ptr(starts), _ptr(vdims), _ptr(types), None, _ptr(xd),
                                      _ptr(dd_), None, 0.0, None)
    torch.cuda.synchronize()
    assert rc == 0
    np.testing.assert_allclose(xd.cpu().numpy(), expect, rtol=1e-10, atol=1e-10 * np.abs(expect).max())


@pytest.mark.parametrize("orders", [(23, 32), (64,), (100,)])
def test_psd_projection_of_large_orders(lib, oracle, orders):
    """PSD blocks of orders 23 .. 100 (more svec slots than a warp's
    registers hold: projected through device scratch) among SOC blocks,
    spectra of mixed signs, against the oracle's Jacobi restatement and
    numpy's eigh: 1e-10 relative to the block scale."""
    import torch
    rng = np.random.default_rng(sum(orders))
    blocks, parts, st = [], [], 0
    for order in orders:
        M = rng.standard_normal((order, order))
        M = (M + M.T) / 2
        v = _svec(M)
        blocks.append((st, order, capi.CONE_PSD, M))
        parts.append(v)
        st += len(v)
        L = int(rng.integers(3, 40))
        blocks.append((st, L - 2, capi.CONE_STANDARD_SOC, None))
        parts.append(rng.standard_normal(L))
        st += L
    x = np.concatenate(parts)
    d = rng.uniform(0.5, 2.0, st)
    expect = x.copy()
    for s0, vd, t, M in blocks:
        L = vd * (vd + 1) // 2 if t == capi.CONE_PSD else vd + 2
        blk = expect[s0:s0 + L].copy()
        dd = d[s0:s0 + L].copy()
        oracle.oracle_project_cone_block(t, vd, 0.0, blk.ctypes.data_as(_dp), dd.ctypes.data_as(_dp), None, 0.0)
        expect[s0:s0 + L] = blk
        if M is not None:
            w, V = np.linalg.eigh(M)
            np.testing.assert_allclose(blk, _svec((V * np.maximum(w, 0)) @ V.T), atol=1e-10 * (1 + np.abs(M).max()))
    starts = _dev([b[0] for b in blocks], np.int32)
    vdims = _dev([b[1] for b in blocks], np.int32)
    types = _dev([b[2] for b in blocks], np.int32)
    xd, dd_ = _dev(x), _dev(d)
    rc = lib.pdhcg_b200_project_cones(len(blocks), _ptr(starts), _ptr(vdims), _ptr(types), None, _ptr(xd),
                                      _ptr(dd_), None, 0.0, None)
    torch.cuda.synchronize()
    assert rc == 0
    np.testing.assert_allclose(xd.cpu().numpy(), expect, rtol=1e-10, atol=1e-10 * np.abs(expect).max())


def test_cone_projection_rejects_unbuilt_cone_types(lib):
    """An unknown cone type is refused (-3) and x is left untouched."""
    import torch
    x = np.arange(8, dtype=np.float64)
    xd = _dev(x)
    starts, vdims = _dev([0, 3], np.int32), _dev([1, 3], np.int32)
    types = _dev([capi.CONE_STANDARD_SOC, 9], np.int32)
    d = _dev(np.ones(8))
    rc = lib.pdhcg_b200_project_cones(2, _ptr(starts), _ptr(vdims), _ptr(types), None, _ptr(xd), _ptr(d), None,
                                      1.0, None)
    torch.cuda.synchronize()
    assert rc == -3
    np.testing.assert_array_equal(xd.cpu().numpy(), x)


@pytest.mark.parametrize("with_q,with_cones", [(False, False), (True, False), (False, True), (True, True)])
def test_fused_step_matches_oracle(lib, oracle, with_q, with_cones):
    import torch
    p = instances.conic_lp(seed=21, with_q=with_q) if with_cones else (
        instances.diag_qp(seed=22) if with_q else instances.box_lp(seed=23))
    rng = np.random.default_rng(5)
    n, m = p.n, p.A.m
    A = p.A.to_scipy().tocsr()
    At = A.T.tocsr()
    At.sort_indices()
    q = p.Q.val.copy() if with_q else None
    vr = rng.uniform(0.5, 2.0, n)
    for k in p.cones:
        vr[k.start:k.start + k.v_dim + 2] = vr[k.start]
    x0, x, y0, y = (rng.standard_normal(n), rng.standard_normal(n), rng.standard_normal(m), rng.standard_normal(m))
    tau, sigma, w, rho = 0.3, 0.7, 5.0 / 6.0, 1.0
    lb = np.where(np.isfinite(p.var_lb), p.var_lb, -np.inf)
    ub = np.where(np.isfinite(p.var_ub), p.var_ub, np.inf)

    # oracle
    class OStep(C.Structure):
        _fields_ = [("n", C.c_int), ("m", C.c_int)] + [(f, C.c_void_p) for f in (
            "A_row_ptr", "A_col_ind", "A_val", "At_row_ptr", "At_col_ind", "At_val", "c", "var_lb", "var_ub",
            "q_diag", "con_lb", "con_ub", "affine_offset", "var_rescale")] + [
            ("num_cones", C.c_int)] + [(f, C.c_void_p) for f in ("cone_start", "cone_vdim", "cone_type", "cone_alpha")] + [
            (f, C.c_double) for f in ("tau", "sigma", "halpern_weight", "reflection")] + [
            (f, C.c_void_p) for f in ("x_init", "x_cur", "y_init", "y_cur", "x_pdhg", "x_refl", "y_pdhg", "y_refl",
                                      "Aty", "Ax")]

    host = {}

    def h(name, a, dt=np.float64):
        host[name] = np.array(a, dtype=dt, copy=True)  # the oracle updates x, y in place
        return host[name].ctypes.data

    cst = [k.start for k in p.cones]
    cvd = [k.v_dim for k in p.cones]
    cty = [k.type for k in p.cones]
    o = OStep()
    o.n, o.m = n, m
    o.A_row_ptr, o.A_col_ind, o.A_val = h("arp", A.indptr, np.int32), h("aci", A.indices, np.int32), h("av", A.data)
    o.At_row_ptr, o.At_col_ind, o.At_val = (h("trp", At.indptr, np.int32), h("tci", At.indices, np.int32),
                                            h("tv", At.data))
    o.c, o.var_lb, o.var_ub = h("c", p.c), h("lb", lb), h("ub", ub)
    o.q_diag = h("q", q) if with_q else None
    o.con_lb, o.con_ub, o.affine_offset = h("lc", p.con_lb), h("uc", p.con_ub), None
    o.var_rescale = h("vr", vr)
    o.num_cones = len(cst)
    o.cone_start, o.cone_vdim, o.cone_type = (h("cs", cst, np.int32), h("cv", cvd, np.int32),
                                              h("ct", cty, np.int32))
    o.cone_alpha = None
    o.tau, o.sigma, o.halpern_weight, o.reflection = tau, sigma, w, rho
    o.x_init, o.x_cur, o.y_init, o.y_cur = h("x0", x0), h("x", x), h("y0", y0), h("y", y)
    for f, k in (("x_pdhg", n), ("x_refl", n), ("y_pdhg", m), ("y_refl", m), ("Aty", n), ("Ax", m)):
        setattr(o, f, h(f, np.zeros(k)))
    oracle.oracle_pdhg_step.argtypes = [C.POINTER(OStep)]
    oracle.oracle_pdhg_step(C.byref(o))

    # device
    dev = {}

    def d(name, a, dt=np.float64):
        dev[name] = _dev(a, dt)
        return dev[name].data_ptr()

    s = native.StepArgs()
    s.n, s.m = n, m
    s.A_row_ptr, s.A_col_ind, s.A_val = d("arp", A.indptr, np.int32), d("aci", A.indices, np.int32), d("av", A.data)
    s.At_row_ptr, s.At_col_ind, s.At_val = (d("trp", At.indptr, np.int32), d("tci", At.indices, np.int32),
                                            d("tv", At.data))
    s.c, s.var_lb, s.var_ub = d("c", p.c), d("lb", lb), d("ub", ub)
    s.q_diag = d("q", q) if with_q else None
    s.con_lb, s.con_ub, s.affine_offset = d("lc", p.con_lb), d("uc", p.con_ub), None
    s.var_rescale = d("vr", vr)
    s.num_cones = len(cst)
    if cst:
        s.cone_start, s.cone_vdim, s.cone_type = d("cs", cst, np.int32), d("cv", cvd, np.int32), d("ct", cty, np.int32)
    s.tau, s.sigma, s.halpern_weight, s.reflection = tau, sigma, w, rho
    s.x_init, s.x_cur, s.y_init, s.y_cur = d("x0", x0), d("x", x), d("y0", y0), d("y", y)
    for f, k in (("x_pdhg", n), ("x_refl", n), ("y_pdhg", m), ("y_refl", m), ("Aty", n), ("Ax", m)):
        setattr(s, f, d(f, np.zeros(k)))
    assert lib.pdhcg_b200_pdhg_step(C.byref(s), None) == 0
    torch.cuda.synchronize()
    tol = 1e-9 if with_cones else 1e-12
    for key in ("x_pdhg", "x_refl", "x", "y_pdhg", "y"):
        np.testing.assert_allclose(dev[key].cpu().numpy(), host[key], rtol=tol, atol=tol, err_msg=key)
