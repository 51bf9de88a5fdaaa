"""pdhcg_b200_project_cones_noalloc (scratch in a file-scope device array)
against pdhcg_b200_project_cones (stream-ordered temporary) through the C
ABI.  Both run the same projection kernel on the same data, so the results
must agree to 1e-12 relative (they are expected to be bit-identical).
Different calls in a row check that a call sees none of the previous
call's scratch; SOC, rotated-SOC, exponential and power blocks (with their
exponents) all go through the shared array.  The device's free memory and
the default memory pool's reservation are read before and after each
no-allocation call and must be unchanged."""
import ctypes as C

import numpy as np
import pytest

from pdhcg_b200 import capi

pytestmark = pytest.mark.gpu

NOALLOC_MAX_CONES = 65536  # PDHCG_B200_NOALLOC_MAX_CONES in include/pdhcg_b200.h


def _dev(a, dtype):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _case(seed, shapes, weighted):
    rng = np.random.default_rng(seed)
    blocks, st = [], 0
    for L, t in shapes:
        blocks.append((st, L, t))
        st += L
    x = rng.standard_normal(st) * 2
    d = rng.uniform(0.5, 2.0, st)
    q = rng.uniform(0.0, 2.0, st) if weighted else None
    return blocks, x, d, q


def _device_args(blocks, x, d, q, alpha=None):
    """Device copies of one call's arguments (allocated before the call)."""
    starts = _dev([b[0] for b in blocks], np.int32)
    vdims = _dev([b[1] - 2 for b in blocks], np.int32)
    types = _dev([b[2] for b in blocks], np.int32)
    al = _dev(alpha, np.float64) if alpha is not None else None
    xd, dd, qd = _dev(x, np.float64), _dev(d, np.float64), (_dev(q, np.float64) if q is not None else None)
    return starts, vdims, types, al, xd, dd, qd


def _call(fn, n, args, tau):
    starts, vdims, types, al, xd, dd, qd = args
    return fn(n, _ptr(starts), _ptr(vdims), _ptr(types), _ptr(al), _ptr(xd), _ptr(dd), _ptr(qd), tau, None)


def _run(fn, blocks, x, d, q, tau, alpha=None):
    import torch
    args = _device_args(blocks, x, d, q, alpha)
    rc = _call(fn, len(blocks), args, tau)
    torch.cuda.synchronize()
    return rc, args[4].cpu().numpy()


def _device_memory():
    """(free bytes, bytes reserved and in use by the default memory pool) of
    the current device, through the CUDA runtime's own queries."""
    from cuda.bindings import runtime as rt
    err, free, _total = rt.cudaMemGetInfo()
    assert err == rt.cudaError_t.cudaSuccess
    err, dev = rt.cudaGetDevice()
    err, pool = rt.cudaDeviceGetDefaultMemPool(dev)
    assert err == rt.cudaError_t.cudaSuccess
    out = [free]
    for attr in (rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent,
                 rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh):
        err, v = rt.cudaMemPoolGetAttribute(pool, attr)
        assert err == rt.cudaError_t.cudaSuccess
        out.append(int(v))
    return tuple(out)


def test_noalloc_projection_matches_allocating_entry_point(lib):
    import torch
    E, P = capi.CONE_EXPONENTIAL, capi.CONE_POWER
    cases = [
        (_case(11, [(3, 1), (5, 0), (50, 1), (33, 1), (102, 0), (4, 0), (250, 1), (64, 0)] * 40, True), 0.37),
        # second call: fewer, shorter blocks and other types in other places
        (_case(12, [(7, 0), (12, 1), (3, 1)] * 25, False), 1.3),
        # exponential and power blocks, which read cone_alpha, among SOC / RSOC blocks
        (_case(15, [(3, E), (3, P), (20, 1), (3, P), (9, 0), (3, E)] * 30, True), 0.8),
    ]
    for (blocks, x, d, q), tau in cases:
        alpha = np.where(np.array([b[2] for b in blocks]) == P,
                         np.random.default_rng(len(blocks)).uniform(0.2, 0.8, len(blocks)), 0.0)
        rc_ref, ref = _run(lib.pdhcg_b200_project_cones, blocks, x, d, q, tau, alpha)
        # a first call loads the entry point's kernels (lazy module loading
        # takes device memory for their code); it must give the same answer
        rc_w, warm = _run(lib.pdhcg_b200_project_cones_noalloc, blocks, x, d, q, tau, alpha)
        assert rc_w == 0
        np.testing.assert_allclose(warm, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
        # every argument of the measured call is on the device before the
        # call, so the device's free memory and the default pool's
        # reservation must not move across it
        args = _device_args(blocks, x, d, q, alpha)
        torch.cuda.synchronize()
        before = _device_memory()
        rc_na = _call(lib.pdhcg_b200_project_cones_noalloc, len(blocks), args, tau)
        torch.cuda.synchronize()
        after = _device_memory()
        got = args[4].cpu().numpy()
        assert rc_ref == 0 and rc_na == 0
        assert before == after, (before, after)
        assert not np.array_equal(ref, x)  # the projection did something
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_noalloc_projection_limits_and_errors(lib):
    # beyond the scratch size: refused before any launch or pointer use
    assert lib.pdhcg_b200_project_cones_noalloc(NOALLOC_MAX_CONES + 1, None, None, None, None, None, None, None,
                                                1.0, None) == -4
    # a cone type without a projection: -3, x untouched
    blocks, x, d, _ = _case(13, [(3, 1), (3, capi.CONE_PSD)], False)
    rc, got = _run(lib.pdhcg_b200_project_cones_noalloc, blocks, x, d, None, 1.0)
    assert rc == -3
    np.testing.assert_array_equal(got, x)
    # a block longer than 256 slots: -2, as pdhcg_b200_project_cones
    blocks, x, d, _ = _case(14, [(300, 1)], False)
    rc, got = _run(lib.pdhcg_b200_project_cones_noalloc, blocks, x, d, None, 1.0)
    assert rc == -2
    rc_ref, _ = _run(lib.pdhcg_b200_project_cones, blocks, x, d, None, 1.0)
    assert rc_ref == -2
