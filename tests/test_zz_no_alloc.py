"""pdhcg_b200_project_cones_noalloc (scratch in a file-scope device array)
against pdhcg_b200_project_cones (stream-ordered temporary) through the C
ABI.  Both run the same projection kernel on the same data, so the results
must agree to 1e-12 relative (they are expected to be bit-identical).  Two
different calls in a row check that the second call sees none of the
first call's scratch."""
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


def _run(fn, blocks, x, d, q, tau):
    import torch
    starts = _dev([b[0] for b in blocks], np.int32)
    vdims = _dev([b[1] - 2 for b in blocks], np.int32)
    types = _dev([b[2] for b in blocks], np.int32)
    xd, dd, qd = _dev(x, np.float64), _dev(d, np.float64), (_dev(q, np.float64) if q is not None else None)
    rc = fn(len(blocks), _ptr(starts), _ptr(vdims), _ptr(types), None, _ptr(xd), _ptr(dd), _ptr(qd), tau, None)
    torch.cuda.synchronize()
    return rc, xd.cpu().numpy()


def test_noalloc_projection_matches_allocating_entry_point(lib):
    cases = [
        (_case(11, [(3, 1), (5, 0), (50, 1), (33, 1), (102, 0), (4, 0), (250, 1), (64, 0)] * 40, True), 0.37),
        # second call: fewer, shorter blocks and other types in other places
        (_case(12, [(7, 0), (12, 1), (3, 1)] * 25, False), 1.3),
    ]
    for (blocks, x, d, q), tau in cases:
        rc_ref, ref = _run(lib.pdhcg_b200_project_cones, blocks, x, d, q, tau)
        rc_na, got = _run(lib.pdhcg_b200_project_cones_noalloc, blocks, x, d, q, tau)
        assert rc_ref == 0 and rc_na == 0
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
