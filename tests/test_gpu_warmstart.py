"""Learned warm start: the MLP's device forward/backward against the CPU
oracle (oracle/mlp_oracle.py), training on the GPU, and what the trained
network gains over cold starts on held-out instances of a parametric family
(every solve, warm or cold, must reach the same tolerance)."""
import ctypes as C
import importlib.util
import os

import numpy as np
import pytest

from pdhcg_b200 import native, warmstart

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _oracle():
    spec = importlib.util.spec_from_file_location("mlp_oracle", os.path.join(ROOT, "oracle", "mlp_oracle.py"))
    mo = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mo)
    return mo


def _fp(a):
    return np.ascontiguousarray(a, np.float32).ctypes.data_as(C.POINTER(C.c_float))


@pytest.mark.parametrize("dims,batch", [((5, 16, 4, 30), 7), ((32, 64, 8, 200), 64), ((7, 70, 3, 129), 33)])
def test_mlp_loss_and_gradient_match_oracle(lib, dims, batch):
    """Device loss and packed gradient equal the oracle's (same BF16 weights)
    to FP32 accumulation round-off: 1e-5 relative on the loss, 2e-4 of each
    block's largest entry on the gradient."""
    mo = _oracle()
    rng = np.random.default_rng(sum(dims))
    net = lib.pdhcg_b200_mlp_create(*dims, 7)
    try:
        npar = lib.pdhcg_b200_mlp_num_params(net)
        assert npar == sum(int(np.prod(s)) for s in mo.shapes(*dims))
        w = (rng.standard_normal(npar) * 0.3).astype(np.float32)
        assert lib.pdhcg_b200_mlp_set_params(net, _fp(w)) == 0
        x = rng.standard_normal((batch, dims[0])).astype(np.float32)
        t = rng.standard_normal((batch, dims[3])).astype(np.float32)
        tl = rng.standard_normal(batch).astype(np.float32)
        loss = C.c_double()
        g = np.zeros(npar, np.float32)
        assert lib.pdhcg_b200_mlp_loss_grad(net, batch, _fp(x), _fp(t), _fp(tl), C.byref(loss),
                                            g.ctypes.data_as(C.POINTER(C.c_float))) == 0
        lo, go, oo, lwo = mo.loss_grad(w.astype(np.float64), x.astype(np.float64), t, tl, *dims)
        assert abs(loss.value - lo) <= 1e-5 * abs(lo)
        o = 0
        for sh in mo.shapes(*dims):
            k = int(np.prod(sh))
            ref = go[o:o + k]
            np.testing.assert_allclose(g[o:o + k], ref, rtol=0, atol=2e-4 * max(np.abs(ref).max(), 1e-12))
            o += k
        out = np.zeros((batch, dims[3]), np.float32)
        lw = np.zeros(batch, np.float32)
        assert lib.pdhcg_b200_mlp_predict(net, batch, _fp(x), out.ctypes.data_as(C.POINTER(C.c_float)),
                                          lw.ctypes.data_as(C.POINTER(C.c_float))) == 0
        np.testing.assert_allclose(out, oo, rtol=1e-4, atol=1e-4 * np.abs(oo).max())
        np.testing.assert_allclose(lw, lwo, rtol=1e-4, atol=1e-4 * np.abs(lwo).max())
    finally:
        lib.pdhcg_b200_mlp_free(net)


def test_mlp_training_fits_a_low_rank_map(lib):
    """Adam on the GPU drives the loss of a smooth low-rank map down by 10x."""
    rng = np.random.default_rng(3)
    n_in, out, B = 16, 300, 512
    X = rng.standard_normal((B, n_in)).astype(np.float32)
    M = rng.standard_normal((n_in, 6)) @ rng.standard_normal((6, out)) / 4
    T = np.tanh(X @ M).astype(np.float32)
    TL = (X[:, 0] * 0.3).astype(np.float32)
    net = lib.pdhcg_b200_mlp_create(n_in, 128, 16, out, 11)
    try:
        l0, l1 = C.c_double(), C.c_double()
        assert lib.pdhcg_b200_mlp_loss_grad(net, B, _fp(X), _fp(T), _fp(TL), C.byref(l0), None) == 0
        assert lib.pdhcg_b200_mlp_train(net, B, _fp(X), _fp(T), _fp(TL), 300, 64, 2e-3, C.byref(l1)) == 0
        assert l1.value < 0.1 * l0.value
    finally:
        lib.pdhcg_b200_mlp_free(net)


def test_warm_start_gains_over_cold_start(lib):
    """A family of n = 2000: train on 96 cold solves, then 12 held-out
    instances solved three ways at eps 1e-6 -- cold, from the training
    targets' mean, and from the network's prediction -- all with the
    family's cached step size, so the forms differ only in their start.
    Every answer is OPTIMAL with objectives within 10 eps of the cold one,
    and the network's starts need fewer iterations on average than the cold
    ones."""
    eps = 1e-6
    params = {"termination_criteria.eps_optimal_relative": eps, "termination_criteria.eps_feasible_relative": eps,
              "termination_criteria.iteration_limit": 200000}
    fam = warmstart.ParametricQP(seed=9, n=2000)
    ws = warmstart.WarmStart(fam, hidden=256, rank=32, seed=2)
    try:
        train = fam.thetas(96, seed=1)
        X, lw, its = ws.collect(train, params)
        assert ws.step_size and ws.step_size > 0  # recorded by the first cold solve
        ws.fit(train, X, lw, epochs=300, batch=32, lr=1e-3)
        its = {"cold": [], "mean": [], "net": []}
        for th in fam.thetas(12, seed=2):
            res = {f: ws.solve(th, params, start=f) for f in its}
            ref = res["cold"]["primal_objective_value"]
            for f, d in res.items():
                assert d["status"] == "OPTIMAL", (f, d["status"])
                assert abs(d["primal_objective_value"] - ref) <= 10 * eps * (1 + abs(ref)), f
                its[f].append(d["total_count"])
        assert np.mean(its["net"]) < np.mean(its["cold"]), its
    finally:
        ws.close()
