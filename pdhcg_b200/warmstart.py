"""Learned warm start on a parametric QP family.

A parametric family shares A, Q and the variable box; an instance's
parameter theta (dim 32) moves the objective and the row bounds:
``c = c0 + C theta``, ``[l, u] = [l0, u0] + L theta``.  ``WarmStart``
collects cold solves of training parameters with the library's own solver,
fits the MLP of ``pdhcg_b200_mlp_*`` (trained on the GPU by the library's
kernels) from theta to the solution (x, y) and the final primal weight, and
solves a new instance from the predicted point
(``set_start_values`` + ``initial_primal_weight``), reusing the step size of
the family's fixed constraint matrix (``initial_step_size``).  The cold solve stays the
reference: a warm solve must meet the same termination tolerance.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import capi, native
from .capi import CsrMatrix, Problem
from .instances import random_csr


class ParametricQP:
    """Fixed-sparsity QP family: n variables, m = n / 2 rows with 6 nnz/row
    N(0, 1), Q = diag U(0.1, 1), box [-10, 10]; theta ~ N(0, I_dim) gives
    c = c0 + C theta (C n x dim, N(0, 0.1^2)) and row bounds shifted by
    L theta (L m x dim, N(0, 0.1^2)) around l0 = A x0 - U(0, 1),
    u0 = A x0 + U(0, 1), x0 ~ U(-1, 1)."""

    def __init__(self, seed: int = 5, n: int = 50000, dim: int = 32):
        rng = np.random.default_rng(seed)
        self.n, self.m, self.dim = n, n // 2, dim
        self.A = random_csr(rng, self.m, n, 6)
        self.q = rng.uniform(0.1, 1.0, n)
        self.c0 = rng.standard_normal(n)
        self.C = rng.standard_normal((n, dim)) * 0.1
        self.L = rng.standard_normal((self.m, dim)) * 0.1
        x0 = rng.uniform(-1, 1, n)
        ax = self.A.to_scipy() @ x0
        self.l0 = ax - rng.uniform(0, 1, self.m)
        self.u0 = ax + rng.uniform(0, 1, self.m)
        self.Q = CsrMatrix(n, n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), self.q)

    def thetas(self, count: int, seed: int) -> np.ndarray:
        return np.random.default_rng(seed).standard_normal((count, self.dim))

    def problem(self, theta: np.ndarray) -> Problem:
        shift = self.L @ theta
        return Problem(c=self.c0 + self.C @ theta, A=self.A, con_lb=self.l0 + shift, con_ub=self.u0 + shift,
                       var_lb=np.full(self.n, -10.0), var_ub=np.full(self.n, 10.0), Q=self.Q)


def _fp(a):
    return np.ascontiguousarray(a, dtype=np.float32).ctypes.data_as(C.POINTER(C.c_float))


class WarmStart:
    """theta -> (x, y, primal weight) with the library's MLP."""

    def __init__(self, family: ParametricQP, hidden: int = 512, rank: int = 64, seed: int = 1):
        self.lib = native.load()
        self.family = family
        self.out_dim = family.n + family.m
        self.net = self.lib.pdhcg_b200_mlp_create(family.dim, hidden, rank, self.out_dim, seed)
        if not self.net:
            raise RuntimeError("pdhcg_b200_mlp_create failed")
        self.mean = np.zeros(self.out_dim)
        self.mean_log_weight = 0.0
        self.scale = np.ones(self.out_dim)
        # 0.998 / sigma_max of the scaled A, shared by the whole family (A and
        # the scaling parameters are fixed), recorded by the first cold solve
        self.step_size = None

    def close(self):
        if self.net:
            self.lib.pdhcg_b200_mlp_free(self.net)
            self.net = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- data -------------------------------------------------------------
    def solve(self, theta, params: dict, warm: bool = False, start: str | None = None) -> dict:
        """One solve of the instance theta from one of three starts:

        - ``"cold"``: x = 0, y = 0 and the solver's own primal weight;
        - ``"mean"``: the mean of the training targets (x, y) and their mean
          log primal weight, the same for every instance (what a start
          without the network gets from the training data);
        - ``"net"`` (``warm=True``): the network's prediction for theta.

        Once a cold solve has recorded the family's step size (0.998 /
        sigma_max of the scaled A, shared by the family: A and the scaling
        parameters are fixed), every form reuses it and skips the power
        method, so the forms differ only in their start.  ``wall_s`` is the
        wall time of the whole call, the network's prediction included."""
        start = start or ("net" if warm else "cold")
        lib = self.lib
        t0 = time.perf_counter()
        p = self.family.problem(theta)
        prob, keep = capi.build(lib, p)
        opts = native.default_options()
        if start in ("net", "mean"):
            if start == "net":
                x, y, w = self.predict(theta[None, :])
                x, y, w = x[0], y[0], float(w[0])
            else:
                x, y = self.mean[:self.family.n], self.mean[self.family.n:]
                w = float(np.exp(self.mean_log_weight))
            xs, ys = np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64)
            dp = C.POINTER(C.c_double)
            lib.set_start_values(prob, xs.ctypes.data_as(dp), ys.ctypes.data_as(dp))
            opts.has_initial_primal_weight = 1
            opts.initial_primal_weight = w
        if self.step_size:
            opts.has_initial_step_size = 1
            opts.initial_step_size = self.step_size
        prm = capi.default_params(lib, **params)
        r = lib.pdhcg_b200_solve(prob, C.byref(prm), C.byref(opts))
        if not r:
            lib.qp_problem_free(prob)
            raise RuntimeError("solve failed")
        d = capi.result_dict(r, p.n, p.A.m)
        st = native.last_stats()
        d["final_primal_weight"] = st["primal_weight"]
        if self.step_size is None:
            self.step_size = st["step_size"]
        lib.pdhcg_result_free(r)
        lib.qp_problem_free(prob)
        d["wall_s"] = time.perf_counter() - t0
        d["stats"] = st
        return d

    def collect(self, thetas: np.ndarray, params: dict):
        """Cold solves of the training parameters: targets (x, y) and log weight."""
        X = np.zeros((len(thetas), self.out_dim), np.float32)
        lw = np.zeros(len(thetas), np.float32)
        its = []
        for i, th in enumerate(thetas):
            d = self.solve(th, params)
            X[i, :self.family.n] = d["x"]
            X[i, self.family.n:] = d["y"]
            lw[i] = np.log(d["final_primal_weight"])
            its.append(d["total_count"])
        return X, lw, np.array(its)

    # ---- network ----------------------------------------------------------
    def fit(self, thetas: np.ndarray, X: np.ndarray, lw: np.ndarray, epochs: int = 200, batch: int = 64,
            lr: float = 1e-3) -> float:
        """Normalise the targets per output (mean, scale) and train on the GPU."""
        self.mean = X.mean(0).astype(np.float64)
        self.mean_log_weight = float(np.mean(lw))
        sd = X.std(0).astype(np.float64)
        self.scale = np.where(sd > 1e-8, sd, 1.0)
        T = ((X - self.mean) / self.scale).astype(np.float32)
        loss = C.c_double()
        rc = self.lib.pdhcg_b200_mlp_train(self.net, len(thetas), _fp(thetas), _fp(T), _fp(lw), epochs,
                                           min(batch, len(thetas)), lr, C.byref(loss))
        if rc != 0:
            raise RuntimeError("pdhcg_b200_mlp_train failed")
        return loss.value

    def predict(self, thetas: np.ndarray):
        B = len(thetas)
        out = np.zeros((B, self.out_dim), np.float32)
        lw = np.zeros(B, np.float32)
        rc = self.lib.pdhcg_b200_mlp_predict(self.net, B, _fp(thetas), out.ctypes.data_as(C.POINTER(C.c_float)),
                                             lw.ctypes.data_as(C.POINTER(C.c_float)))
        if rc != 0:
            raise RuntimeError("pdhcg_b200_mlp_predict failed")
        full = out.astype(np.float64) * self.scale + self.mean
        return full[:, :self.family.n], full[:, self.family.n:], np.exp(lw.astype(np.float64))
