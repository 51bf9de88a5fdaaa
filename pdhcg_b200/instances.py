"""Seeded synthetic instances of the benchmark workloads.

The reference publishes no benchmark data, so every workload is generated
from a seed with the shapes and value distributions of its description:

- ``sparse_qp``      random sparse convex QP, n=10000, m=5000, 8 nnz/row,
                     Q = B'B + 0.1 I with B 2000 x n, 4 nnz/row (BB inner solve)
- ``soc_qp``         SOC-constrained QP, n=1e6, m=5e5, 10 nnz/row, diagonal Q,
                     20000 SOC blocks of 50 slots, equality rows b = A x0 with
                     x0 strictly inside the cones
- ``portfolio``      low-rank portfolio QP with a rotated-SOC tracking-error block
- ``mpc_batch``      batched uneven MPC-style QPs
- ``parametric_qp``  parametric family for the learned warm start

Every generator takes a ``scale`` in (0, 1] that shrinks the sizes for
parity tests while keeping the structure.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .capi import (CONE_EXPONENTIAL, CONE_POWER, CONE_PSD, CONE_ROTATED_SOC, CONE_STANDARD_SOC, Cone, CsrMatrix,
                   Problem)


def random_csr(rng: np.random.Generator, m: int, n: int, per_row: int, values: str = "normal") -> CsrMatrix:
    """m x n CSR with exactly ``per_row`` distinct uniform columns per row."""
    k = min(per_row, n)
    cols = rng.integers(0, n, size=(m, k), dtype=np.int64)
    cols.sort(axis=1)
    for _ in range(64):
        dup = np.zeros_like(cols, dtype=bool)
        dup[:, 1:] = cols[:, 1:] == cols[:, :-1]
        nd = int(dup.sum())
        if nd == 0:
            break
        cols[dup] = rng.integers(0, n, size=nd)
        cols.sort(axis=1)
    vals = rng.standard_normal((m, k)) if values == "normal" else rng.uniform(-1, 1, (m, k))
    row_ptr = np.arange(0, (m + 1) * k, k, dtype=np.int32)
    return CsrMatrix(m, n, row_ptr, cols.reshape(-1).astype(np.int32), vals.reshape(-1).astype(np.float64))


def sparse_qp(seed: int = 1, scale: float = 1.0) -> Problem:
    """Random sparse convex QP (sparse Q, inner BB solve)."""
    rng = np.random.default_rng(seed)
    n = max(20, int(10000 * scale))
    m = max(10, int(5000 * scale))
    nb = max(4, int(2000 * scale))
    A = random_csr(rng, m, n, 8)
    B = random_csr(rng, nb, n, 4).to_scipy()
    Q = (B.T @ B + 0.1 * sp.identity(n, format="csr")).tocsr()
    Q.sort_indices()
    c = rng.standard_normal(n)
    x0 = rng.uniform(-1, 1, n)
    ax = A.to_scipy() @ x0
    lo = ax - rng.uniform(0, 1, m)
    up = ax + rng.uniform(0, 1, m)
    return Problem(c=c, A=A, con_lb=lo, con_ub=up, var_lb=np.full(n, -10.0), var_ub=np.full(n, 10.0),
                   Q=CsrMatrix.from_scipy(Q))


def soc_qp(seed: int = 2, scale: float = 1.0, block: int = 50) -> Problem:
    """SOC-constrained QP with a diagonal Q; all variables in SOC blocks."""
    rng = np.random.default_rng(seed)
    nblocks = max(2, int(20000 * scale))
    n = nblocks * block
    m = n // 2
    A = random_csr(rng, m, n, 10)
    q = rng.uniform(0.01, 1.0, n)
    c = rng.standard_normal(n)
    # x0 strictly inside every block: z = |(v, w)| + 1
    x0 = rng.standard_normal(n)
    xb = x0.reshape(nblocks, block)
    xb[:, -1] = np.linalg.norm(xb[:, :-1], axis=1) + 1.0
    x0 = xb.reshape(-1)
    b = A.to_scipy() @ x0
    cones = [Cone(CONE_STANDARD_SOC, i * block, block - 2) for i in range(nblocks)]
    Q = CsrMatrix(n, n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), q)
    return Problem(c=c, A=A, con_lb=b, con_ub=b.copy(), var_lb=np.full(n, -np.inf), var_ub=np.full(n, np.inf),
                   Q=Q, cones=cones)


def box_lp(seed: int = 3, n: int = 300, m: int = 150) -> Problem:
    """Feasible random LP with row ranges and a box."""
    rng = np.random.default_rng(seed)
    A = random_csr(rng, m, n, 6)
    x0 = rng.uniform(-1, 1, n)
    ax = A.to_scipy() @ x0
    lo = ax - rng.uniform(0, 1, m)
    up = ax + rng.uniform(0, 1, m)
    eq = rng.random(m) < 0.3
    up[eq] = lo[eq] = ax[eq]
    return Problem(c=rng.standard_normal(n), A=A, con_lb=lo, con_ub=up, var_lb=np.full(n, -2.0),
                   var_ub=np.full(n, 2.0))


def dense_rows_qp(seed: int = 21, n: int = 6000, m: int = 3000, ndense: int = 3, with_q: bool = False) -> Problem:
    """Box LP (or diagonal QP) whose A has ``ndense`` dense rows (n entries)
    among rows of 6 random entries, and one dense column (variable 0 in
    every row): rows and columns longer than the products' long-row
    threshold.  Row ranges through a random point, so it is feasible."""
    rng = np.random.default_rng(seed)
    B = random_csr(rng, m, n, 6).to_scipy().tolil()
    dense = rng.choice(m, ndense, replace=False)
    for r in dense:
        B[int(r), :] = rng.standard_normal(n) / np.sqrt(n)
    B[:, 0] = rng.standard_normal((m, 1))
    A = B.tocsr()
    A.sort_indices()
    x0 = rng.uniform(-1, 1, n)
    ax = A @ x0
    lo = ax - rng.uniform(0, 1, m)
    up = ax + rng.uniform(0, 1, m)
    p = Problem(c=rng.standard_normal(n), A=CsrMatrix.from_scipy(A), con_lb=lo, con_ub=up,
                var_lb=np.full(n, -2.0), var_ub=np.full(n, 2.0))
    if with_q:
        p.Q = CsrMatrix(n, n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32),
                        rng.uniform(0.05, 1.0, n))
    return p


def diag_qp(seed: int = 4, n: int = 300, m: int = 150) -> Problem:
    p = box_lp(seed, n, m)
    rng = np.random.default_rng(seed + 100)
    q = rng.uniform(0.05, 1.0, n)
    p.Q = CsrMatrix(n, n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), q)
    return p


def conic_lp(seed: int = 5, nfree: int = 60, nsoc: int = 10, soc_len: int = 12, nrsoc: int = 4,
             rsoc_len: int = 8, with_q: bool = False, nexp: int = 0, npow: int = 0) -> Problem:
    """Free box variables plus SOC, rotated-SOC, exponential and power
    blocks (exponents U(0.2, 0.8)), equality rows through a strictly
    feasible point (so the problem is feasible) and an objective inside the
    dual cone on the cone slots (so it is bounded)."""
    return _conic_lp_point(seed, nfree, nsoc, soc_len, nrsoc, rsoc_len, with_q, nexp, npow)[0]


def fixed_cone_qp(seed: int = 21, with_q: bool = False, sparse_q: bool = False, nexp: int = 6, npow: int = 6,
                  soc_len: int = 12, nsoc: int = 10) -> Problem:
    """conic_lp with slots of about half the cone blocks fixed by
    set_cone_fixed at the strictly feasible point the rows pass through, so
    every section is nonempty and the problem stays feasible and bounded.
    The fixed slots cover every kind the section projectors handle: the SOC
    apex, w or a vector slot; the rotated-SOC s, t, both, or a vector slot;
    one or two axes of exponential and power blocks.  sparse_q couples
    neighbouring free variables in Q (the inner BB solve)."""
    p, x0 = _conic_lp_point(seed, 60, nsoc, soc_len, 4, 8, with_q or sparse_q, nexp, npow)
    rng = np.random.default_rng(seed + 1000)
    fixed = []
    for ci, k in enumerate(p.cones):
        if rng.random() < 0.45:
            continue
        L = k.v_dim + 2
        if k.type == CONE_STANDARD_SOC:
            slots = [[L - 1], [L - 2], [0], [0, L - 1]][rng.integers(4)]
        elif k.type == CONE_ROTATED_SOC:
            slots = [[L - 2], [L - 1], [L - 2, L - 1], [0]][rng.integers(4)]
        else:
            slots = [[0], [1], [2], [0, 1], [1, 2], [0, 2]][rng.integers(6)]
        for sl in slots:
            fixed.append((ci, sl, float(x0[k.start + sl])))
    p.fixed = fixed
    if sparse_q:
        n = p.n
        q = p.Q.val.copy()
        rows = [[] for _ in range(n)]
        for i in range(n):
            rows[i].append((i, q[i]))
        for i in range(0, 59, 2):  # pairs of free variables, diagonally dominant
            w = 0.3 * min(q[i], q[i + 1])
            rows[i].append((i + 1, w))
            rows[i + 1].append((i, w))
        rp = np.zeros(n + 1, np.int32)
        ci_, v_ = [], []
        for i in range(n):
            for j, w in sorted(rows[i]):
                ci_.append(j)
                v_.append(w)
            rp[i + 1] = len(ci_)
        p.Q = CsrMatrix(n, n, rp, np.array(ci_, np.int32), np.array(v_))
    return p


def _conic_lp_point(seed, nfree, nsoc, soc_len, nrsoc, rsoc_len, with_q, nexp, npow):
    rng = np.random.default_rng(seed)
    n = nfree + nsoc * soc_len + nrsoc * rsoc_len + 3 * (nexp + npow)
    m = n // 3
    A = random_csr(rng, m, n, 5)
    x0 = np.zeros(n)
    x0[:nfree] = rng.uniform(-0.5, 0.5, nfree)
    cones = []
    st = nfree
    for _ in range(nsoc):
        v = rng.standard_normal(soc_len - 1)
        x0[st:st + soc_len - 1] = v
        x0[st + soc_len - 1] = np.linalg.norm(v) + 1.0
        cones.append(Cone(CONE_STANDARD_SOC, st, soc_len - 2))
        st += soc_len
    for _ in range(nrsoc):
        v = rng.standard_normal(rsoc_len - 2)
        s_ = 1.0 + rng.random()
        x0[st:st + rsoc_len - 2] = v
        x0[st + rsoc_len - 2] = s_
        x0[st + rsoc_len - 1] = (v @ v) / (2 * s_) + 1.0
        cones.append(Cone(CONE_ROTATED_SOC, st, rsoc_len - 2))
        st += rsoc_len
    for _ in range(nexp):  # y exp(x / y) < z
        xe, ye = rng.standard_normal(), 1.0 + rng.random()
        x0[st:st + 3] = xe, ye, ye * np.exp(xe / ye) + 1.0
        cones.append(Cone(CONE_EXPONENTIAL, st, 1))
        st += 3
    for _ in range(npow):  # x^a y^(1-a) > |z|
        a = rng.uniform(0.2, 0.8)
        xp_, yp_ = 1.0 + rng.random(), 1.0 + rng.random()
        x0[st:st + 3] = xp_, yp_, 0.5 * xp_ ** a * yp_ ** (1 - a) * rng.choice([-1.0, 1.0])
        cones.append(Cone(CONE_POWER, st, 1, a))
        st += 3
    b = A.to_scipy() @ x0
    lb = np.full(n, -np.inf)
    ub = np.full(n, np.inf)
    lb[:nfree] = -1.0
    ub[:nfree] = 1.0
    # a bounded objective: c in the interior of the dual cone on cone slots
    c = rng.standard_normal(n) * 0.5
    st = nfree
    for k in cones:
        L = k.v_dim + 2
        if k.type == CONE_STANDARD_SOC:
            c[st + L - 1] = np.linalg.norm(c[st:st + L - 1]) + 1.0
        elif k.type == CONE_EXPONENTIAL:  # K* = {(u, v, w): u < 0, -u exp(v / u) <= e w}
            u = -(0.5 + rng.random())
            c[st] = u
            c[st + 2] = -u * np.exp(c[st + 1] / u) / np.e + 1.0
        elif k.type == CONE_POWER:  # K* = {(u, v, w): (u / a)^a (v / (1 - a))^(1 - a) >= |w|}
            a = k.alpha
            c[st], c[st + 1] = 0.5 + rng.random(), 0.5 + rng.random()
            c[st + 2] = 0.5 * (c[st] / a) ** a * (c[st + 1] / (1 - a)) ** (1 - a) * np.sign(c[st + 2])
        else:
            c[st + L - 2] = abs(c[st + L - 2]) + 1.0
            c[st + L - 1] = (c[st:st + L - 2] @ c[st:st + L - 2]) / (2 * c[st + L - 2]) + 1.0
        st += L
    p = Problem(c=c, A=A, con_lb=b, con_ub=b.copy(), var_lb=lb, var_ub=ub, cones=cones)
    if with_q:
        q = rng.uniform(0.1, 1.0, n)
        p.Q = CsrMatrix(n, n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), q)
    return p, x0


def _svec(X: np.ndarray) -> np.ndarray:
    """Lower triangle down the columns, off-diagonal entries times sqrt 2."""
    n = X.shape[0]
    return np.array([X[r, c] if r == c else X[r, c] * np.sqrt(2.0) for c in range(n) for r in range(c, n)])


def psd_lp(seed: int = 6, nfree: int = 40, orders=(2, 3, 4, 5, 3, 6), with_q: bool = False) -> Problem:
    """Box variables plus PSD blocks (svec packing, orders ``orders``),
    equality rows through a point whose PSD blocks are positive definite,
    and an objective positive definite on each PSD block (so the problem is
    feasible and bounded).  with_q adds a diagonal Q (the inner BB solve)."""
    rng = np.random.default_rng(seed)
    lens = [k * (k + 1) // 2 for k in orders]
    n = nfree + sum(lens)
    m = n // 3
    A = random_csr(rng, m, n, 5)
    x0 = np.zeros(n)
    c = rng.standard_normal(n) * 0.5
    x0[:nfree] = rng.uniform(-0.5, 0.5, nfree)
    cones, st = [], nfree
    for k, L in zip(orders, lens):
        B = rng.standard_normal((k, k))
        x0[st:st + L] = _svec(B @ B.T + np.eye(k))
        C2 = rng.standard_normal((k, k))
        c[st:st + L] = _svec(C2 @ C2.T / k + 0.5 * np.eye(k))
        cones.append(Cone(CONE_PSD, st, k))
        st += L
    b = A.to_scipy() @ x0
    lb = np.full(n, -np.inf)
    ub = np.full(n, np.inf)
    lb[:nfree] = -1.0
    ub[:nfree] = 1.0
    p = Problem(c=c, A=A, con_lb=b, con_ub=b.copy(), var_lb=lb, var_ub=ub, cones=cones)
    if with_q:
        p.Q = CsrMatrix(n, n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32),
                        rng.uniform(0.1, 1.0, n))
    return p


def affine_cone_qp(seed: int = 9, n: int = 80, m_scalar: int = 20,
                   blocks=((1, 6), (0, 4), (2, 1), (3, 1), (4, 3), (1, 10)), with_q: bool = False) -> Problem:
    """Box variables, m_scalar equality rows and affine cone rows F x + g in
    K (blocks of (cone type, v_dim): SOC, RSOC, exponential, power with
    alpha U(0.2, 0.8), PSD), F with 4 random entries per row; g puts F x0 + g
    strictly inside each cone at a random x0 inside the box, so the problem
    is feasible; the box keeps it bounded."""
    rng = np.random.default_rng(seed)
    x0 = rng.uniform(-0.5, 0.5, n)
    A = random_csr(rng, m_scalar, n, 5)
    b = A.to_scipy() @ x0
    lens = [3 if t in (2, 3) else (k * (k + 1) // 2 if t == 4 else k + 2) for t, k in blocks]
    F = random_csr(rng, sum(lens), n, 4)
    u0, cones, st = [], [], 0
    for (t, k), L in zip(blocks, lens):
        if t == 1:  # [v, w, z], |(v, w)| < z
            v = rng.standard_normal(L - 1)
            u = np.concatenate([v, [np.linalg.norm(v) + 1.0]])
        elif t == 0:  # [v, s, t], |v|^2 < 2 s t
            v = rng.standard_normal(L - 2)
            s_ = 1.0 + rng.random()
            u = np.concatenate([v, [s_, (v @ v) / (2 * s_) + 1.0]])
        elif t == 2:  # y exp(x / y) < z
            xe, ye = rng.standard_normal(), 1.0 + rng.random()
            u = np.array([xe, ye, ye * np.exp(xe / ye) + 1.0])
        elif t == 3:  # x^a y^(1-a) > |z|
            a = rng.uniform(0.2, 0.8)
            xp_, yp_ = 1.0 + rng.random(), 1.0 + rng.random()
            u = np.array([xp_, yp_, 0.5 * xp_ ** a * yp_ ** (1 - a)])
        else:  # svec of a positive definite matrix
            B = rng.standard_normal((k, k))
            u = _svec(B @ B.T + np.eye(k))
        cones.append(Cone(t, st, k, rng.uniform(0.2, 0.8) if t == 3 else 0.0))
        if t == 3:  # rebuild the point for the drawn exponent
            a = cones[-1].alpha
            u = np.array([u[0], u[1], 0.5 * u[0] ** a * u[1] ** (1 - a)])
        u0.append(u)
        st += L
    g = np.concatenate(u0) - F.to_scipy() @ x0
    p = Problem(c=rng.standard_normal(n), A=A, con_lb=b, con_ub=b.copy(), var_lb=np.full(n, -1.0),
                var_ub=np.full(n, 1.0), F=F, g=g, affine_cones=cones)
    if with_q:
        p.Q = CsrMatrix(n, n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32),
                        rng.uniform(0.1, 1.0, n))
    return p


def portfolio(seed: int = 3, scale: float = 1.0, rank: int = 100, sectors: int = 500) -> Problem:
    """Low-rank portfolio QP with a rotated-SOC tracking-error block.

    Variables: weights x (n assets), factor exposures z (rank), s, t.
    Objective 1/2 x'(R'DR + Q)x - mu'x with R rank x n dense N(0, 1/sqrt(n))
    (passed as a dense matrix), D = diag U(0.5, 2), Q = diag U(1e-4, 1e-2).
    Rows: budget sum x = 1; one row per sector with upper bound 0.05; the
    exposure rows z - diag(sqrt D) R x = 0; s = TE^2 / 2 and t = 1.
    Cone: [z, s, t] in the rotated SOC, i.e. |sqrt(D) R x|^2 <= TE^2.
    Box: 0 <= x <= 0.02; z, s, t free (cone slots).
    """
    rng = np.random.default_rng(seed)
    n = max(100, int(200000 * scale))
    k = rank if scale >= 0.05 else max(4, int(rank * scale * 20))
    nsec = max(2, min(sectors, n // 20))
    R = rng.standard_normal((k, n)) / np.sqrt(n)
    Dd = rng.uniform(0.5, 2.0, k)
    qd = rng.uniform(1e-4, 1e-2, n)
    mu = rng.uniform(0.0, 1e-3, n)
    N = n + k + 2
    sec = rng.integers(0, nsec, n)
    x0 = np.full(n, 1.0 / n)
    z0 = np.sqrt(Dd) * (R @ x0)
    te2 = 1.5 * float(z0 @ z0) + 1e-8
    rows, cols, vals = [], [], []
    # budget
    rows.append(np.zeros(n, np.int64)); cols.append(np.arange(n)); vals.append(np.ones(n))
    # sectors
    rows.append(1 + sec); cols.append(np.arange(n)); vals.append(np.ones(n))
    # exposures: z_r - sqrt(D_r) R_r x = 0
    base = 1 + nsec
    rr = np.repeat(np.arange(k), n)
    rows.append(base + rr); cols.append(np.tile(np.arange(n), k)); vals.append((-np.sqrt(Dd)[:, None] * R).ravel())
    rows.append(base + np.arange(k)); cols.append(n + np.arange(k)); vals.append(np.ones(k))
    # s and t
    rows.append(np.array([base + k, base + k + 1])); cols.append(np.array([n + k, n + k + 1])); vals.append(np.ones(2))
    m = base + k + 2
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(m, N))
    A.sort_indices()
    lo = np.full(m, -np.inf)
    up = np.full(m, np.inf)
    lo[0] = up[0] = 1.0
    up[1:base] = 0.05
    lo[base:base + k] = up[base:base + k] = 0.0
    lo[base + k] = up[base + k] = 0.5 * te2
    lo[base + k + 1] = up[base + k + 1] = 1.0
    lb = np.concatenate([np.zeros(n), np.full(k + 2, -np.inf)])
    ub = np.concatenate([np.full(n, 0.02), np.full(k + 2, np.inf)])
    c = np.concatenate([-mu, np.zeros(k + 2)])
    Qd = np.concatenate([qd, np.zeros(k + 2)])
    qidx = np.arange(n)
    Q = CsrMatrix(N, N, np.concatenate([np.arange(n + 1), np.full(k + 2, n)]).astype(np.int32),
                  qidx.astype(np.int32), qd)
    Rfull = np.zeros((k, N))
    Rfull[:, :n] = R
    Dm = CsrMatrix(k, k, np.arange(k + 1, dtype=np.int32), np.arange(k, dtype=np.int32), Dd)
    return Problem(c=c, A=CsrMatrix.from_scipy(A), con_lb=lo, con_ub=up, var_lb=lb, var_ub=ub, Q=Q,
                   R_dense=Rfull, D=Dm, cones=[Cone(CONE_ROTATED_SOC, n, k)])


def mpc_qp(seed: int, horizon: int, nx: int = 8, nu: int = 4) -> Problem:
    """One MPC-style QP: states x_1..x_T (nx each) and inputs u_0..u_{T-1}
    (nu each), n = (nx + nu) T, dynamics rows x_{t+1} - A_t x_t - B_t u_t = 0
    (the first block row carries A_0 x_0 as its right-hand side), so each
    row has 1 + nx + nu nonzeros.  A_t = I + E_t with E_t entries
    N(0, (0.3 / sqrt(nx))^2), rescaled to spectral radius <= 1 so a horizon
    of 100 stays bounded; B_t entries N(0, 0.3^2); x_0 ~ N(0, I);
    Q = diag U(0.1, 1); inputs in [-1, 1]; states free; c = 0."""
    rng = np.random.default_rng(seed)
    T = horizon
    nxT, nuT = nx * T, nu * T
    n = nxT + nuT
    m = nxT
    x0 = rng.standard_normal(nx)
    # the draws in their stage order (E_0, B_0, E_1, B_1, ...), then the
    # stages' arithmetic on the stacks
    E = np.empty((T, nx, nx))
    Bs = np.empty((T, nx, nu))
    for t in range(T):
        E[t] = rng.standard_normal((nx, nx))
        Bs[t] = rng.standard_normal((nx, nu))
    At = np.eye(nx) + E * (0.3 / np.sqrt(nx))
    rad = np.max(np.abs(np.linalg.eigvals(At)), axis=1)
    At[rad > 1.0] /= rad[rad > 1.0][:, None, None]
    Bt = Bs * 0.3
    b = np.zeros(m)
    b[:nx] = At[0] @ x0
    # CSR rows in column order: -A_t (from stage 1 on), the identity of
    # x_{t+1}, -B_t; stage 0 rows have 1 + nu entries, the others nx + 1 + nu
    i = np.arange(nx)
    c0 = np.concatenate([i[:, None], nxT + np.broadcast_to(np.arange(nu), (nx, nu))], axis=1)
    v0 = np.concatenate([np.ones((nx, 1)), -Bt[0]], axis=1)
    t = np.arange(1, T)[:, None, None]
    ca = np.broadcast_to((t - 1) * nx + np.arange(nx)[None, None, :], (T - 1, nx, nx))
    ci = np.broadcast_to(t * nx + i[None, :, None], (T - 1, nx, 1))
    cb = np.broadcast_to(nxT + t * nu + np.arange(nu)[None, None, :], (T - 1, nx, nu))
    c1 = np.concatenate([ca, ci, cb], axis=2)
    v1 = np.concatenate([-At[1:], np.ones((T - 1, nx, 1)), -Bt[1:]], axis=2)
    col = np.concatenate([c0.ravel(), c1.ravel()])
    val = np.concatenate([v0.ravel(), v1.ravel()])
    per = np.full(m, 1 + nu, dtype=np.int64)
    per[nx:] += nx
    row_ptr = np.concatenate([[0], np.cumsum(per)])
    A = CsrMatrix(m, n, row_ptr.astype(np.int32), col.astype(np.int32), val)
    q = rng.uniform(0.1, 1.0, n)
    lb = np.concatenate([np.full(nxT, -np.inf), np.full(nuT, -1.0)])
    ub = np.concatenate([np.full(nxT, np.inf), np.full(nuT, 1.0)])
    Q = CsrMatrix(n, n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), q)
    return Problem(c=np.zeros(n), A=A, con_lb=b, con_ub=b.copy(), var_lb=lb, var_ub=ub, Q=Q)


def mpc_horizons(seed: int = 4, count: int = 4096, tmin: int = 10, tmax: int = 100) -> np.ndarray:
    """The horizons of mpc_batch(seed, count), without building the instances."""
    return np.random.default_rng(seed).integers(tmin, tmax + 1, size=count)


def mpc_nnz(horizon: int, nx: int = 8, nu: int = 4) -> int:
    """Nonzeros of mpc_qp(., horizon)'s constraint matrix: per stage the
    identity of x_{t+1}, A_t (except the first stage, whose A_0 x_0 is the
    right-hand side) and B_t."""
    return int(horizon * (nx + nx * nu) + (horizon - 1) * nx * nx)


def mpc_batch(seed: int = 4, count: int = 4096, tmin: int = 10, tmax: int = 100, indices=None) -> list:
    """`count` MPC QPs of uneven horizons T ~ U{tmin..tmax}, instance i seeded
    by (seed, i); ``indices`` builds only those instances of the batch."""
    horizons = mpc_horizons(seed, count, tmin, tmax)
    idx = range(count) if indices is None else indices
    return [mpc_qp(seed * 1000003 + i, int(horizons[i])) for i in idx]
