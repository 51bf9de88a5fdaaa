"""CPU oracle of the learned-warm-start MLP (test infrastructure only).

A numpy restatement of the network, loss and gradient that
pdhcg_b200/csrc/mlp.cu computes, used to check the device forward and
backward kernels.  Weights are rounded to BF16 (round to nearest even)
before every product, as the device does; accumulation is FP64 here (the
device accumulates in FP32, so the tests compare to FP32 round-off).

    h1 = relu(W1 x + b1); h2 = relu(W2 h1 + b2); z = W3 h2 + b3
    o = U z + bu; lw = wp . h2 + bp
    loss = mean((o - t)^2) + mean((lw - t_lw)^2)
Packed parameter order: W1, b1, W2, b2, W3, b3, U, bu, wp, bp.
"""
import numpy as np


def shapes(n_in, hid, rank, out):
    return [(hid, n_in), (hid,), (hid, hid), (hid,), (rank, hid), (rank,), (out, rank), (out,), (hid,), (1,)]


def unpack(flat, n_in, hid, rank, out):
    parts, o = [], 0
    for sh in shapes(n_in, hid, rank, out):
        k = int(np.prod(sh))
        parts.append(np.asarray(flat[o:o + k], dtype=np.float64).reshape(sh))
        o += k
    return parts


def bf16(a):
    """Round float32 values to bfloat16 (nearest even) and back."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def loss_grad(flat, x, t, tl, n_in, hid, rank, out, quantize=True):
    """Loss, packed gradient, outputs and log weights.  quantize=False skips
    the BF16 rounding (for finite-difference checks of the formulas)."""
    W1, b1, W2, b2, W3, b3, U, bu, wp, bp = unpack(flat, n_in, hid, rank, out)
    q = bf16 if quantize else (lambda a: a)
    W1q, W2q, W3q, Uq = q(W1), q(W2), q(W3), q(U)
    x = np.asarray(x, np.float64)
    B = x.shape[0]
    a1 = x @ W1q.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2q.T + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ W3q.T + b3
    o = z @ Uq.T + bu
    lw = h2 @ wp + bp[0]
    r = o - t
    rl = lw - tl
    loss = np.mean(r * r) + np.mean(rl * rl)
    dO = 2.0 * r / r.size
    dlw = 2.0 * rl / B
    gU = dO.T @ z
    gbu = dO.sum(0)
    dZ = dO @ Uq
    gW3 = dZ.T @ h2
    gb3 = dZ.sum(0)
    dH2 = dZ @ W3q + np.outer(dlw, wp)
    gwp = dlw @ h2
    gbp = np.array([dlw.sum()])
    dH2 = dH2 * (h2 > 0)
    gW2 = dH2.T @ h1
    gb2 = dH2.sum(0)
    dH1 = (dH2 @ W2q) * (h1 > 0)
    gW1 = dH1.T @ x
    gb1 = dH1.sum(0)
    grad = np.concatenate([g.ravel() for g in (gW1, gb1, gW2, gb2, gW3, gb3, gU, gbu, gwp, gbp)])
    return loss, grad, o, lw
