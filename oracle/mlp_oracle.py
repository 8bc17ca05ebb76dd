"""CPU ORACLE of the predictor network (test infrastructure only).

A numpy restatement of zerork_b200/csrc/mlp.cu's forward and backward passes
with the same rounding points: inputs, hidden activations and the backward
deltas that feed matrix products are rounded to BF16 (round to nearest
even), weights are the BF16 copies of the FP32 masters, biases stay FP32,
and products accumulate in FP64 here (FP32 on the GPU), so GPU and oracle
gradients differ only by accumulation order and the rare BF16 rounding that
order flips.  The network has no counterpart in the reference.
"""
import numpy as np


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def pad16(n):
    return (n + 15) // 16 * 16


def dims(n_in, hidden, layers, n_out):
    return [pad16(n_in)] + [pad16(hidden)] * layers + [pad16(n_out)]


def unpack(w_flat, b_flat, d):
    """Per-layer (W [d_l x d_{l+1}], b [d_{l+1}]) views of the flat arrays."""
    W, B, ow, ob = [], [], 0, 0
    for l in range(len(d) - 1):
        W.append(w_flat[ow:ow + d[l] * d[l + 1]].reshape(d[l], d[l + 1]))
        B.append(b_flat[ob:ob + d[l + 1]])
        ow += d[l] * d[l + 1]
        ob += d[l + 1]
    return W, B


def silu(z):
    return z / (1.0 + np.exp(-z))


def forward_backward(w_flat, b_flat, d, x, t):
    """Loss sum of squared errors and the flat (dW, db) of the mean squared
    error over the batch, for inputs x [n, n_in] and targets t [n, n_out]."""
    W, B = unpack(np.asarray(w_flat, np.float32), np.asarray(b_flat, np.float32), d)
    Wb = [bf16(w).astype(np.float64) for w in W]
    n, n_in = x.shape
    n_out = t.shape[1]
    L = len(W)
    X = [np.zeros((n, d[0]), np.float64)]
    X[0][:, :n_in] = bf16(x.astype(np.float32))
    Z = [None]
    for l in range(L):
        z = (X[l] @ Wb[l]).astype(np.float32) + B[l]
        Z.append(z.astype(np.float32))
        if l + 1 < L:
            X.append(bf16(silu(z.astype(np.float32)).astype(np.float32)).astype(np.float64))
    y = Z[L][:, :n_out].astype(np.float64)
    e = y - t
    loss = float(np.sum(e * e))
    g = np.zeros((n, d[L]), np.float32)
    g[:, :n_out] = (2.0 / (n * n_out)) * e
    dW, dB = [None] * L, [None] * L
    dzf = g
    dz = bf16(g).astype(np.float64)
    for l in range(L - 1, -1, -1):
        dW[l] = (X[l].T @ dz).astype(np.float32)
        dB[l] = dzf.astype(np.float64).sum(axis=0).astype(np.float32)
        if l == 0:
            break
        da = (dz @ Wb[l].T).astype(np.float32)
        z = Z[l]
        s = 1.0 / (1.0 + np.exp(-z.astype(np.float64)))
        dzf = (da * s * (1.0 + z * (1.0 - s))).astype(np.float32)
        dz = bf16(dzf).astype(np.float64)
    return loss, np.concatenate([w.ravel() for w in dW]), np.concatenate([b.ravel() for b in dB]), y
