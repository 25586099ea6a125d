"""CPU restatement of the proposal network's math (TEST INFRASTRUCTURE ONLY).

Checks the GPU kernels of tensorfim_b200/csrc/mlp.cu: the forward pass reads BF16
copies of the weight matrices (round to nearest even) and accumulates in FP32/FP64; the
loss is mean_i w_i * BCE(sigmoid(z_i), y_i) with w_i = pos_weight for positives; the
gradient is taken with respect to the weights as the forward pass sees them.
Parameter layout: W1[64][32], b1[64], W2[64][64], b2[64], W3[64], b3.
"""
import numpy as np

IN, H = 32, 64
O_W1, O_B1 = 0, H * IN
O_W2 = O_B1 + H
O_B2 = O_W2 + H * H
O_W3 = O_B2 + H
O_B3 = O_W3 + H
N_PARAMS = O_B3 + 1


def bf16(x):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p, dtype=np.float32)
    W1 = bf16(p[O_W1:O_B1]).reshape(H, IN).astype(np.float64)
    W2 = bf16(p[O_W2:O_B2]).reshape(H, H).astype(np.float64)
    W3 = bf16(p[O_W3:O_B3]).astype(np.float64)
    return W1, p[O_B1:O_W2].astype(np.float64), W2, p[O_B2:O_W3].astype(np.float64), W3, float(p[O_B3])


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    z = h2 @ W3 + b3
    return z, (X, a1, h1, a2, h2)


def predict(p, X):
    z, _ = forward(p, X)
    return 1.0 / (1.0 + np.exp(-z))


def grad(p, X, y, pos_weight=1.0):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    z, (X, a1, h1, a2, h2) = forward(p, X)
    y = np.asarray(y, dtype=np.float64)
    n = X.shape[0]
    w = np.where(y > 0.5, pos_weight, 1.0)
    prob = 1.0 / (1.0 + np.exp(-z))
    loss = float(np.mean(w * (np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))))
    dz = w * (prob - y) / n
    d2 = (dz[:, None] * W3[None, :]) * (a2 > 0)
    d1 = (d2 @ W2) * (a1 > 0)
    g = np.zeros(N_PARAMS)
    g[O_W1:O_B1] = (d1.T @ X).reshape(-1)
    g[O_B1:O_W2] = d1.sum(0)
    g[O_W2:O_B2] = (d2.T @ h1).reshape(-1)
    g[O_B2:O_W3] = d2.sum(0)
    g[O_W3:O_B3] = dz @ h2
    g[O_B3] = dz.sum()
    return g, loss
