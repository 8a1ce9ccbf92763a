"""Float64 numpy restatement of the triage MLP (12-64-64-1, ReLU, sigmoid output) and of its
weighted binary cross-entropy gradient: the check for the BF16 tensor-core kernels.

Parameter layout (gd_triage_set_model): mean[12], scale[12], W1[64][12], b1[64],
W2[64][64], b2[64], W3[64], b3.  Test infrastructure only.
"""

import numpy as np

NF, H = 12, 64
OFF_MEAN, OFF_STD, OFF_W1 = 0, 12, 24
OFF_B1 = OFF_W1 + H * NF
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAM = OFF_B3 + 1


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OFF_MEAN:OFF_MEAN + NF], p[OFF_STD:OFF_STD + NF], p[OFF_W1:OFF_B1].reshape(H, NF), p[OFF_B1:OFF_W2],
            p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def bf16(x):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.asarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(p, x, emulate_bf16=False):
    mean, std, W1, b1, W2, b2, W3, b3 = unpack(p)
    r = bf16 if emulate_bf16 else (lambda v: np.asarray(v, np.float64))
    X = r((np.asarray(x, np.float64) - mean) / std)
    A1 = X @ r(W1).T + b1
    H1 = r(np.maximum(A1, 0))
    A2 = H1 @ r(W2).T + b2
    H2 = r(np.maximum(A2, 0))
    z = H2 @ r(W3) + b3
    return X, H1, H2, z


def prob(p, x, emulate_bf16=False):
    return 1.0 / (1.0 + np.exp(-forward(p, x, emulate_bf16)[3]))


def loss_grad(p, x, y, pos_weight=1.0):
    """Mean weighted BCE over the rows and its gradient (mean/scale entries zero)."""
    mean, std, W1, b1, W2, b2, W3, b3 = unpack(p)
    X, H1, H2, z = forward(p, x)
    y = np.asarray(y, np.float64)
    n = len(y)
    w = np.where(y > 0.5, pos_weight, 1.0)
    loss = float(np.sum(w * (np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))) / n)
    dz = w * (1.0 / (1.0 + np.exp(-z)) - y) / n
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = H2.T @ dz
    g[OFF_B3] = dz.sum()
    dA2 = np.outer(dz, W3) * (H2 > 0)
    g[OFF_W2:OFF_B2] = (dA2.T @ H1).ravel()
    g[OFF_B2:OFF_W3] = dA2.sum(0)
    dA1 = (dA2 @ W2) * (H1 > 0)
    g[OFF_W1:OFF_B1] = (dA1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = dA1.sum(0)
    return loss, g


def loss_grad_bf16(p, x, y, pos_weight=1.0):
    """The gradient with the kernels' roundings: standardised inputs, weights, activations and
    the back-propagated dH2 / dH1 in bf16, everything else (biases, W3, dz, sums) at full
    precision.  Tracks the device gradient far more tightly than loss_grad, whose
    difference from the device is dominated by the bf16 forward pass."""
    mean, std, W1, b1, W2, b2, W3, b3 = unpack(p)
    x = np.asarray(x, np.float32)
    X = bf16((x - np.float32(mean)) / np.float32(std))
    H1 = bf16(np.maximum(X @ bf16(W1).T + b1, 0))
    H2 = bf16(np.maximum(H1 @ bf16(W2).T + b2, 0))
    z = H2 @ bf16(W3) + b3
    y = np.asarray(y, np.float64)
    n = len(y)
    w = np.where(y > 0.5, pos_weight, 1.0)
    loss = float(np.sum(w * (np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))) / n)
    dz = w * (1.0 / (1.0 + np.exp(-z)) - y) / n
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = H2.T @ dz
    g[OFF_B3] = dz.sum()
    dA2 = np.outer(dz, W3) * (H2 > 0)
    g[OFF_B2:OFF_W3] = dA2.sum(0)
    dH2 = bf16(dA2)
    g[OFF_W2:OFF_B2] = (dH2.T @ H1).ravel()
    dH1 = bf16((dH2 @ bf16(W2)) * (H1 > 0))
    g[OFF_W1:OFF_B1] = (dH1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = dH1.sum(0)
    return loss, g
