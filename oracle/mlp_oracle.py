"""ORACLE — test infrastructure only: numpy restatement of the warm-start MLP (forward, loss gradient, AdamW).

Only tests/ may import this module, as the checker of the CUDA kernels in diffphd_b200/csrc/mlp.cu.

There is no counterpart in the reference (its PD path has no learned part; the warm start starts every PD loop
from q, deformable_projective_dynamics_forward_gpu.cpp's q_sol initialisation).  The network is a per-node MLP
15 -> 128 -> 128 -> 3 with exact (erf) GELU, trained on the mean over nodes of the squared error summed over the
three outputs.

Parameter layout (one flat float array, shared with the CUDA kernels):
    W1 [16][128] | W2 [128][128] | W3 [128][8] | b1 [128] | b2 [128] | b3 [8]
Row 15 of W1 and columns 3..7 of W3 / b3 are structurally unused (their gradients are reported as 0).

`emulate=True` rounds to BF16 exactly where the tensor-core kernels do (inputs, weights, hidden activations,
GELU derivatives and the back-propagated pre-activation gradients) and keeps everything else in FP64, so that the
comparison with the GPU is limited by FP32 accumulation order.  `emulate=False` is the exact FP64 network.
"""
from __future__ import annotations

import math

import numpy as np

N_IN, N_HID, N_OUT, N_USED = 16, 128, 8, 4
OFF_W1 = 0
OFF_W2 = OFF_W1 + N_IN * N_HID
OFF_W3 = OFF_W2 + N_HID * N_HID
OFF_B1 = OFF_W3 + N_HID * N_OUT
OFF_B2 = OFF_B1 + N_HID
OFF_B3 = OFF_B2 + N_HID
N_PARAMS = OFF_B3 + N_OUT


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64).reshape(a.shape)


_erf = np.vectorize(math.erf, otypes=[np.float64])


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unpack(master):
    p = np.asarray(master, dtype=np.float64)
    W1 = p[OFF_W1:OFF_W2].reshape(N_IN, N_HID).copy()
    W2 = p[OFF_W2:OFF_W3].reshape(N_HID, N_HID).copy()
    W3 = p[OFF_W3:OFF_B1].reshape(N_HID, N_OUT).copy()
    b1, b2, b3 = p[OFF_B1:OFF_B2].copy(), p[OFF_B2:OFF_B3].copy(), p[OFF_B3:N_PARAMS].copy()
    W1[N_IN - 1, :] = 0.0
    W3[:, N_USED:] = 0.0
    return W1, W2, W3, b1, b2, b3


def forward(master, X, emulate=True):
    """Outputs [n][8] (columns 4..7 carry only b3) and the activations needed by the backward pass."""
    W1, W2, W3, b1, b2, b3 = unpack(master)
    r = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    x = r(X)
    z1 = x @ r(W1) + b1
    a1 = r(gelu(z1))
    z2 = a1 @ r(W2) + b2
    a2 = r(gelu(z2))
    out = a2 @ r(W3) + b3
    return out, (x, z1, a1, z2, a2)


def loss_and_grad(master, X, Y, emulate=True):
    """loss = sum((out[:, :4] - Y)^2) / n and its gradient in the flat layout."""
    W1, W2, W3, b1, b2, b3 = unpack(master)
    r = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    n = X.shape[0]
    out, (x, z1, a1, z2, a2) = forward(master, X, emulate)
    d = out[:, :N_USED] - np.asarray(Y, dtype=np.float64).reshape(n, N_USED)
    loss = float(np.sum(d * d))
    dz3 = np.zeros((n, N_OUT))
    dz3[:, :N_USED] = 2.0 * d / n
    dz3b = r(dz3)
    dz2 = (dz3b @ r(W3).T) * r(gelu_d(z2))
    dz2b = r(dz2)
    dz1 = (dz2b @ r(W2).T) * r(gelu_d(z1))
    dz1b = r(dz1)
    g = np.zeros(N_PARAMS)
    gW1 = x.T @ dz1b
    gW1[N_IN - 1, :] = 0.0
    gW3 = a2.T @ dz3b
    gW3[:, N_USED:] = 0.0
    gb3 = dz3.sum(axis=0)
    gb3[N_USED:] = 0.0
    g[OFF_W1:OFF_W2] = gW1.ravel()
    g[OFF_W2:OFF_W3] = (a1.T @ dz2b).ravel()
    g[OFF_W3:OFF_B1] = gW3.ravel()
    g[OFF_B1:OFF_B2] = dz1.sum(axis=0)
    g[OFF_B2:OFF_B3] = dz2.sum(axis=0)
    g[OFF_B3:N_PARAMS] = gb3
    return loss / n, g


def used_mask():
    m = np.ones(N_PARAMS, dtype=bool)
    m[OFF_W1:OFF_W2] = (np.arange(N_IN * N_HID) // N_HID) < N_IN - 1
    m[OFF_W3:OFF_B1] = (np.arange(N_HID * N_OUT) % N_OUT) < N_USED
    m[OFF_B3:N_PARAMS] = np.arange(N_OUT) < N_USED
    return m


def adamw(master, grad, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
    """One bias-corrected AdamW update (decoupled decay on the weight matrices only); returns new arrays."""
    used = used_mask()
    w = np.asarray(master, dtype=np.float64).copy()
    m = np.asarray(m, dtype=np.float64).copy()
    v = np.asarray(v, dtype=np.float64).copy()
    g = np.where(used, grad, 0.0)
    m[used] = beta1 * m[used] + (1 - beta1) * g[used]
    v[used] = beta2 * v[used] + (1 - beta2) * g[used] ** 2
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    decay = np.zeros(N_PARAMS, dtype=bool)
    decay[:OFF_B1] = True
    w = np.where(used & decay, w - lr * weight_decay * w, w)
    w = np.where(used, w - lr * mh / (np.sqrt(vh) + eps), w)
    return w, m, v
