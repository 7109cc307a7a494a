"""float64 restatement of the GPU scorer's arithmetic (test oracle only).

Same operand roundings as the kernels in ``coldcore_b200/csrc/mlp.cu``:
inputs, hidden activations, W1 / W2 and the backward deltas dz2 / dz1 are
rounded to bfloat16 (round to nearest even) where the kernels round them;
every sum is exact float64 here (FP32 on the device), so gradients agree to
FP32-accumulation error."""
import numpy as np

N_IN, N_HID = 32, 128


def bf16(a):
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + N_IN * N_HID].reshape(N_IN, N_HID); o += N_IN * N_HID
    b1 = p[o:o + N_HID]; o += N_HID
    W2 = p[o:o + N_HID * N_HID].reshape(N_HID, N_HID); o += N_HID * N_HID
    b2 = p[o:o + N_HID]; o += N_HID
    w3 = p[o:o + N_HID]; o += N_HID
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    x = bf16(X)
    h1 = bf16(np.maximum(x @ bf16(W1) + b1, 0))
    h2 = bf16(np.maximum(h1 @ bf16(W2) + b2, 0))
    y = h2 @ w3 + b3
    return x, h1, h2, y


def grad(p, X, T):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    x, h1, h2, y = forward(p, X)
    n = len(T)
    dy = (1 / (1 + np.exp(-y)) - np.asarray(T, dtype=np.float64)) / n
    gw3 = h2.T @ dy
    gb3 = dy.sum()
    dz2 = bf16(np.where(h2 > 0, dy[:, None] * w3[None, :], 0.0))
    gW2 = h1.T @ dz2
    gb2 = dz2.sum(axis=0)
    dz1 = bf16(np.where(h1 > 0, dz2 @ bf16(W2).T, 0.0))
    gW1 = x.T @ dz1
    gb1 = dz1.sum(axis=0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])


def loss(p, X, T):
    y = forward(p, X)[3]
    T = np.asarray(T, dtype=np.float64)
    return float(np.mean(np.logaddexp(0, y) - T * y))
