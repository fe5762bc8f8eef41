"""Oracle (test infrastructure only): the turn-leaf value network's forward and backward pass
on the CPU in float64, with the activations rounded to bfloat16 at the points where the
device stores them (inputs, weights, pre-activations Z, activations H, output gradient dY,
hidden gradients dZ), so the device's gradients can be checked against it.

Network: x (2706) -> 4 x [Linear(1024) + GELU (erf form)] -> Linear(2652); loss = mean
squared error over all outputs of the batch. Weights W[l] are (fan_out, fan_in).
"""
import math

import numpy as np


def bf16(a):
    """Round float values to bfloat16 (round to nearest even), returned as float64."""
    a = np.asarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def inputs(ranges, boards, scalars):
    """[n][2706]: both ranges, the 4 board cards as 52 0/1 values, pot and stack scaled."""
    n = len(boards)
    x = np.zeros((n, 2706))
    x[:, :2652] = ranges.reshape(n, 2652)
    for i, b in enumerate(boards):
        for c in range(52):
            x[i, 2652 + c] = (int(b) >> c) & 1
    x[:, 2704:2706] = scalars
    return x


def forward_backward(W, b, x, target):
    """Loss and gradients (dW, db) of the bf16-rounded network; W, b lists of 5 arrays."""
    n = x.shape[0]
    h = bf16(x)
    Wr = [bf16(w) for w in W]
    Zs, Hs = [], [h]
    for l in range(4):
        z = Hs[-1] @ Wr[l].T + b[l]
        Zs.append(bf16(z))           # the stored pre-activation
        Hs.append(bf16(gelu(z)))     # GELU of the unrounded pre-activation
    y = Hs[-1] @ Wr[4].T + b[4]
    d = y - target
    loss = float(np.mean(d * d))
    dy = bf16(2.0 * d / d.size)
    dW = [None] * 5
    db = [None] * 5
    dW[4] = dy.T @ Hs[4]
    db[4] = dy.sum(axis=0)
    g = dy @ Wr[4]
    for l in range(3, -1, -1):
        dz = bf16(g * gelu_grad(Zs[l]))
        dW[l] = dz.T @ Hs[l]
        db[l] = dz.sum(axis=0)
        g = dz @ Wr[l]
    return loss, dW, db, y
