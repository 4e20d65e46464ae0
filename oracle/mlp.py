"""CPU restatement of the learned SHAKE warm-start network (test
infrastructure only: the checker of heddle_b200's tensor-core MLP kernels).

The network has no counterpart in the reference (its SHAKE starts from zero
multipliers, kernels/shake.cu:108-348); this module states the arithmetic the
device kernels perform so that their forward pass and gradients can be
checked: FP64 everywhere except that the operands the tensor cores read are
rounded to bfloat16 (round to nearest even) at the same points:

  z1 = bf(x) bf(W1)^T + b1,  h1 = tanh z1
  z2 = bf(h1) bf(W2)^T + b2, h2 = tanh z2,  y = h2 . w3 + b3
  dy = 2 (y - t) / B, dz2 = dy w3 (1 - h2^2)
  dh1 = bf(dz2) bf(W2), dz1 = dh1 (1 - h1^2)
  dW2 = bf(dz2)^T bf(h1), dW1 = bf(dz1)^T bf(x)
  db1 = sum dz1, db2 = sum dz2, dw3 = sum dy h2, db3 = sum dy
with x standardised ((x - mean) * inv_std) and t divided by the target scale.
Parameters are packed W1 [64][8], b1 [64], W2 [64][64], b2 [64], w3 [64], b3.
"""

from __future__ import annotations

import numpy as np

NF, HID = 8, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * NF
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + HID
NPARAM = OFF_B3 + 1


def bf16(x, enable: bool = True) -> np.ndarray:
    """Round to bfloat16 (nearest even) and return as float64."""
    x = np.asarray(x, dtype=np.float64)
    if not enable:
        return x
    a = x.astype(np.float32).view(np.uint32).astype(np.uint64)
    a = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return a.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(HID, NF), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(HID, HID),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def forward(p, x, mean=None, inv_std=None, t_scale: float = 1.0, use_bf16: bool = True):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    if mean is not None:
        x = (x - np.asarray(mean, dtype=np.float32)) * np.asarray(inv_std, dtype=np.float32)
    z1 = bf16(x, use_bf16) @ bf16(W1, use_bf16).T + b1
    h1 = np.tanh(z1)
    z2 = bf16(h1, use_bf16) @ bf16(W2, use_bf16).T + b2
    h2 = np.tanh(z2)
    y = h2 @ w3 + b3
    return y * t_scale, (x, h1, h2, y)


def gradients(p, x, t, mean=None, inv_std=None, t_scale: float = 1.0, use_bf16: bool = True):
    """(gradient of the mean squared error in normalised units, loss)."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    _, (xs, h1, h2, y) = forward(p, x, mean, inv_std, 1.0, use_bf16)
    t = np.asarray(t, dtype=np.float64) / t_scale
    B = len(t)
    e = y - t
    loss = float((e * e).sum() / B)
    dy = 2.0 * e / B
    dz2 = dy[:, None] * w3[None, :] * (1.0 - h2 * h2)
    dh1 = bf16(dz2, use_bf16) @ bf16(W2, use_bf16)
    dz1 = dh1 * (1.0 - h1 * h1)
    g = np.zeros(NPARAM)
    g[OFF_W2:OFF_B2] = (bf16(dz2, use_bf16).T @ bf16(h1, use_bf16)).reshape(-1)
    g[OFF_W1:OFF_B1] = (bf16(dz1, use_bf16).T @ bf16(xs, use_bf16)).reshape(-1)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    g[OFF_W3:OFF_B3] = (dy[:, None] * h2).sum(0)
    g[OFF_B3] = dy.sum()
    return g, loss
