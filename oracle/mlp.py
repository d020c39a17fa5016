"""Float64 numpy forward/backward of the temperature MLP.  Test infrastructure only.

Restates the network of the learned Newton guess (8 -> 64 -> 64 -> 1, tanh,
mean-squared-error loss) so the device gradients can be checked.  With
``emulate_bf16`` the operands the device feeds to its bf16 tensor cores
(inputs, hidden activations, weights, pre-activation gradients) are rounded
to bf16 first, so only float32 accumulation differences remain.
"""

from __future__ import annotations

import numpy as np


def bf16(a):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a32 = np.asarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(p, x, emulate_bf16=False):
    r = bf16 if emulate_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    xb = r(x)
    w1, w2 = r(p["w1"]), r(p["w2"])
    z1 = xb @ w1.T + p["b1"]
    h1 = np.tanh(z1)
    z2 = r(h1) @ w2.T + p["b2"]
    h2 = np.tanh(z2)
    y = h2 @ p["w3"] + p["b3"]
    return {"x": xb, "h1": h1, "h2": h2, "y": y}


def loss_and_grad(p, x, t, emulate_bf16=False):
    r = bf16 if emulate_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    n = x.shape[0]
    f = forward(p, x, emulate_bf16)
    res = f["y"] - t
    loss = np.mean(res ** 2)
    dy = 2 * res / n
    g = {"b3": dy.sum(), "w3": f["h2"].T @ dy}
    dz2 = np.outer(dy, p["w3"]) * (1 - f["h2"] ** 2)
    g["b2"] = dz2.sum(axis=0)
    g["w2"] = r(dz2).T @ r(f["h1"])
    dh1 = r(dz2) @ r(p["w2"])
    dz1 = dh1 * (1 - f["h1"] ** 2)
    g["b1"] = dz1.sum(axis=0)
    g["w1"] = r(dz1).T @ f["x"]
    return loss, g
