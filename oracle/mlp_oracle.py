"""ORACLE / TEST INFRASTRUCTURE ONLY: the surrogate perceptron in FP64 on the CPU (numpy), the checker of the GPU's
forward pass and gradients.  The reference has no such network (its AI chapter fits a 3-layer tanh MLP to XVA
adjustments, src/ai/surrogate.cpp), so this is a project-written statement of the standard MLP algebra:

    z1 = x W1^T + b1, h1 = silu(z1), z2 = h1 W2^T + b2, h2 = silu(z2), z3 = h2 W3^T + b3, h3 = silu(z3),
    pred = h3 . w4 + b4, loss = mean (pred - y)^2 on standardised inputs and targets.

With emulate=True values are rounded to bf16 exactly where the GPU stores them (the standardised inputs, the
matrix weights, the pre-activations and activations, the back-propagated dZ), so what remains is FP32 against
FP64 accumulation; with emulate=False it is the exact FP64 network on the same parameters.  Its gradient is
checked against finite differences of its own loss (tests/test_mlp_oracle.py).
"""
from __future__ import annotations

import numpy as np

IN, HID = 16, 128


def bf16(a):
    u = np.ascontiguousarray(a, np.float32).view(np.uint32)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32) << 16
    return r.view(np.float32).astype(np.float64)


def _split(p):
    p = np.asarray(p, np.float64)
    o, out = 0, []
    for shape in ((HID, IN), (HID,), (HID, HID), (HID,), (HID, HID), (HID,), (HID,), (1,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def standardise(x, y, scaling):
    sc = np.asarray(scaling, np.float32)
    xs = (np.asarray(x, np.float32) - sc[:16]) * sc[16:32]
    yy = None if y is None else (np.asarray(y, np.float64) - float(sc[32])) / float(sc[33])
    return xs, yy


def forward(p, scaling, x, emulate=True):
    W1, b1, W2, b2, W3, b3, w4, b4 = _split(p)
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    X = r(standardise(x, None, scaling)[0])
    z1 = X @ r(W1).T + b1
    h1 = r(silu(z1))
    z2 = h1 @ r(W2).T + b2
    h2 = r(silu(z2))
    z3 = h2 @ r(W3).T + b3
    h3 = r(silu(z3))
    pred = h3 @ w4 + b4[0]
    return {"X": X, "z1": z1, "h1": h1, "z2": z2, "h2": h2, "z3": z3, "h3": h3, "pred": pred}


def predict(p, scaling, x, emulate=True):
    return forward(p, scaling, x, emulate)["pred"] * float(scaling[33]) + float(scaling[32])


def loss_and_grads(p, scaling, x, y, emulate=True):
    W1, b1, W2, b2, W3, b3, w4, b4 = _split(p)
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    f = forward(p, scaling, x, emulate)
    ys = standardise(x, y, scaling)[1]
    n = len(ys)
    d = f["pred"] - ys
    loss = float(np.mean(d * d))
    dout = 2.0 * d / n
    z1, z2, z3 = (r(f[k]) for k in ("z1", "z2", "z3"))  # the GPU keeps the pre-activations in bf16
    dw4 = f["h3"].T @ dout
    db4 = np.array([dout.sum()])
    dz3 = r(np.outer(dout, w4) * silu_grad(z3))
    dW3, db3 = dz3.T @ f["h2"], dz3.sum(0)
    dz2 = r((dz3 @ r(W3)) * silu_grad(z2))
    dW2, db2 = dz2.T @ f["h1"], dz2.sum(0)
    dz1 = r((dz2 @ r(W2)) * silu_grad(z1))
    dW1, db1 = dz1.T @ f["X"], dz1.sum(0)
    return loss, np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3, dw4, db4])
