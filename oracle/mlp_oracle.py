"""CPU oracle for the learned cost model -- TEST INFRASTRUCTURE ONLY.

The tests load this module to check the CUDA training kernels
(rqs-svg_b200/csrc/cost_model.cu): it restates, in float64 numpy, the same
MLP 6 -> 64 -> 64 -> 1 with ReLU activations, the mean squared error and its
gradient with respect to every parameter, in the parameter layout the
library uses: W1[64x6], b1[64], W2[64x64], b2[64], W3[64], b3[1].

The model has no counterpart in the reference simulator (its fusion planner
is an addition of the B200 build); parity here is against this restatement.
"""

import numpy as np

IN, HID = 6, 64
SIZES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (1, HID)), ("b3", (1,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    out, off = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = p[off:off + n].reshape(shape)
        off += n
    return out


def forward(params, x):
    w = unpack(params)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = np.maximum(z2, 0.0)
    y = h2 @ w["W3"].T + w["b3"]
    return y[:, 0], (z1, h1, z2, h2)


def loss_and_gradients(params, x, t):
    """Mean squared error and its gradient (flat, library layout)."""
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    w = unpack(params)
    y, (z1, h1, z2, h2) = forward(params, x)
    B = len(t)
    dy = 2.0 * (y - t) / B
    dW3 = dy[None, :] @ h2
    db3 = np.array([dy.sum()])
    dh2 = dy[:, None] * w["W3"][0][None, :]
    dz2 = dh2 * (z2 > 0)
    dW2 = dz2.T @ h1
    db2 = dz2.sum(axis=0)
    dh1 = dz2 @ w["W2"]
    dz1 = dh1 * (z1 > 0)
    dW1 = dz1.T @ x
    db1 = dz1.sum(axis=0)
    grads = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return float(np.mean((y - t) ** 2)), grads
