"""CPU oracle (test infrastructure only) of the learned EDrSVD parameter predictor.

Restates in NumPy FP64 what the library's predictor kernels compute, so the GPU forward and
backward passes and one Adam step can be checked against it:

* the network: 8 inputs -> 64 (ReLU) -> 64 (ReLU) -> 3 (linear), parameters packed as
  W1 (64 x 8, row-major), b1 (64), W2 (64 x 64), b2 (64), W3 (3 x 64), b3 (3);
* the loss: mean over the batch of the summed squared error of the 3 outputs;
* Adam (Kingma & Ba 2015, bias-corrected, beta1 0.9, beta2 0.999, eps 1e-8).

The reference has no learned component (its EDrSVD takes rank, oversampling and power-iteration
count as fixed arguments, ttdec_gpu_float_rsvd_lu_half.cu:797-798), so there is nothing of the
reference to pin this against; it is checked by finite differences instead.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 8, 64, 3
SIZES = [("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
         ("W3", (N_OUT, N_HID)), ("b3", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SIZES])


def forward(p: np.ndarray, x: np.ndarray):
    """Outputs (n x 3) and the activations the backward pass needs."""
    w = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = np.maximum(z2, 0.0)
    y = h2 @ w["W3"].T + w["b3"]
    return y, (x, z1, h1, z2, h2)


def loss_and_grad(p: np.ndarray, x: np.ndarray, t: np.ndarray):
    """Mean squared error over the batch (summed over outputs) and its gradient (packed)."""
    w = unpack(p)
    y, (x, z1, h1, z2, h2) = forward(p, x)
    n = x.shape[0]
    r = y - np.asarray(t, dtype=np.float64)
    loss = float(np.sum(r * r) / n)
    dy = 2.0 * r / n
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dh2 = (dy @ w["W3"]) * (z2 > 0)
    g["W2"] = dh2.T @ h1
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ w["W2"]) * (z1 > 0)
    g["W1"] = dh1.T @ x
    g["b1"] = dh1.sum(0)
    return loss, pack(g)


def adam_step(p, g, m, v, step: int, lr: float, b1=0.9, b2=0.999, eps=1e-8):
    """One bias-corrected Adam update (step counts from 1); returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v


def init_params(seed: int) -> np.ndarray:
    """He-uniform weights, zero biases (any initialisation works for the checks)."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in SIZES:
        if name.startswith("W"):
            lim = np.sqrt(6.0 / shape[1])
            d[name] = rng.uniform(-lim, lim, size=shape)
        else:
            d[name] = np.zeros(shape)
    return pack(d)
