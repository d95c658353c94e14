"""FP64 CPU restatement of the surrogate network — TEST INFRASTRUCTURE ONLY.

The network of include/qm_surrogate.h (32 -> 4 x (256, GELU) -> 8) in numpy double precision:
forward pass, mean-squared-error loss on normalised labels and its gradient by backpropagation.
With `bf16=True` the weights, the normalised inputs and every hidden activation are rounded to
BF16 (round to nearest even) where the device rounds them, so the device's products can be checked
against the same operands. Only tests/ import this module.
"""

import numpy as np

DIMS = (32, 256, 256, 256, 256, 8)
WEIGHTS = sum(DIMS[k + 1] * DIMS[k] + DIMS[k + 1] for k in range(5))


def bf16(x):
    """Rounds to BF16 (nearest, ties to even) and returns float64."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    a = (a + 0x7FFF + ((a >> 16) & 1)) & 0xFFFF0000
    return a.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    ws, bs, o = [], [], 0
    for k in range(5):
        n = DIMS[k + 1] * DIMS[k]
        ws.append(p[o:o + n].reshape(DIMS[k + 1], DIMS[k]))
        o += n
        bs.append(p[o:o + DIMS[k + 1]])
        o += DIMS[k + 1]
    q = WEIGHTS
    scales = dict(in_shift=p[q:q + 32], in_scale=p[q + 32:q + 64], out_shift=p[q + 64:q + 72],
                  out_scale=p[q + 72:q + 80])
    return ws, bs, scales


GELU_C, GELU_A = np.sqrt(2.0 / np.pi), 0.044715


def gelu(z):
    """GELU in its tanh form (Hendrycks and Gimpel, 2016), as the device computes it."""
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_A * z ** 3)))


def gelu_grad(z):
    t = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * z * z)


def _forward(ws, bs, x, round_):
    zs, hs = [], [x]
    h = x
    for k in range(5):
        z = h @ round_(ws[k]).T + bs[k]
        zs.append(z)
        if k < 4:
            h = round_(gelu(z))
            hs.append(h)
    return zs, hs


def normalised_inputs(params, features, bf16_round=False):
    _, _, s = unpack(params)
    x = (np.asarray(features, np.float64) - s["in_shift"]) * s["in_scale"]
    return bf16(x) if bf16_round else x


def forward(params, features, bf16_round=False):
    """A_boundary (dB) per row."""
    ws, bs, s = unpack(params)
    round_ = bf16 if bf16_round else (lambda a: a)
    x = normalised_inputs(params, features, bf16_round)
    zs, _ = _forward(ws, bs, x, round_)
    return zs[-1] * s["out_scale"] + s["out_shift"]


def gradients(params, features, labels, bf16_round=False):
    """(gradient of the loss w.r.t. the packed weights and biases, loss); the loss is the mean of
    ((A - out_shift) / out_scale - y)^2 over rows and bands."""
    ws, bs, s = unpack(params)
    round_ = bf16 if bf16_round else (lambda a: a)
    x = normalised_inputs(params, features, bf16_round)
    y = (np.asarray(labels, np.float64) - s["out_shift"]) / s["out_scale"]
    zs, hs = _forward(ws, bs, x, round_)
    n = len(x)
    d = zs[-1] - y
    loss = float(np.mean(d * d))
    dz = 2.0 * d / (n * 8)
    grads = [None] * 5
    for k in range(4, -1, -1):
        gw = dz.T @ hs[k]
        gb = dz.sum(axis=0)
        grads[k] = (gw, gb)
        if k > 0:
            dz = (dz @ round_(ws[k])) * gelu_grad(zs[k - 1])
    out = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return out, loss
