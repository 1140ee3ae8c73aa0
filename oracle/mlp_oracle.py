"""CPU restatement of the learned face-flux network.  TEST INFRASTRUCTURE ONLY.

The network (16 -> 128 -> 128 -> 128 -> 8, GELU hidden layers) has no
counterpart in the reference; this module is the oracle the tensor-core
inference and training kernels are checked against.  It reproduces their
rounding points, with products and sums in float64 (the kernels accumulate in
FP32) and biases unrounded:

- ``forward`` / ``loss_and_grad`` (the training kernels): inputs, weights and
  hidden activations rounded to BF16 (round to nearest even);
- ``infer`` (the tensor-core inference kernel): inputs and weights rounded to
  FP16, each hidden pre-activation rounded to FP16 before its GELU and twice
  the GELU's value rounded to FP16 (the next layer's weights halved).

Parameter vector order: W1[128x16], b1[128], W2[128x128], b2[128],
W3[128x128], b3[128], W4[8x128], b4[8] (row-major).
"""
from __future__ import annotations

import numpy as np

NIN, NH, NOUT = 16, 128, 8
SHAPES = [(NH, NIN), (NH,), (NH, NH), (NH,), (NH, NH), (NH,), (NOUT, NH), (NOUT,)]
NPARAM = sum(int(np.prod(s)) for s in SHAPES)
C_GELU = 0.7978845608028654


def bf16(x):
    """Round to the nearest BF16 value (ties to even); returns float32."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def f16(x):
    """Round to the nearest FP16 value (ties to even) by way of FP32, as the
    kernel rounds its FP32 values; returns float32."""
    return np.asarray(x, np.float32).astype(np.float16).astype(np.float32)


def unpack(p):
    p = np.asarray(p, np.float64).ravel()
    out, o = [], 0
    for s in SHAPES:
        k = int(np.prod(s))
        out.append(p[o:o + k].reshape(s))
        o += k
    return out


def pack(parts):
    return np.concatenate([np.asarray(a, np.float64).ravel() for a in parts])


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C_GELU * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    u = C_GELU * (x + 0.044715 * x ** 3)
    t = np.tanh(u)
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C_GELU * (1.0 + 3 * 0.044715 * x * x)


def forward(p, X, keep=False):
    """Outputs (n x 8); with keep, also the pre-activations and the BF16
    layer inputs for the backward pass."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)
    Ws = [bf16(W).astype(np.float64) for W in (W1, W2, W3, W4)]
    a = bf16(X).astype(np.float64)
    ins, pre = [a], []
    for W, b in zip(Ws[:3], (b1, b2, b3)):
        z = a @ W.T + b
        pre.append(z)
        a = bf16(gelu(z)).astype(np.float64)
        ins.append(a)
    y = a @ Ws[3].T + b4
    return (y, ins, pre, Ws) if keep else y


def infer(p, X):
    """Outputs (n x 8) of the inference kernel's rounded network, in the
    kernel's own form: each hidden layer stores twice its GELU and the next
    layer's weights are halved before rounding (W2, W3, W4)."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)
    a = f16(X).astype(np.float64)
    z = a @ f16(W1).astype(np.float64).T + b1
    for W, b in ((W2, b2), (W3, b3), (W4, b4)):
        x = f16(z).astype(np.float64)
        a = f16(2.0 * gelu(x)).astype(np.float64)
        z = a @ f16(0.5 * W).astype(np.float64).T + b
    return z


def loss_and_grad(p, X, Y, wt=None):
    """Mean squared error over outputs (optionally weighted per output) and
    its gradient with respect to every parameter (the backward pass of the
    same rounded network; gradients flow through the BF16 roundings as
    identities)."""
    y, ins, pre, Ws = forward(p, X, keep=True)
    n = X.shape[0]
    w = np.ones(NOUT) if wt is None else np.asarray(wt, np.float64)
    r = y - Y
    loss = float((w * r * r).sum() / (n * NOUT))
    g = 2.0 * w * r / (n * NOUT)
    grads = [None] * 8
    grads[6] = g.T @ ins[3]
    grads[7] = g.sum(0)
    d = g @ Ws[3]
    for L in (2, 1, 0):
        dz = d * gelu_grad(pre[L])
        grads[2 * L] = dz.T @ ins[L]
        grads[2 * L + 1] = dz.sum(0)
        d = dz @ Ws[L]
    return loss, pack(grads)


def init_params(seed=0):
    """He-style uniform initialisation (seeded)."""
    rng = np.random.default_rng(seed)
    parts = []
    for s in SHAPES:
        if len(s) == 2:
            lim = np.sqrt(6.0 / s[1])
            parts.append(rng.uniform(-lim, lim, s))
        else:
            parts.append(np.zeros(s))
    return pack(parts).astype(np.float32)
