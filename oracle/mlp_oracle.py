"""CPU (numpy, FP64) forward and backward of the density-guess MLP: the
checker of the BF16 tensor-core kernels.  TEST INFRASTRUCTURE ONLY.

Inputs are the same BF16-rounded operands the kernels see, so the only
differences left are FP32-vs-FP64 accumulation order and the BF16 rounding
of hidden activations and of dZ inside the kernels.
"""
import numpy as np


def _identity(a):
    return a


def forward(x, Ws, bs, rnd=_identity):
    """Layers y = act(x W^T + b), ReLU on all but the last.  ``rnd`` rounds
    the hidden activations the way the kernels store them (BF16).  Returns
    the output and the per-layer (input, pre-activation) pairs."""
    h = x
    cache = []
    for i, (W, b) in enumerate(zip(Ws, bs)):
        z = h @ W.T + b
        cache.append((h, z))
        h = z if i == len(Ws) - 1 else rnd(np.maximum(z, 0.))
    return h, cache


def backward(dy, Ws, cache, rnd=_identity):
    """Gradients (dWs, dbs) of a loss with output gradient dy; ``rnd`` rounds
    dZ where the kernels feed it to the tensor cores (BF16)."""
    g = dy
    dWs, dbs = [None] * len(Ws), [None] * len(Ws)
    for i in reversed(range(len(Ws))):
        h, z = cache[i]
        dz = g if i == len(Ws) - 1 else g * (z > 0)
        dbs[i] = dz.sum(axis=0)
        dzr = rnd(dz)
        dWs[i] = dzr.T @ h
        g = dzr @ Ws[i]
    return dWs, dbs
