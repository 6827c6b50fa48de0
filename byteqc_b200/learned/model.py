"""The density-guess MLP on the device: 3 hidden layers of width 256,
BF16 weights and activations, FP32 accumulation, trained with the library's
own forward, backward and Adam kernels (BQCmlp_*).

    x (FEAT_DIM) -> 256 -> 256 -> 256 -> OUT_DIM,  ReLU between layers.
"""
import ctypes

import numpy as np
import torch

from .. import lib as _libmod
from .features import FEAT_DIM, OUT_DIM

WIDTH = 256


def layers(out_dim=OUT_DIM):
    return [(WIDTH, FEAT_DIM), (WIDTH, WIDTH), (WIDTH, WIDTH), (out_dim, WIDTH)]


LAYERS = layers()


def _vp(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class DensityMLP:
    def __init__(self, seed=0, device='cuda', out_dim=OUT_DIM):
        self.lib = _libmod.load_library()
        self.device = torch.device(device)
        self.layers = layers(out_dim)
        rng = np.random.default_rng(seed)
        self.W, self.b = [], []
        for n, k in self.layers:
            w = rng.normal(size=(n, k)) * np.sqrt(2. / k)
            self.W.append(torch.as_tensor(w, dtype=torch.float32, device=self.device))
            self.b.append(torch.zeros(n, dtype=torch.float32, device=self.device))
        self._sync_bf16()
        self.m = [torch.zeros_like(t) for t in self.W + self.b]
        self.v = [torch.zeros_like(t) for t in self.W + self.b]
        self.step = 0

    def _sync_bf16(self):
        self.Wb = [w.to(torch.bfloat16) for w in self.W]

    # -- state -----------------------------------------------------------------
    def state(self):
        return {'W%d' % i: w.cpu().numpy() for i, w in enumerate(self.W)} | \
               {'b%d' % i: b.cpu().numpy() for i, b in enumerate(self.b)}

    def load(self, state):
        self.layers = layers(int(state['W%d' % (len(self.layers) - 1)].shape[0]))
        for i in range(len(self.layers)):
            self.W[i] = torch.as_tensor(state['W%d' % i], dtype=torch.float32, device=self.device)
            self.b[i] = torch.as_tensor(state['b%d' % i], dtype=torch.float32, device=self.device)
        self._sync_bf16()
        return self

    # -- forward / backward ----------------------------------------------------
    def forward(self, x, keep=False):
        """x: (M, FEAT_DIM) float tensor, M a multiple of 16.  Returns the FP32
        output (M, OUT_DIM); with keep, the activations for backward."""
        M = x.shape[0]
        h = x.to(torch.bfloat16).contiguous()
        acts, zs = [h], []
        for i, (n, k) in enumerate(self.layers):
            last = i == len(self.layers) - 1
            z = torch.empty((M, n), dtype=torch.float32, device=self.device)
            yb = None if last else torch.empty((M, n), dtype=torch.bfloat16, device=self.device)
            err = self.lib.BQCmlp_linear_fwd(_vp(h), _vp(self.Wb[i]), _vp(self.b[i]), _vp(z), None,
                                             _vp(yb), M, n, k, 0 if last else 1, _stream())
            if err:
                raise RuntimeError('BQCmlp_linear_fwd failed (%d)' % err)
            zs.append(z)
            if not last:
                h = yb
                acts.append(h)
        out = zs[-1]
        if keep:
            self._cache = (acts, zs)
        return out

    def backward(self, dy):
        """dy: (M, OUT_DIM) FP32 gradient of the loss w.r.t. the output.
        Returns FP32 gradients [dW...] + [db...]."""
        acts, zs = self._cache
        M = dy.shape[0]
        dWs, dbs = [None] * len(self.layers), [None] * len(self.layers)
        g = dy.contiguous()
        for i in reversed(range(len(self.layers))):
            n, k = self.layers[i]
            last = i == len(self.layers) - 1
            dW = torch.empty((n, k), dtype=torch.float32, device=self.device)
            db = torch.empty(n, dtype=torch.float32, device=self.device)
            dx = torch.empty((M, k), dtype=torch.float32, device=self.device) if i > 0 else None
            dz = torch.empty((M, n), dtype=torch.bfloat16, device=self.device)
            err = self.lib.BQCmlp_linear_bwd(_vp(g), None if last else _vp(zs[i]), _vp(acts[i]),
                                             _vp(self.Wb[i]), _vp(dz), _vp(dx), _vp(dW), _vp(db),
                                             M, n, k, _stream())
            if err:
                raise RuntimeError('BQCmlp_linear_bwd failed (%d)' % err)
            dWs[i], dbs[i] = dW, db
            g = dx
        return dWs + dbs

    def adam(self, grads, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        params = self.W + self.b
        for j, (p, g) in enumerate(zip(params, grads)):
            wb = self.Wb[j] if j < len(self.W) else None
            err = self.lib.BQCmlp_adam(_vp(p), _vp(g), _vp(self.m[j]), _vp(self.v[j]), _vp(wb),
                                       p.numel(), lr, b1, b2, eps, self.step, _stream())
            if err:
                raise RuntimeError('BQCmlp_adam failed (%d)' % err)

    def predict(self, x):
        M = x.shape[0]
        Mp = (M + 15) // 16 * 16
        xp = torch.zeros((Mp, FEAT_DIM), dtype=torch.float32, device=self.device)
        xp[:M] = torch.as_tensor(x, dtype=torch.float32, device=self.device)
        return self.forward(xp)[:M]
