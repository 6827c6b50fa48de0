"""BF16 tensor-core MLP kernels against the FP64 numpy oracle (needs a B200)."""
import numpy as np
import pytest

from oracle import mlp_oracle

pytestmark = pytest.mark.gpu


def _bf16(a):
    import torch
    return torch.as_tensor(a, dtype=torch.float32).to(torch.bfloat16).float().numpy().astype(np.float64)


def test_forward_backward_match_oracle(cuda):
    import torch
    from byteqc_b200.learned.model import DensityMLP, LAYERS
    model = DensityMLP(seed=3)
    rng = np.random.default_rng(0)
    M = 64
    x = rng.normal(size=(M, LAYERS[0][1]))
    y = model.forward(torch.as_tensor(x, dtype=torch.float32, device=cuda), keep=True)
    Ws = [_bf16(w.cpu().numpy()) for w in model.W]
    bs = [b.cpu().numpy().astype(np.float64) for b in model.b]
    ref, cache = mlp_oracle.forward(_bf16(x), Ws, bs, rnd=_bf16)
    y = y.cpu().numpy()
    assert np.abs(y - ref).max() < 2e-3 * np.abs(ref).max()
    dy = rng.normal(size=y.shape) / M
    grads = model.backward(torch.as_tensor(dy, dtype=torch.float32, device=cuda))
    dWs, dbs = mlp_oracle.backward(dy, Ws, cache, rnd=_bf16)
    for g, r in zip(grads, dWs + dbs):
        g = g.cpu().numpy()
        rel = np.abs(g - r).max() / max(np.abs(r).max(), 1e-12)
        assert rel < 5e-3, rel


def test_training_reduces_loss(cuda):
    import torch
    from byteqc_b200.learned.model import DensityMLP, LAYERS
    from byteqc_b200.learned.features import OUT_DIM
    rng = np.random.default_rng(1)
    M = 256
    x = torch.as_tensor(rng.normal(size=(M, LAYERS[0][1])), dtype=torch.float32, device=cuda)
    t = torch.as_tensor(np.tanh(rng.normal(size=(M, OUT_DIM))), dtype=torch.float32, device=cuda)
    model = DensityMLP(seed=0)
    losses = []
    for _ in range(60):
        y = model.forward(x, keep=True)
        d = y - t
        losses.append(float((d * d).mean()))
        model.adam(model.backward(2 * d / d.numel()), lr=3e-3)
    assert losses[-1] < 0.5 * losses[0]
