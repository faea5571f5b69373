"""The CPU restatement of the surrogate's network (oracle/mlp.py), checked before it checks the
library: its gradient against central differences, its BF16 rounding against torch's."""
import numpy as np

from oracle import mlp


def test_gradient_matches_central_differences():
    rng = np.random.default_rng(3)
    w = mlp.glorot(1).astype(np.float64)
    x = rng.normal(size=(16, mlp.IN))
    t = rng.normal(size=(16, mlp.OUT))
    _, g = mlp.loss_grad(w, x, t)
    for idx in rng.choice(mlp.NPARAM, 60, replace=False):
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[idx] += h
        wm[idx] -= h
        fd = (mlp.loss_grad(wp, x, t)[0] - mlp.loss_grad(wm, x, t)[0]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 + 1e-5 * abs(fd), (idx, fd, g[idx])


def test_bf16_rounding_matches_torch():
    import torch
    v = np.random.default_rng(0).normal(scale=10.0, size=4096).astype(np.float32)
    ref = torch.from_numpy(v).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(mlp.bf16(v), ref)
