"""CPU restatement of the evaporation surrogate's network (test infrastructure: only the tests use it).

The network of ice_b200/csrc/ice_mlp.cuh: 7 inputs -> 4 hidden layers of 128 with SiLU -> 2 outputs,
its FP32 parameters flat in the library's order (for each layer l: W_l [out][in] row-major, then b_l).
`forward`/`backward` are float64 (the gradient check of the library's FP32 training kernels);
`forward_bf16` rounds where the library's tensor-core inference rounds: the inputs, the weights and
the layer-0 bias (folded into the weights) to BF16, every hidden activation to BF16 after SiLU, FP32
accumulation and biases of layers 1-4. The network and the loss are this project's own (the reference
evaluates its closure directly: Lib_Evaporation.f90:145-261); nothing here restates reference code.
"""
from __future__ import annotations

import numpy as np

IN, H, OUT, NL = 7, 128, 2, 5


def dims(l):
    return (IN if l == 0 else H), (OUT if l == NL - 1 else H)


def offsets():
    o, out = 0, []
    for l in range(NL):
        i, n = dims(l)
        out.append((o, o + i * n))          # W_l at o, b_l at o + i n
        o += i * n + n
    return out, o


OFFS, NPARAM = offsets()


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    layers = []
    for l, (ow, ob) in enumerate(OFFS):
        i, n = dims(l)
        layers.append((w[ow:ow + i * n].reshape(n, i), w[ob:ob + n]))
    return layers


def silu(z):
    return z / (1.0 + np.exp(-z))


def forward(w, x):
    """float64 forward: returns the outputs and the per-layer (input, pre-activation) pairs."""
    a = np.asarray(x, dtype=np.float64)
    cache = []
    for l, (W, b) in enumerate(unpack(w)):
        z = a @ W.T + b
        cache.append((a, z))
        a = silu(z) if l < NL - 1 else z
    return a, cache


def loss_grad(w, x, t):
    """Mean-square loss over all n x 2 outputs and its gradient with respect to the flat parameters."""
    y, cache = forward(w, x)
    t = np.asarray(t, dtype=np.float64)
    d = y - t
    loss = float(np.mean(d * d))
    g = np.zeros(NPARAM)
    dz = 2.0 * d / d.size
    layers = unpack(w)
    for l in range(NL - 1, -1, -1):
        a_in, z = cache[l]
        if l < NL - 1:
            s = 1.0 / (1.0 + np.exp(-z))
            dz = dz * s * (1.0 + z * (1.0 - s))
        W, _ = layers[l]
        ow, ob = OFFS[l]
        g[ow:ow + W.size] = (dz.T @ a_in).reshape(-1)
        g[ob:ob + W.shape[0]] = dz.sum(axis=0)
        dz = dz @ W
    return loss, g


def bf16(v):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(v, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_bf16(w, x):
    """The tensor-core inference as the library rounds it (FP32 sums in float64 here)."""
    layers = unpack(w)
    a = bf16(x)
    for l, (W, b) in enumerate(layers):
        if l == 0:
            z = a @ bf16(W).T + bf16(b)
        else:
            z = a @ bf16(W).T + b.astype(np.float32).astype(np.float64)
        a = bf16(silu(z)) if l < NL - 1 else z
    return a


def glorot(seed=0):
    rng = np.random.default_rng(seed)
    w = np.zeros(NPARAM, dtype=np.float32)
    for l, (ow, ob) in enumerate(OFFS):
        i, n = dims(l)
        a = np.sqrt(6.0 / (i + n))
        w[ow:ow + i * n] = rng.uniform(-a, a, i * n)
        w[ob:ob + n] = rng.uniform(-0.1, 0.1, n)
    return w
