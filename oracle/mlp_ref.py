"""CPU FP64 restatement of the surrogate network (test infrastructure only).

The oracle for the GPU training kernels of elasticscattering_b200/csrc/es_mlp.cu:
the same network (5 -> 256 x 4 -> 2, GELU, one member) evaluated in FP64, with
values rounded to BF16 exactly where the GPU path stores BF16 (inputs, hidden
weights, hidden activations that feed the next hidden layer, back-propagated
gradients of the hidden layers) and kept exact where the GPU keeps FP32 (the
256 -> 2 head's weights and activations, the loss gradient), so that the only
differences left are the GPU's FP32 accumulation and FP32 GELU.
Only tests use it. No part of the reference corresponds to it: the surrogate has
no reference counterpart.
"""
from __future__ import annotations

import math

import numpy as np

DIMS = (5, 256, 256, 256, 256, 2)


def bf16(a) -> np.ndarray:
    """Round to the nearest BF16 (ties to even) via FP32, returned as FP64."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split_params(p: np.ndarray):
    """Flat FP32 parameters of one member -> [(W [N][K], b [N])] per layer."""
    out, o = [], 0
    for k, n in zip(DIMS[:-1], DIMS[1:]):
        w = p[o:o + n * k].reshape(n, k)
        o += n * k
        b = p[o:o + n]
        o += n
        out.append((w, b))
    assert o == p.size
    return out


def param_count() -> int:
    return sum(k * n + n for k, n in zip(DIMS[:-1], DIMS[1:]))


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def _exact(a) -> np.ndarray:
    return np.asarray(a, dtype=np.float64)


def forward(p: np.ndarray, x: np.ndarray, rounding: bool = True):
    """Output [M][2] and the per-layer (A_in, Z) pairs. rounding=False skips every
    BF16 rounding (the plain FP64 network, for finite-difference checks)."""
    bf16_ = bf16 if rounding else _exact
    layers = split_params(np.asarray(p, dtype=np.float64))
    a = bf16_(x)
    cache = []
    last = len(layers) - 1
    for li, (w, b) in enumerate(layers):
        # the hidden layers take BF16 weights; the output head FP32 weights
        z = a @ (w if li == last else bf16_(w)).T + b
        cache.append((a, z))
        if li + 1 < last:
            a = bf16_(gelu(z))
        elif li + 1 == last:
            a = gelu(z)  # the head's FP32 activations
    return z, cache


def loss_and_grads(p: np.ndarray, x: np.ndarray, y: np.ndarray, rounding: bool = True):
    """Mean squared error and its gradient w.r.t. the flat parameters."""
    bf16_ = bf16 if rounding else _exact
    layers = split_params(np.asarray(p, dtype=np.float64))
    out, cache = forward(p, x, rounding)
    m = x.shape[0]
    d = out - y
    loss = float(np.mean(d * d))
    dz = 2.0 / (m * DIMS[-1]) * d  # FP32 on the GPU: no BF16 rounding
    grads = [None] * len(layers)
    last = len(layers) - 1
    for li in range(last, -1, -1):
        a, _ = cache[li]
        w, _ = layers[li]
        grads[li] = (dz.T @ a, dz.sum(axis=0))
        if li == 0:
            break
        _, z_prev = cache[li - 1]
        dz = bf16_((dz @ (w if li == last else bf16_(w))) * gelu_grad(z_prev))
    flat = []
    for gw, gb in grads:
        flat += [gw.ravel(), gb.ravel()]
    return loss, np.concatenate(flat)
