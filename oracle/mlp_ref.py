"""CPU oracle of the learned Newton predictor's network (test infrastructure only).

A per-node MLP: features -> 128 GELU -> 128 GELU -> outputs.  The GPU kernels multiply bf16
operands on the tensor cores with fp32 accumulation; this restatement applies the same bf16
roundings to the same operands (weights, layer inputs, and the backward operands dY / dZ) and
accumulates in float64, so a comparison measures the GPU's accumulation error rather than adding
its own.  GELU is the tanh form.  Used by the tests to check the GPU forward pass, the gradients
of the backward pass and the Adam step; the product path never imports it.

Strut has no learned predictor; the network is the one the north-star configuration specifies
(2 hidden layers of 128 units, GELU, bf16 weights with fp32 accumulation).
"""
from __future__ import annotations

import numpy as np

GELU_C = np.float32(0.7978845608028654)  # sqrt(2 / pi)
GELU_A = np.float32(0.044715)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 to bfloat16 (round to nearest even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def gelu(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.float32)
    t = np.tanh(GELU_C * (z + GELU_A * z * z * z))
    return (np.float32(0.5) * z * (np.float32(1.0) + t)).astype(np.float32)


def gelu_grad(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.float32)
    t = np.tanh(GELU_C * (z + GELU_A * z * z * z))
    dt = (np.float32(1.0) - t * t) * GELU_C * (np.float32(1.0) + np.float32(3.0) * GELU_A * z * z)
    return (np.float32(0.5) * (np.float32(1.0) + t) + np.float32(0.5) * z * dt).astype(np.float32)


def _mm(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return (a.astype(np.float64) @ b.astype(np.float64)).astype(np.float32)


def forward(params: dict, x: np.ndarray):
    """params: W1 (K x H), b1 (H), W2 (H x H), b2 (H), W3 (H x O), b3 (O), float32 masters.
    x: (N, K) float32 features.  Returns (y, cache)."""
    xb = bf16(x)
    z1 = _mm(xb, bf16(params["W1"])) + params["b1"]
    h1b = bf16(gelu(z1))
    z2 = _mm(h1b, bf16(params["W2"])) + params["b2"]
    h2b = bf16(gelu(z2))
    y = _mm(h2b, bf16(params["W3"])) + params["b3"]
    return y.astype(np.float32), dict(xb=xb, z1=z1, h1b=h1b, z2=z2, h2b=h2b)


def loss_and_grads(params: dict, x: np.ndarray, t: np.ndarray):
    """Mean squared error over all outputs and its gradients (with the GPU backward's roundings)."""
    y, c = forward(params, x)
    n = y.size
    d = (y - t).astype(np.float32)
    loss = float(np.mean(d.astype(np.float64) ** 2))
    dy = (np.float32(2.0 / n) * d).astype(np.float32)
    dyb = bf16(dy)
    g = {}
    g["W3"] = _mm(c["h2b"].T, dyb)
    g["b3"] = dy.astype(np.float64).sum(0).astype(np.float32)
    dz2 = (_mm(dyb, bf16(params["W3"]).T) * gelu_grad(c["z2"])).astype(np.float32)
    dz2b = bf16(dz2)
    g["W2"] = _mm(c["h1b"].T, dz2b)
    g["b2"] = dz2.astype(np.float64).sum(0).astype(np.float32)
    dz1 = (_mm(dz2b, bf16(params["W2"]).T) * gelu_grad(c["z1"])).astype(np.float32)
    dz1b = bf16(dz1)
    g["W1"] = _mm(c["xb"].T, dz1b)
    g["b1"] = dz1.astype(np.float64).sum(0).astype(np.float32)
    return loss, g


def adam_step(params: dict, grads: dict, m: dict, v: dict, step: int, lr=1e-3, b1=0.9, b2=0.999,
              eps=1e-8):
    """One Adam update of the float32 masters (step counts from 1)."""
    c1 = np.float32(1.0 - b1 ** step)
    c2 = np.float32(1.0 - b2 ** step)
    for k in params:
        m[k] = (np.float32(b1) * m[k] + np.float32(1.0 - b1) * grads[k]).astype(np.float32)
        v[k] = (np.float32(b2) * v[k] + np.float32(1.0 - b2) * grads[k] * grads[k]).astype(np.float32)
        mh = m[k] / c1
        vh = v[k] / c2
        params[k] = (params[k] - np.float32(lr) * mh / (np.sqrt(vh) + np.float32(eps))).astype(np.float32)
    return params, m, v
