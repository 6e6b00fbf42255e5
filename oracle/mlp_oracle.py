"""CPU oracle of the learned sizer's network — TEST INFRASTRUCTURE.

Imported only by tests/ as the checker of the GPU forward / backward /
training kernels (gpudbmetalcodegen_b200/csrc/kernels/sizer_mlp.cu); never
by the product package.

The reference has no learned component (it sizes tables by an exact max-key
pass, codegen/execution/max_key_symbols.cpp:188-235), so this oracle states
the network itself: 16 -> 64 -> 64 -> 64 -> 2, ReLU hidden layers, linear
output, mean squared error over all outputs, weights rounded to BF16
(round to nearest even) before use, activations and accumulation in float64
here (FP32 on the GPU). Parameter layout (9,538 floats): W1[64][16] b1[64]
W2[64][64] b2[64] W3[64][64] b3[64] W4[2][64] b4[2], weights out-major.
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

SHAPES: List[Tuple[str, Tuple[int, ...]]] = [
    ("W1", (64, 16)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)),
    ("W3", (64, 64)), ("b3", (64,)), ("W4", (2, 64)), ("b4", (2,)),
]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)
assert NPARAMS == 9538


def bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 -> float32, round to nearest even (finite inputs)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray) -> Dict[str, np.ndarray]:
    out, off = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = p[off:off + n].reshape(shape)
        off += n
    return out


def pack(d: Dict[str, np.ndarray]) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], dtype=np.float64).reshape(-1) for name, _ in SHAPES])


def forward(params: np.ndarray, X: np.ndarray, quantize: bool = True):
    w = bf16_round(params).astype(np.float64) if quantize else np.asarray(params, dtype=np.float64)
    P = {k: v.astype(np.float64) for k, v in unpack(w).items()}
    x = np.asarray(X, dtype=np.float64)
    h1 = np.maximum(x @ P["W1"].T + P["b1"], 0.0)
    h2 = np.maximum(h1 @ P["W2"].T + P["b2"], 0.0)
    h3 = np.maximum(h2 @ P["W3"].T + P["b3"], 0.0)
    y = h3 @ P["W4"].T + P["b4"]
    return y, (x, h1, h2, h3, P)


def loss_and_grads(params: np.ndarray, X: np.ndarray, Y: np.ndarray, quantize: bool = True):
    """MSE over n samples x 2 outputs and its gradient w.r.t. the parameters
    (evaluated at the BF16-rounded weights, as the GPU kernels do)."""
    y, (x, h1, h2, h3, P) = forward(params, X, quantize)
    t = np.asarray(Y, dtype=np.float64)
    n = x.shape[0]
    diff = y - t
    loss = float((diff ** 2).sum() / (n * 2))
    dy = 2.0 * diff / (n * 2)
    g = {"W4": dy.T @ h3, "b4": dy.sum(0)}
    d3 = (dy @ P["W4"]) * (h3 > 0)
    g["W3"], g["b3"] = d3.T @ h2, d3.sum(0)
    d2 = (d3 @ P["W3"]) * (h2 > 0)
    g["W2"], g["b2"] = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ P["W2"]) * (h1 > 0)
    g["W1"], g["b1"] = d1.T @ x, d1.sum(0)
    return loss, pack(g)


def adam_step(w, m, v, g, step: int, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
    """One Adam update of the FP32 master weights (bias-corrected)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    w = w - lr * (m / c1) / (np.sqrt(v / c2) + eps)
    return w, m, v
