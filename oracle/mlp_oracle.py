"""CPU oracle for the learned warm start's network (numpy).

TEST INFRASTRUCTURE ONLY: the tests compare the library's tensor-core
forward and backward kernels with this restatement.  It mirrors the device's
roundings: activations and activation gradients are rounded to BF16 (round
to nearest even) where the device stores them as matrix operands; weights
are the BF16 copies of the FP32 parameters; every sum is in float64 (the
device's are FP32 in another order, hence a tolerance).

Forward:  h1 = bf16(relu(x W1 + b1)), h2 = bf16(relu(h1 W2 + b2)),
          y = h2 W3 + b3.
Loss:     mean over n rows and 3 outputs of (y - t)^2.
Backward: dy = bf16(2 (y - t) / 3n), dz2 = bf16((dy W3^T) [h2 > 0]),
          dz1 = bf16((dz2 W2^T) [h1 > 0]); dW3 = h2^T dy, db3 = sum dy,
          dW2 = h1^T dz2, db2 = sum dz2, dW1 = x^T dz1, db1 = sum dz1.
"""
from __future__ import annotations

import numpy as np

INPUTS, HIDDEN, OUTPUTS = 32, 128, 3
SHAPES = [("w1", (INPUTS, HIDDEN)), ("b1", (HIDDEN,)), ("w2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
          ("w3", (HIDDEN, OUTPUTS)), ("b3", (OUTPUTS,))]


def bf16(a) -> np.ndarray:
    """Round float32 values to BF16 (nearest, ties to even), as float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def bf16_bits(a) -> np.ndarray:
    """BF16 bit patterns (uint16) of float32 values."""
    return (bf16(a).astype(np.float32).view(np.uint32) >> 16).astype(np.uint16)


def from_bits(bits) -> np.ndarray:
    return (np.asarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def split(flat, dtype=np.float32):
    out, k = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[k:k + n], dtype).reshape(shape)
        k += n
    return out


def _r(rounding):
    return bf16 if rounding else (lambda a: np.asarray(a, np.float64))


def forward(flat, x_bits, rounding: bool = True, x=None):
    """y, h1, h2.  rounding=False: every value in float64 (x given as
    floats), for checking the formulas themselves."""
    r = _r(rounding)
    p = split(flat) if rounding else split(flat, np.float64)
    x = from_bits(x_bits) if x is None else np.asarray(x, np.float64)
    h1 = r(np.maximum(x @ r(p["w1"]) + p["b1"], 0.0).astype(np.float32 if rounding else np.float64))
    h2 = r(np.maximum(h1 @ r(p["w2"]) + p["b2"], 0.0).astype(np.float32 if rounding else np.float64))
    y = h2 @ r(p["w3"]) + p["b3"]
    return y, h1, h2


def gradient(flat, x_bits, target, rounding: bool = True, x=None):
    r = _r(rounding)
    p = split(flat) if rounding else split(flat, np.float64)
    x = from_bits(x_bits) if x is None else np.asarray(x, np.float64)
    y, h1, h2 = forward(flat, x_bits, rounding, x)
    n = len(x)
    t = np.asarray(target, np.float64)
    loss = float(np.mean((y - t) ** 2))
    f = np.float32 if rounding else np.float64
    dy = r((2.0 * (y - t) / (3.0 * n)).astype(f))
    dz2 = r(((dy @ r(p["w3"]).T) * (h2 > 0)).astype(f))
    dz1 = r(((dz2 @ r(p["w2"]).T) * (h1 > 0)).astype(f))
    g = {"w3": h2.T @ dy, "b3": dy.sum(0), "w2": h1.T @ dz2, "b2": dz2.sum(0), "w1": x.T @ dz1, "b1": dz1.sum(0)}
    return np.concatenate([g[name].reshape(-1) for name, _ in SHAPES]), loss
