"""CPU restatement of the learned-guess MLP (test infrastructure only).

The numpy forward and backward pass of the network the tensor-core kernels
run (billardballraytracing3d_b200/csrc/guess_mlp.cu), with the kernels'
roundings made explicit: inputs, weights and hidden activations rounded to
BF16 (round to nearest even), products accumulated in FP64 here (FP32 on the
device), GELU in its tanh form.  Tests compare the device's forward outputs,
loss and every parameter gradient with this.
"""
from __future__ import annotations

import numpy as np

GELU_C = 0.7978845608028654   # sqrt(2 / pi)
GELU_A = 0.044715


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """float -> BF16 bit pattern (uint16), round to nearest even."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r


def bf16_round(x: np.ndarray) -> np.ndarray:
    """float -> nearest BF16 value, as float64."""
    b = bf16_bits(x).astype(np.uint32) << 16
    return b.view(np.float32).astype(np.float64)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_A * z ** 3)))


def gelu_grad(z):
    th = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + th) + 0.5 * z * (1.0 - th * th) * GELU_C * (1.0 + 3.0 * GELU_A * z * z)
