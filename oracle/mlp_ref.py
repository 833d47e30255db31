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


# ---- the network ------------------------------------------------------------
N_IN, N_H, N_OUT, N_EMB, N_GEO = 64, 128, 16, 32, 9

# Flat FP32 parameter layout shared with the device (guess_mlp.cu):
# W0 [128][64], b0 [128], W1 [128][128], b1, W2 [128][128], b2, W3 [16][128], b3 [16], E [P][32]
SHAPES = (("W0", (N_H, N_IN)), ("b0", (N_H,)), ("W1", (N_H, N_H)), ("b1", (N_H,)),
          ("W2", (N_H, N_H)), ("b2", (N_H,)), ("W3", (N_OUT, N_H)), ("b3", (N_OUT,)))


def offsets():
    off, o = {}, 0
    for name, shp in SHAPES:
        off[name] = o
        o += int(np.prod(shp))
    off["E"] = o
    return off


N_NET = offsets()["E"]


def unpack(params: np.ndarray, n_patches: int):
    off = offsets()
    p = {name: params[off[name]:off[name] + int(np.prod(shp))].reshape(shp).astype(np.float64)
         for name, shp in SHAPES}
    p["E"] = params[off["E"]:off["E"] + n_patches * N_EMB].reshape(n_patches, N_EMB).astype(np.float64)
    return p


def pack(p: dict) -> np.ndarray:
    parts = [np.asarray(p[name], np.float64).ravel() for name, _ in SHAPES] + [np.asarray(p["E"]).ravel()]
    return np.concatenate(parts)


def init_params(n_patches: int, seed: int = 0) -> np.ndarray:
    """Scaled-uniform weights, zero biases, small embeddings; padding rows
    and columns (inputs >= 41, outputs >= 4) zero."""
    rng = np.random.default_rng(seed)
    p = {}
    fan_in = {"W0": 41, "W1": N_H, "W2": N_H, "W3": N_H}
    for name, shp in SHAPES:
        if name.startswith("W"):
            lim = np.sqrt(6.0 / (fan_in[name] + shp[0]))
            p[name] = rng.uniform(-lim, lim, shp)
        else:
            p[name] = np.zeros(shp)
    p["W0"][:, N_GEO + N_EMB:] = 0.0
    p["W3"][4:, :] = 0.0
    p["E"] = rng.normal(0.0, 0.1, (n_patches, N_EMB))
    return pack(p).astype(np.float32)


def forward_backward(params, n_patches, feat, pid, tgt, lbl, rounding=True):
    """Loss, per-row outputs (u, v, s, logit) and parameter gradients (same
    flat layout as params) of one batch, as the device computes them.

    loss = (1/B) sum_rows [ lbl * ((u-u*)^2 + (v-v*)^2 + (s-s*)^2) + BCE(logit, lbl) ]
    With rounding=False every BF16 rounding is skipped (plain FP64 network,
    for the finite-difference check of this function itself)."""
    rd = bf16_round if rounding else (lambda a: np.asarray(a, np.float64))
    p = unpack(np.asarray(params), n_patches)
    B = feat.shape[0]
    x = np.zeros((B, N_IN))
    x[:, :N_GEO] = feat
    x[:, N_GEO:N_GEO + N_EMB] = p["E"][pid]
    X = rd(x)
    W = [rd(p[f"W{l}"]) for l in range(4)]
    b = [p[f"b{l}"] for l in range(4)]
    Z1 = X @ W[0].T + b[0]; H1 = rd(gelu(Z1))
    Z2 = H1 @ W[1].T + b[1]; H2 = rd(gelu(Z2))
    Z3 = H2 @ W[2].T + b[2]; H3 = rd(gelu(Z3))
    Z4 = H3 @ W[3].T + b[3]
    out = Z4[:, :4]
    y = np.asarray(lbl, np.float64)
    t = np.asarray(tgt, np.float64)
    diff = out[:, :3] - t
    logit = out[:, 3]
    bce = np.maximum(logit, 0.0) - logit * y + np.log1p(np.exp(-np.abs(logit)))
    loss = np.sum(y * np.sum(diff * diff, axis=1) + bce) / B
    d4 = np.zeros((B, N_OUT))
    d4[:, :3] = 2.0 * y[:, None] * diff / B
    d4[:, 3] = (1.0 / (1.0 + np.exp(-logit)) - y) / B
    g = {"b3": d4.sum(0)}
    G4 = rd(d4)
    g["W3"] = G4.T @ H3
    dH3 = G4 @ W[3]
    dZ3 = dH3 * gelu_grad(Z3); g["b2"] = dZ3.sum(0); G3 = rd(dZ3)
    g["W2"] = G3.T @ H2
    dH2 = G3 @ W[2]
    dZ2 = dH2 * gelu_grad(Z2); g["b1"] = dZ2.sum(0); G2 = rd(dZ2)
    g["W1"] = G2.T @ H1
    dH1 = G2 @ W[1]
    dZ1 = dH1 * gelu_grad(Z1); g["b0"] = dZ1.sum(0); G1 = rd(dZ1)
    g["W0"] = G1.T @ X
    dX = G1 @ W[0]
    gE = np.zeros((n_patches, N_EMB))
    np.add.at(gE, pid, dX[:, N_GEO:N_GEO + N_EMB])
    g["E"] = gE
    return loss, out, pack(g)
