"""FP64 NumPy restatement of the cut-refinement MLP (16 -> 64 -> 64 -> 64 -> 1; hidden activation
GELU in its sigmoid form x sigma(1.702 x), Hendrycks & Gimpel 2016, or ReLU) with its weighted
binary-cross-entropy gradient.  `act` is "gelu" or "relu" (the library's ARC_MLP_ACT_GELU = 0,
ARC_MLP_ACT_RELU = 1; an int is accepted too).
TEST INFRASTRUCTURE ONLY: the checker for the tensor-core kernels in
antiradiancecuts_b200/csrc/mlp.cu; the product never imports it.

Parameter layout (FP32 master copy of the library): W1[64][16], b1[64], W2[64][64], b2[64],
W3[64][64], b3[64], w4[64], b4.
"""
from __future__ import annotations

import math

import numpy as np

SIZES = [("W1", (64, 16)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)), ("W3", (64, 64)), ("b3", (64,)),
         ("w4", (64,)), ("b4", (1,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SIZES])


_S = 0.851  # 1.702 / 2


def gelu(x):
    """x/2 (1 + tanh(s x)) = x sigma(1.702 x)"""
    return 0.5 * x * (1.0 + np.tanh(_S * x))


def gelu_grad(x):
    th = np.tanh(_S * x)
    return 0.5 * (1.0 + th) + 0.5 * x * _S * (1.0 - th * th)


def relu(x):
    return np.maximum(x, 0.0)


def relu_grad(x):
    return (x > 0.0).astype(np.float64)


def _relu(act) -> bool:
    if act in ("relu", 1):
        return True
    if act in ("gelu", 0):
        return False
    raise ValueError(f"unknown activation {act!r}")


def _act(act):
    return (relu, relu_grad) if _relu(act) else (gelu, gelu_grad)


def forward(p, x, act="gelu"):
    P = unpack(p)
    f, _ = _act(act)
    x = np.asarray(x, np.float64)
    z1 = x @ P["W1"].T + P["b1"]
    h1 = f(z1)
    z2 = h1 @ P["W2"].T + P["b2"]
    h2 = f(z2)
    z3 = h2 @ P["W3"].T + P["b3"]
    h3 = f(z3)
    y = h3 @ P["w4"] + P["b4"][0]
    return y, (x, z1, h1, z2, h2, z3, h3)


def loss_and_grad(p, x, labels, weights=None, loss="bce", act="gelu"):
    """sum(w * loss(y, label)) / sum(w) and its gradient w.r.t. the parameters; loss "bce"
    (binary cross-entropy on the logit y) or "squared" ((y - label)^2)."""
    y, (x, z1, h1, z2, h2, z3, h3) = forward(p, x, act)
    _, fg = _act(act)
    lab = np.asarray(labels, np.float64)
    w = np.ones_like(lab) if weights is None else np.asarray(weights, np.float64)
    ws = w.sum()
    P = unpack(p)
    if loss == "squared":
        loss_v = float(np.sum(w * (y - lab) ** 2) / ws)
        dy = w * 2.0 * (y - lab) / ws
    else:
        loss_v = float(np.sum(w * (np.maximum(y, 0) - y * lab + np.log1p(np.exp(-np.abs(y))))) / ws)
        dy = w * (1.0 / (1.0 + np.exp(-y)) - lab) / ws
    loss = loss_v
    g = {"w4": h3.T @ dy, "b4": np.array([dy.sum()])}
    dz3 = np.outer(dy, P["w4"]) * fg(z3)
    g["W3"], g["b3"] = dz3.T @ h2, dz3.sum(0)
    dz2 = (dz3 @ P["W3"]) * fg(z2)
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = (dz2 @ P["W2"]) * fg(z1)
    g["W1"], g["b1"] = dz1.T @ x, dz1.sum(0)
    return loss, pack(g)


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_bf16(p, x, act="gelu"):
    """The network as the tensor-core kernels evaluate it.  GELU: the activation's constants folded
    into the parameters (s W1, W2 / 2, W3 / 2 rounded to BF16 from FP32 products; s b in FP32;
    w4 / (2 s)), the folded activation g(z) = z + z tanh(z).  ReLU: W1, W2, W3 rounded to BF16,
    the rest FP32 as stored.  Both: BF16 inputs and hidden activations h1, h2; FP64 otherwise
    (accumulation, biases, activation, the 64 -> 1 layer)."""
    P = unpack(p)
    if _relu(act):
        W1, W2, W3 = (bf16(np.asarray(P[k], np.float32)) for k in ("W1", "W2", "W3"))
        b1, b2, b3, w4 = (np.asarray(P[k], np.float32).astype(np.float64) for k in ("b1", "b2", "b3", "w4"))
        h = bf16(x)
        h1 = bf16(relu(h @ W1.T + b1))
        h2 = bf16(relu(h1 @ W2.T + b2))
        h3 = relu(h2 @ W3.T + b3)
        return h3 @ w4 + np.float64(np.float32(P["b4"][0]))
    s32 = np.float32(_S)
    out32 = np.float32(0.5) / s32

    def f32(a):
        return np.asarray(a, np.float32)

    def g(z):
        return z + z * np.tanh(z)

    W1 = bf16(s32 * f32(P["W1"]))
    W2 = bf16(np.float32(0.5) * f32(P["W2"]))
    W3 = bf16(np.float32(0.5) * f32(P["W3"]))
    b1, b2, b3 = (np.float64(s32 * f32(P[k])) for k in ("b1", "b2", "b3"))
    w4 = np.float64(out32 * f32(P["w4"]))
    h = bf16(x)
    h1 = bf16(g(h @ W1.T + b1))
    h2 = bf16(g(h1 @ W2.T + b2))
    h3 = g(h2 @ W3.T + b3)
    return h3 @ w4 + np.float64(np.float32(P["b4"][0]))
