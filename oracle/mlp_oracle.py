"""TEST INFRASTRUCTURE ONLY: CPU restatement of the calibration surrogate's
multilayer perceptron (include/dem_surrogate.h), in numpy FP64.

With bf16=True it rounds to BF16 at exactly the points where the GPU stores
BF16 (normalised inputs, weights, hidden activations, output and hidden
gradients), so the GPU's forward outputs and gradients can be compared with
it at FP32-accumulation accuracy; with bf16=False it is the plain FP64
network whose backward pass the tests pin with central finite differences.
The reference has no surrogate, so this oracle is pinned by those
finite-difference checks, not by reference vectors.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

NI, NH, NO = 4, 256, 3
SHAPES = [("W1", (NH, NI)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NH)), ("b3", (NH,)),
          ("W4", (NO, NH)), ("b4", (NO,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(flat: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = np.asarray(flat[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SHAPES])


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(np.isnan(f), np.nan, out)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(flat, x, norm, bf16_points: bool = True):
    """norm = (in_mean, in_std, out_mean, out_std); returns (y_normalised, cache)."""
    r = bf16 if bf16_points else (lambda a: np.asarray(a, np.float64))
    P = unpack(flat)
    xin = r((np.asarray(x, np.float64) - norm[0]) / norm[1])
    W = {k: r(P[k]) for k in ("W1", "W2", "W3", "W4")}
    z1 = xin @ W["W1"].T + P["b1"]
    h1 = r(gelu(z1))
    z2 = h1 @ W["W2"].T + P["b2"]
    h2 = r(gelu(z2))
    z3 = h2 @ W["W3"].T + P["b3"]
    h3 = r(gelu(z3))
    y = h3 @ W["W4"].T + P["b4"]
    return y, dict(xin=xin, W=W, z1=z1, h1=h1, z2=z2, h2=h2, z3=z3, h3=h3)


def loss_and_grad(flat, x, t, norm, bf16_points: bool = True):
    """Mean squared error over the batch and the 3 normalised outputs, and its
    gradient as a flat vector."""
    r = bf16 if bf16_points else (lambda a: np.asarray(a, np.float64))
    y, c = forward(flat, x, norm, bf16_points)
    n = len(x)
    tn = (np.asarray(t, np.float64) - norm[2]) / norm[3]
    d = y - tn
    loss = float(np.mean(d * d))
    dy = r(2.0 * d / (3.0 * n))
    g = {}
    g["W4"] = dy.T @ c["h3"]
    g["b4"] = dy.sum(0)
    dz3 = r((dy @ c["W"]["W4"]) * gelu_grad(c["z3"]))
    g["W3"] = dz3.T @ c["h2"]
    g["b3"] = dz3.sum(0)
    dz2 = r((dz3 @ c["W"]["W3"]) * gelu_grad(c["z2"]))
    g["W2"] = dz2.T @ c["h1"]
    g["b2"] = dz2.sum(0)
    dz1 = r((dz2 @ c["W"]["W2"]) * gelu_grad(c["z1"]))
    g["W1"] = dz1.T @ c["xin"]
    g["b1"] = dz1.sum(0)
    return loss, pack(g)


def he_uniform(seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in SHAPES:
        if name.startswith("W"):
            a = np.sqrt(6.0 / shape[1])
            d[name] = rng.uniform(-a, a, size=shape)
        else:
            d[name] = np.zeros(shape)
    return pack(d)
