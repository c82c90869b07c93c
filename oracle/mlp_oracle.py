"""CPU oracle of the C2P guess network (test infrastructure only).

Forward and backward of the 8 -> 64 -> 64 -> 64 -> 2 ReLU network of
method_b200/csrc/mlp.cuh in NumPy FP64.  With ``bf16=True`` it rounds to
bfloat16 at the points where the device kernels store BF16 (inputs, weights,
hidden activations, output and hidden gradients), so the device gradient
can be compared at FP32-accumulation tolerance; with ``bf16=False`` it is
plain FP64 and is itself checked against central finite differences.

Parameter layout (packed, FP32 on the device): W1[16][64] (rows 8..15 zero),
b1[64], W2[64][64], b2[64], W3[64][64], b3[64], W4[64][8] (cols 2..7 zero),
b4[8]; W is [in][out].
"""
from __future__ import annotations

import numpy as np

IN, INP, H, OUT, OUTP = 8, 16, 64, 2, 8
SHAPES = [("W1", (INP, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
          ("b3", (H,)), ("W4", (H, OUTP)), ("b4", (OUTP,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(P):
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(P[o:o + n], dtype=np.float64).reshape(shp)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    d = {}
    for name, shp in SHAPES:
        if name.startswith("b"):
            d[name] = rng.uniform(-0.1, 0.1, shp)
        else:
            fan = shp[0] if name != "W1" else IN
            d[name] = rng.uniform(-np.sqrt(6 / fan), np.sqrt(6 / fan), shp)
    d["W1"][IN:, :] = 0.0
    d["W4"][:, OUT:] = 0.0
    d["b4"][OUT:] = 0.0
    return pack(d)


def loss_and_grad(P, x, t, bf=True):
    """Mean-squared error over n samples and its gradient (packed layout)."""
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    p = unpack(P)
    W = {k: (r(v) if k.startswith("W") else v) for k, v in p.items()}
    n = x.shape[0]
    X = np.zeros((n, INP))
    X[:, :IN] = x
    X = r(X)
    z1 = X @ W["W1"] + p["b1"]
    h1 = r(np.maximum(z1, 0.0))
    z2 = h1 @ W["W2"] + p["b2"]
    h2 = r(np.maximum(z2, 0.0))
    z3 = h2 @ W["W3"] + p["b3"]
    h3 = r(np.maximum(z3, 0.0))
    y = h3 @ W["W4"] + p["b4"]
    e = np.zeros((n, OUTP))
    e[:, :OUT] = y[:, :OUT] - t
    denom = n * OUT
    loss = float(np.sum(e * e) / denom)
    dY = r(2.0 * e / denom)
    g = {}
    g["W4"] = h3.T @ dY
    g["b4"] = dY.sum(0)
    dZ3 = r((dY @ W["W4"].T) * (h3 > 0))
    g["W3"] = h2.T @ dZ3
    g["b3"] = dZ3.sum(0)
    dZ2 = r((dZ3 @ W["W3"].T) * (h2 > 0))
    g["W2"] = h1.T @ dZ2
    g["b2"] = dZ2.sum(0)
    dZ1 = r((dZ2 @ W["W2"].T) * (h1 > 0))
    g["W1"] = X.T @ dZ1
    g["b1"] = dZ1.sum(0)
    return loss, pack(g), y[:, :OUT]
