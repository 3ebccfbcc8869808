"""CPU oracle of the near-contact correction network (test infrastructure).

Only tests/ and the smoke check import this module, as the checker of the
GPU network kernels; nothing in the product calls it.

The reference has no learned component, so there is no reference file to
follow: this is the plain restatement of the network the GPU kernels
evaluate and differentiate,
    A0 = x (16),  Z_l = A_{l-1} W_l^T,  A_l = silu(Z_l + b_l)  (l = 1, 2, 3),
    O = A3 W4^T + b4,
    L = (1/n) sum_rows sum_c colw[c] (O[c] - y[c])^2,
with W[out][in] and the same packed parameter order as the kernels.  Two
modes: exact float64 (checked against finite differences), and "bf16",
which rounds every tensor-core operand (weights, the input, activations and
the backpropagated dZ / dO) to bfloat16 (round to nearest even) and sums in
float32 like the FP32 accumulators of the kernels.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 16, 128, 16
SHAPES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)),
          ("b3", (HID,)), ("W4", (OUT, HID)), ("b4", (OUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)
assert NPARAM == 37264


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


def pack(d: dict, dtype=np.float32) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], dtype=dtype).reshape(-1) for name, _ in SHAPES])


def bf16(a: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 (round to nearest, ties to even) -> float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (r.astype(np.uint32) << 16).view(np.float32).reshape(a.shape)


def init_params(seed: int) -> np.ndarray:
    """He-uniform weights scaled for SiLU, zero biases, a small last layer
    (PCG64(seed))."""
    rng = np.random.Generator(np.random.PCG64(seed))
    d = {}
    for name, shape in SHAPES:
        if name.startswith("b"):
            d[name] = np.zeros(shape, np.float32)
        else:
            fan_in = shape[1]
            lim = np.sqrt(6.0 / fan_in) * (0.1 if name == "W4" else 1.0)
            d[name] = rng.uniform(-lim, lim, size=shape).astype(np.float32)
    return pack(d)


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params: np.ndarray, x: np.ndarray, mode: str = "bf16"):
    """Network output O[n][16] and the cache for backward."""
    q = bf16 if mode == "bf16" else (lambda a: a)
    dt = np.float32 if mode == "bf16" else np.float64
    P = {k: v.astype(dt) for k, v in unpack(np.asarray(params)).items()}
    a = q(np.asarray(x, dt))
    cache = {"A0": a}
    for l in (1, 2, 3):
        z = (a @ q(P[f"W{l}"]).T).astype(dt)
        cache[f"Z{l}"] = z
        a = q(_silu(z + P[f"b{l}"]).astype(dt))
        cache[f"A{l}"] = a
    o = (a @ q(P["W4"]).T + P["b4"]).astype(dt)
    return o, cache, P


def gradient(params: np.ndarray, x: np.ndarray, y: np.ndarray, colw: np.ndarray, mode: str = "bf16"):
    """(packed gradient, loss) of the weighted mean squared error."""
    q = bf16 if mode == "bf16" else (lambda a: a)
    dt = np.float32 if mode == "bf16" else np.float64
    o, c, P = forward(params, x, mode)
    n = x.shape[0]
    e = o - np.asarray(y, dt)
    w = np.asarray(colw, dt)
    loss = float(np.sum(w * e * e) / n)
    d = (2.0 * w * e / n).astype(dt)
    g = {"b4": d.sum(0)}
    dq = q(d)
    g["W4"] = (dq.T @ c["A3"]).astype(dt)
    da = (dq @ q(P["W4"])).astype(dt)
    for l in (3, 2, 1):
        dz = (da * _dsilu(c[f"Z{l}"] + P[f"b{l}"])).astype(dt)
        g[f"b{l}"] = dz.sum(0)
        dzq = q(dz)
        g[f"W{l}"] = (dzq.T @ c[f"A{l - 1}"]).astype(dt)
        if l > 1:
            da = (dzq @ q(P[f"W{l}"])).astype(dt)
    return pack(g, dt), loss
