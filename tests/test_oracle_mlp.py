"""The near-contact network oracle (oracle/mlp.py) against finite
differences and its own bf16 emulation (CPU only)."""
import numpy as np

from oracle import mlp


def test_fp64_gradient_matches_finite_differences():
    p = mlp.init_params(1).astype(np.float64)
    rng = np.random.default_rng(0)
    x = rng.normal(size=(9, 16))
    x[:, 10:] = 0.0
    y = rng.normal(size=(9, 16))
    w = np.r_[np.ones(12), np.zeros(4)]
    g, _ = mlp.gradient(p, x, y, w, mode="fp64")
    h = 1e-6
    for i in rng.choice(mlp.NPARAM, 24, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp.gradient(pp, x, y, w, "fp64")[1] - mlp.gradient(pm, x, y, w, "fp64")[1]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_bf16_rounding_and_emulation_error():
    a = np.array([1.0, 1.00390625, 1.0078125, 1.01171875, -3.14159, 0.0], np.float32)
    b = mlp.bf16(a)
    # ties to even at the 8-bit mantissa boundary
    assert b[1] == 1.0 and b[3] == np.float32(1.015625) and b[5] == 0.0
    assert abs(b[4] - a[4]) <= 2.0 ** -8 * abs(a[4])
    p = mlp.init_params(2)
    rng = np.random.default_rng(1)
    x = rng.normal(size=(64, 16)).astype(np.float32)
    o16, _, _ = mlp.forward(p, x, "bf16")
    o64, _, _ = mlp.forward(p.astype(np.float64), x.astype(np.float64), "fp64")
    assert np.abs(o16 - o64).max() <= 3e-2 * np.abs(o64).max()
