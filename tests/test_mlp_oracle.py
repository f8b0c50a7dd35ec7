"""The learned-proposal oracle: its backward pass against finite differences, BF16
rounding, and Adam (CPU only)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as M  # noqa: E402


def _batch(rng, n):
    X = rng.normal(0, 1, (n, M.IN))
    Y = rng.normal(0, 0.5, (n, M.NDIM))
    Mk = (rng.random((n, M.NDIM)) < 0.7).astype(np.float64)
    return X, Y, Mk


def test_bf16_rounding_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.14159265, 65504.0, 1e-30], np.float32)
    r = M.bf16(v)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to the even mantissa (1.0)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
    for x, y in zip(v, r):
        assert abs(y - x) <= abs(x) * 2 ** -8


def test_param_layout():
    assert M.param_count() == 672 * 256 + 256 + 2 * (256 * 256 + 256) + 256 * 64 + 64
    p = M.init_params(1)
    assert p.dtype == np.float32 and p.size == M.param_count()
    assert np.allclose(M.pack(M.unpack(p)), p)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = M.init_params(2).astype(np.float64)
    p += rng.normal(0, 0.01, p.size)          # nonzero biases
    X, Y, Mk = _batch(rng, 6)
    loss, g = M.loss_grad(p, X, Y, Mk, rnd=False)
    idx = rng.choice(p.size, 60, replace=False)
    # include bias entries of every layer
    offs = np.cumsum([0] + [int(np.prod(s)) for s in M.SHAPES])
    idx = np.concatenate([idx, offs[1:-1:2] + 3, [offs[-2] + 5]])
    h = 1e-5
    for i in idx:
        pp = p.copy(); pp[i] += h
        pm = p.copy(); pm[i] -= h
        fd = (M.loss_grad(pp, X, Y, Mk, rnd=False)[0] - M.loss_grad(pm, X, Y, Mk, rnd=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_logvar_clamp_stops_gradient():
    out = np.zeros((2, M.OUT))
    out[:, M.NDIM:2 * M.NDIM] = 10.0           # above the clamp
    _, d = M.loss_and_dout(out, np.ones((2, M.NDIM)), np.ones((2, M.NDIM)))
    assert np.all(d[:, M.NDIM:2 * M.NDIM] == 0.0)
    assert np.all(d[:, 2 * M.NDIM:] == 0.0)


def test_adam_reduces_loss():
    rng = np.random.default_rng(4)
    p = M.init_params(3)
    X, Y, Mk = _batch(rng, 64)
    m = np.zeros_like(p); v = np.zeros_like(p)
    l0 = M.loss_grad(p, X, Y, Mk)[0]
    for t in range(1, 31):
        _, g = M.loss_grad(p, X, Y, Mk)
        p, m, v = M.adam_step(p, g, m, v, t, 1e-3)
    assert M.loss_grad(p, X, Y, Mk)[0] < l0 - 0.1
