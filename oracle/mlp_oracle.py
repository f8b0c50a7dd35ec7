"""CPU oracle of the learned move proposal (test infrastructure only).

The proposal network has no counterpart in the reference: it replaces the random draw of
`mutate_pose_tile` (reference src/cuda/mc.cu:146-256) with a sample from a Gaussian whose
mean and log-variance a small MLP predicts from the chain's current pose.  This module
restates, in float64 numpy, exactly the arithmetic the CUDA kernels perform:

* BF16 operands with wide accumulation: inputs, weights, hidden activations and the
  back-propagated pre-activation gradients are rounded to bfloat16 (round to nearest
  even) at the same points as on the GPU; products of BF16 values are exact in float64,
  so the oracle differs from the GPU only by the GPU's float32 summation order.
* Layers: 672 -> 256 -> 256 -> 256 -> 64, ReLU after each hidden layer.
* Output: mean[0:26], raw log-variance[26:52] (clamped to [-8, 4]); columns 52..63 unused.
* Loss: mean over samples of the masked Gaussian negative log-likelihood
  sum_d mask_d * 0.5 * (logvar_d + (y_d - mean_d)^2 * exp(-logvar_d)).
* Optimiser: Adam (Kingma & Ba 2015) on float32 master weights.

Parameter order (flat vector, the C ABI's layout): W1[672x256], b1[256], W2[256x256], b2,
W3[256x256], b3, W4[256x64], b4[64]; weight matrices row-major [in x out].
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 672, 256, 64
NDIM = 26                 # 6 rigid-body + up to 20 torsion move dimensions
NATOM_MAX, NMAP, TMAX = 80, 8, 20
LOGVAR_MIN, LOGVAR_MAX = -8.0, 4.0
SHAPES = [(IN, HID), (HID,), (HID, HID), (HID,), (HID, HID), (HID,), (HID, OUT), (OUT,)]


def param_count() -> int:
    return int(sum(int(np.prod(s)) for s in SHAPES))


def bf16(a) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    x = np.ascontiguousarray(np.asarray(a, np.float32))
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(flat: np.ndarray):
    out, o = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        out.append(np.asarray(flat[o:o + n], np.float64).reshape(s))
        o += n
    return out


def pack(parts) -> np.ndarray:
    return np.concatenate([np.asarray(p, np.float64).reshape(-1) for p in parts]).astype(np.float32)


def _rounder(rnd: bool):
    return (lambda a: bf16(np.asarray(a, np.float32))) if rnd else (lambda a: np.asarray(a, np.float64))


def forward(flat, X, rnd: bool = True):
    """Returns (out[n x 64] float64, cache) with the GPU's rounding points (rnd=False:
    exact float64 arithmetic, for finite-difference checks of the algebra)."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(flat)
    q = _rounder(rnd)
    h = q(X)
    hs = [h]
    for W, b in ((W1, b1), (W2, b2), (W3, b3)):
        pre = h @ q(W) + b
        h = q(np.maximum(pre, 0.0))
        hs.append(h)
    out = h @ q(W4) + b4
    return out, hs


def loss_and_dout(out, Y, M):
    """Mean masked Gaussian NLL and its gradient w.r.t. the 64 outputs."""
    n = out.shape[0]
    mean = out[:, :NDIM]
    raw = out[:, NDIM:2 * NDIM]
    lv = np.clip(raw, LOGVAR_MIN, LOGVAR_MAX)
    r = Y - mean
    iv = np.exp(-lv)
    loss = float(np.sum(M * 0.5 * (lv + r * r * iv)) / n)
    d = np.zeros_like(out)
    d[:, :NDIM] = -M * r * iv / n
    inside = (raw >= LOGVAR_MIN) & (raw <= LOGVAR_MAX)
    d[:, NDIM:2 * NDIM] = M * 0.5 * (1.0 - r * r * iv) / n * inside
    return loss, d


def backward(flat, hs, dout, rnd: bool = True):
    """Gradients of all parameters (flat, float64) for dL/dout."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(flat)
    q = _rounder(rnd)
    Ws = [W1, W2, W3, W4]
    grads = [None] * 8
    dpre = dout                                   # output layer has no activation
    for l in (3, 2, 1, 0):
        d16 = q(dpre)
        grads[2 * l] = hs[l].T @ d16
        grads[2 * l + 1] = np.sum(dpre, axis=0)
        if l > 0:
            dh = d16 @ q(Ws[l]).T
            dpre = dh * (hs[l] > 0)
    return np.concatenate([g.reshape(-1) for g in grads])


def loss_grad(flat, X, Y, M, rnd: bool = True):
    out, hs = forward(flat, X, rnd)
    loss, d = loss_and_dout(out, Y, M)
    return loss, backward(flat, hs, d, rnd)


def init_params(seed: int) -> np.ndarray:
    """He-normal weights, zero biases (the GPU initialiser draws its own values; this one
    serves the CPU tests)."""
    rng = np.random.default_rng(seed)
    parts = []
    for s in SHAPES:
        if len(s) == 2:
            parts.append(rng.normal(0.0, np.sqrt(2.0 / s[0]), s))
        else:
            parts.append(np.zeros(s))
    return pack(parts)


def adam_step(flat, grad, m, v, t, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update (float32 state), t counted from 1."""
    flat = np.asarray(flat, np.float32)
    g = np.asarray(grad, np.float32)
    m = (beta1 * m + (1 - beta1) * g).astype(np.float32)
    v = (beta2 * v + (1 - beta2) * g * g).astype(np.float32)
    mh = m / np.float32(1 - beta1 ** t)
    vh = v / np.float32(1 - beta2 ** t)
    return (flat - np.float32(lr) * mh / (np.sqrt(vh) + np.float32(eps))).astype(np.float32), m, v
