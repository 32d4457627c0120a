"""CPU oracle of the learned gas-optics network: forward pass, loss and
backward pass in numpy FP64, optionally rounding to BF16 at the points where
the GPU kernels store BF16 (inputs, weights, activations, output gradients).

TEST INFRASTRUCTURE ONLY: used by tests/ to check the GPU kernels of
ccpp_physics_b200/csrc/lw_mlp.cu; never called by the library.

Network: x[8] (7 normalised features + 1) -> z1 = W1 x -> h1 = silu(z1)
-> z2 = W2 h1 + b2 -> h2 = silu(z2) -> y = W3 h2 + b3 (288, padded rows zero).
Loss: mean over the 280 real outputs and the batch of (y - t)^2.
"""
from __future__ import annotations

import numpy as np

HID, NOP = 128, 288
PAD = np.r_[140:144, 284:288]
P_W1, P_W2 = 0, 128 * 8
P_B2 = P_W2 + 128 * 128
P_W3 = P_B2 + 128
P_B3 = P_W3 + 288 * 128
P_N = P_B3 + 288


def bf16(a):
    """Round float values to bfloat16 (nearest even) and back."""
    x = np.ascontiguousarray(a, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def unpack(w):
    """Natural-shape parameters from the 53,656-float export (W3/b3 280 rows)."""
    w = np.asarray(w, dtype=np.float64)
    k = 0
    W1 = w[k:k + 1024].reshape(128, 8); k += 1024
    W2 = w[k:k + 16384].reshape(128, 128); k += 16384
    b2 = w[k:k + 128]; k += 128
    W3r = w[k:k + 280 * 128].reshape(280, 128); k += 280 * 128
    b3r = w[k:k + 280]
    W3 = np.zeros((NOP, HID)); b3 = np.zeros(NOP)
    keep = np.setdiff1d(np.arange(NOP), PAD)
    W3[keep] = W3r
    b3[keep] = b3r
    return W1, W2, b2, W3, b3


def normalise(feats, norm):
    x = (np.asarray(feats, np.float64)[:, :7] - norm[0:7]) / norm[8:15]
    return np.concatenate([x, np.ones((x.shape[0], 1))], axis=1)


def forward(x, params, emulate_bf16=True):
    W1, W2, b2, W3, b3 = params
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    xq = r(x)
    z1 = xq @ r(W1).T
    h1 = r(silu(z1))
    z2 = h1 @ r(W2).T + b2
    h2 = r(silu(z2))
    y = h2 @ r(W3).T + b3
    return dict(x=xq, z1=z1, h1=h1, z2=z2, h2=h2, y=y)


def loss_and_grads(x, t, params, emulate_bf16=True):
    """MSE and gradients (W1, W2, b2, W3, b3) of one batch."""
    W1, W2, b2, W3, b3 = params
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    f = forward(x, params, emulate_bf16)
    B = x.shape[0]
    mask = np.ones(NOP)
    mask[PAD] = 0
    e = (f["y"] - t) * mask
    loss = float(np.sum(e * e) / (B * 280))
    dy = r(e * (2.0 / (B * 280)))
    gW3 = dy.T @ f["h2"]
    gb3 = dy.sum(0)
    dz2 = r((dy @ r(W3)) * dsilu(r(f["z2"])))
    gW2 = dz2.T @ f["h1"]
    gb2 = dz2.sum(0)
    dz1 = r((dz2 @ r(W2)) * dsilu(r(f["z1"])))
    gW1 = dz1.T @ f["x"]
    return loss, (gW1, gW2, gb2, gW3 * mask[:, None], gb3 * mask)


def pack_grads(g):
    """Padded parameter order of rrtmg_lw_gpu_surrogate_grads."""
    gW1, gW2, gb2, gW3, gb3 = g
    return np.concatenate([gW1.ravel(), gW2.ravel(), gb2, gW3.ravel(), gb3])
