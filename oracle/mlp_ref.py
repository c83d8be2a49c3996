"""TEST INFRASTRUCTURE: a numpy restatement of the learned warm start's
network (espice_b200/csrc/host/mlp_host.cu with kernels/mlp.cu), used only
by tests/ to check the tensor-core kernels' forward pass and gradients.

It rounds to BF16 exactly where the GPU does (GEMM operands: the
standardised inputs, the hidden activations, dZ and the weights) and
accumulates in float64, so the two differ by FP32 summation order only.
"""

from __future__ import annotations

import numpy as np


def bf16(a):
    """Round-to-nearest-even to bfloat16, returned as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def forward(layers, x, in_mu, in_sig):
    """layers: [(W n x k, b n)] padded as the GPU stores them; x [rows][n_in].
    Returns (bf16 layer inputs, pre-activations)."""
    k0 = layers[0][0].shape[1]
    xs = np.zeros((x.shape[0], k0), np.float32)
    xs[:, :x.shape[1]] = (x.astype(np.float32) - in_mu) / in_sig
    hs, zs = [bf16(xs)], []
    for i, (w, b) in enumerate(layers):
        z = (hs[-1].astype(np.float64) @ bf16(w).astype(np.float64).T + b).astype(np.float32)
        zs.append(z)
        if i + 1 < len(layers):
            hs.append(bf16(np.tanh(z)))
    return hs, zs


def gradients(layers, x, y, in_mu, in_sig, out_mu, out_sig):
    """The loss and [(dW, db)] of one pass, as esl_mlp_gradients defines them."""
    hs, zs = forward(layers, x, in_mu, in_sig)
    rows, n_out = y.shape
    t = (y.astype(np.float32) - out_mu) / out_sig
    out = zs[-1][:, :n_out]
    e = out - t
    loss = float(np.mean(e.astype(np.float64) ** 2))
    dz = np.zeros_like(zs[-1])
    dz[:, :n_out] = 2.0 * e / (rows * n_out)
    grads = [None] * len(layers)
    for i in range(len(layers) - 1, -1, -1):
        w, _ = layers[i]
        if i != len(layers) - 1:
            th = np.tanh(zs[i])
            dz = (dh * (1.0 - th * th)).astype(np.float32)
        dzb = bf16(dz).astype(np.float64)
        dw = (dzb.T @ hs[i].astype(np.float64)).astype(np.float32)
        db = dz.sum(axis=0).astype(np.float32)
        grads[i] = (dw, db)
        if i > 0:
            dh = (dzb @ bf16(w).astype(np.float64)).astype(np.float32)
    return loss, grads
