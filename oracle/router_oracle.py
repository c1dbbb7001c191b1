"""FP64 NumPy statement of the router MLP's loss and gradients.

TEST INFRASTRUCTURE ONLY: the checker for the library's router training
kernels (forward, backward, top-8 cross-entropy).  The network:
  z0 = (x - centre) * scale,  z_{l+1} = ReLU(W_l z_l + b_l) (no ReLU on the
  last layer), loss = mean_rows -sum_t w_t log softmax(z_L)_{idx_t}.
Weights enter the forward and backward passes rounded to bf16, as in the
library (BF16 weights, fp32 accumulation); gradients are taken with respect
to those rounded weights and applied to the fp32 masters.
"""
from __future__ import annotations

import numpy as np


def bf16(a):
    a = np.ascontiguousarray(a, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def loss_grad(layers, x, centre, scale, tidx, tw):
    """layers: [(W, b)] (W: out x in).  Returns (loss, [(dW, db)])."""
    acts = [((x.astype(np.float64) - centre) * scale)]
    Wq = [bf16(W).astype(np.float64) for W, _ in layers]
    for l, (W, b) in enumerate(layers):
        h = acts[-1] @ Wq[l].T + b.astype(np.float64)
        if l + 1 < len(layers):
            h = np.maximum(h, 0.0)
        acts.append(h)
    z = acts[-1]
    B, K = z.shape
    mx = z.max(1, keepdims=True)
    lse = mx + np.log(np.exp(z - mx).sum(1, keepdims=True))
    sm = np.exp(z - lse)
    t = np.zeros_like(z)
    for u in range(tidx.shape[1]):
        np.add.at(t, (np.arange(B), tidx[:, u]), tw[:, u])
    loss = float(-(t * (z - lse)).sum() / B)
    g = (sm - t) / B
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        dW = g.T @ acts[l]
        db = g.sum(0)
        grads[l] = (dW, db)
        if l > 0:
            g = (g @ Wq[l]) * (acts[l] > 0)
    return loss, grads
