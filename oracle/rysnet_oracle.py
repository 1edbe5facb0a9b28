"""Test oracle for the learned Rys-root network (cintx_b200/csrc/rysnet.cu): a float64 numpy
restatement of RysNet's forward pass, loss and gradient, used by the tests to check the device
training kernel (rysnet_train_kernel) and nothing else.  Parameter layout, feature scaling and
loss follow include/cintx_cuda.h (CINTX_RYSNET_NPARAM): W1[64][2], b1[64], W2[64][64], b2[64],
W3[18][64], b3[18]; loss = mean over samples of sum of squared errors of the 2*nroots used
outputs / (2*nroots).  This file is test infrastructure: product code never imports it.
"""
from __future__ import annotations

import numpy as np

H, OUT, HALF, NIN = 64, 18, 9, 2
SIZES = [("W1", (H, NIN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (OUT, H)), ("b3", (OUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    out, o = {}, 0
    for name, shp in SIZES:
        k = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + k], dtype=np.float64).reshape(shp)
        o += k
    return out


def features(n, x):
    """Network inputs for order n at x (rysnet_features)."""
    n = np.asarray(n, dtype=np.float64)
    x = np.maximum(np.asarray(x, dtype=np.float64), 1e-7)
    return np.stack([(n - 5) * 0.25, (np.log(x) + 5.75) / 10.35], axis=-1)


def _silu(a):
    s = 1.0 / (1.0 + np.exp(-a))
    return a * s, s * (1.0 + a * (1.0 - s))


def forward(p, feat):
    q = unpack(p)
    a1 = feat @ q["W1"].T + q["b1"]
    h1, _ = _silu(a1)
    a2 = h1 @ q["W2"].T + q["b2"]
    h2, _ = _silu(a2)
    return h2 @ q["W3"].T + q["b3"]


def loss_grad(p, feat, tgt, nroots):
    """Loss and gradient (float64) of the training objective for one batch."""
    q = unpack(p)
    feat = np.asarray(feat, dtype=np.float64)
    tgt = np.asarray(tgt, dtype=np.float64)
    n = np.asarray(nroots, dtype=np.float64)
    B = feat.shape[0]
    a1 = feat @ q["W1"].T + q["b1"]
    h1, s1 = _silu(a1)
    a2 = h1 @ q["W2"].T + q["b2"]
    h2, s2 = _silu(a2)
    y = h2 @ q["W3"].T + q["b3"]
    mask = (np.arange(OUT)[None, :] % HALF) < n[:, None]
    d = np.where(mask, y - tgt, 0.0)
    loss = float(np.sum(np.sum(d * d, axis=1) / (2 * n)) / B)
    dy = d / (n[:, None] * B)
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dz2 = (dy @ q["W3"]) * s2
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ q["W2"]) * s1
    g["W1"] = dz1.T @ feat
    g["b1"] = dz1.sum(0)
    return loss, np.concatenate([g[name].ravel() for name, _ in SIZES])
