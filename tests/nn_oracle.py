"""FP32 numpy restatement of the learned-guess U-Net (artss_b200.learned.UNet):
forward, loss and backward, used as the CPU oracle of the network's
gradients.  Test infrastructure only."""
from __future__ import annotations

import numpy as np

from artss_b200 import learned as LN


def conv(x, w, b, relu):
    """x [D][H][W][ci]; w [27][co][ci]; -> [D][H][W][co]"""
    wt = np.ascontiguousarray(w.reshape(3, 3, 3, w.shape[1], w.shape[2]).transpose(3, 4, 0, 1, 2))
    y = LN.conv3d_ref(x, wt, b, relu)
    return y


def conv_bwd(x, w, y, dy, relu):
    if relu:
        dy = dy * (y > 0)
    db = dy.sum(axis=(0, 1, 2))
    dw = LN.conv3d_wgrad_ref(x, dy)
    wt = np.ascontiguousarray(w.reshape(3, 3, 3, w.shape[1], w.shape[2]).transpose(3, 4, 0, 1, 2))
    dx = LN.conv3d_ref(dy, LN.flip_weights(wt))
    return dx, dw, db


def pool(x):
    D, H, W, C = x.shape
    return x.reshape(D // 2, 2, H // 2, 2, W // 2, 2, C).mean(axis=(1, 3, 5))


def pool_bwd(dy):
    return np.repeat(np.repeat(np.repeat(dy, 2, 0), 2, 1), 2, 2) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 0), 2, 1), 2, 2)


def up_bwd(dy):
    D, H, W, C = dy.shape
    return dy.reshape(D // 2, 2, H // 2, 2, W // 2, 2, C).sum(axis=(1, 3, 5))


ORDER = ["e0a", "e0b", "e1a", "e1b", "b2a", "b2b", "d1a", "d1b", "d0a", "d0b"]
RELU = {k: k != "d0b" for k in ORDER}


def forward(P, x):
    a = {}
    a["x"] = x
    a["a0"] = conv(x, *P["e0a"], RELU["e0a"])
    a["s0"] = conv(a["a0"], *P["e0b"], True)
    a["p0"] = pool(a["s0"])
    a["a1"] = conv(a["p0"], *P["e1a"], True)
    a["s1"] = conv(a["a1"], *P["e1b"], True)
    a["p1"] = pool(a["s1"])
    a["a2"] = conv(a["p1"], *P["b2a"], True)
    a["b2"] = conv(a["a2"], *P["b2b"], True)
    a["cat1"] = np.concatenate([up(a["b2"]), a["s1"]], axis=3)
    a["e1"] = conv(a["cat1"], *P["d1a"], True)
    a["d1"] = conv(a["e1"], *P["d1b"], True)
    a["cat0"] = np.concatenate([up(a["d1"]), a["s0"]], axis=3)
    a["e0"] = conv(a["cat0"], *P["d0a"], True)
    a["out"] = conv(a["e0"], *P["d0b"], False)
    return a


def loss_and_grads(P, x, target, mask):
    a = forward(P, x)
    n = max(int(mask.sum()), 1)
    d = (a["out"][..., 0] - target) * mask
    loss = 0.5 * float((d * d).sum()) / n
    g = {}
    dout = np.zeros_like(a["out"])
    dout[..., 0] = d / n
    de0, *g["d0b"] = conv_bwd(a["e0"], P["d0b"][0], a["out"], dout, False)
    dcat0, *g["d0a"] = conv_bwd(a["cat0"], P["d0a"][0], a["e0"], de0, True)
    dd1 = up_bwd(dcat0[..., :32])
    ds0 = dcat0[..., 32:].copy()
    de1, *g["d1b"] = conv_bwd(a["e1"], P["d1b"][0], a["d1"], dd1, True)
    dcat1, *g["d1a"] = conv_bwd(a["cat1"], P["d1a"][0], a["e1"], de1, True)
    db2 = up_bwd(dcat1[..., :64])
    ds1 = dcat1[..., 64:].copy()
    da2, *g["b2b"] = conv_bwd(a["a2"], P["b2b"][0], a["b2"], db2, True)
    dp1, *g["b2a"] = conv_bwd(a["p1"], P["b2a"][0], a["a2"], da2, True)
    ds1 = ds1 + pool_bwd(dp1)
    da1, *g["e1b"] = conv_bwd(a["a1"], P["e1b"][0], a["s1"], ds1, True)
    dp0, *g["e1a"] = conv_bwd(a["p0"], P["e1a"][0], a["a1"], da1, True)
    ds0 = ds0 + pool_bwd(dp0)
    da0, *g["e0b"] = conv_bwd(a["a0"], P["e0b"][0], a["s0"], ds0, True)
    _, *g["e0a"] = conv_bwd(a["x"], P["e0a"][0], a["a0"], da0, True)
    return loss, g, a
