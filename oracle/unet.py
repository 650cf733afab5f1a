"""FP64 CPU oracle of the traveltime surrogate (test infrastructure only).

Restates, in float64 numpy, the network that libtomo_b200 trains and runs on the device
(seismic_tomography_3d_b200/csrc/api_net.cpp, net.cu): its input features, forward pass,
masked mean-squared tau loss and the gradient of that loss w.r.t. every parameter, with
the library's parameter layout (per convolution w[cout][27][cin] then b[cout]; then the
head wh[16], bh).  The reference has no learned component, so there is nothing of it to
pin against; this oracle is itself checked against torch-CPU autograd in float64
(tests/test_net_cpu.py).  Only tests use it.

Layout: volumes are [B][D][H][W][C] with D = y, H = x, W = z (the model's z-fastest order
read as channels-last).  Convolutions are 3x3x3, zero padded, tap = (dd*3 + dh)*3 + dw.
"""
from __future__ import annotations

import numpy as np

CONVS = [(16, 16), (16, 16), (16, 32), (32, 32), (32, 48), (48, 48), (48, 64), (64, 64),
         (112, 48), (48, 48), (80, 32), (32, 32), (48, 16), (16, 16)]


def layout():
    """[(w_off, b_off, cin, cout)] per convolution and the head offset, as the library."""
    out, off = [], 0
    for cin, cout in CONVS:
        w = off
        off += 27 * cin * cout
        out.append((w, off, cin, cout))
        off += cout
    return out, off, off + 17


def unpack(p):
    convs, head, n = layout()
    assert p.size == n
    W = [(p[w:w + 27 * ci * co].reshape(co, 27, ci).astype(np.float64), p[b:b + co].astype(np.float64))
         for w, b, ci, co in convs]
    return W, p[head:head + 16].astype(np.float64), float(p[head + 16])


def features(slow, window, nz, src, h, pad):
    """Input features of one sample (FP64): slow natural [y][x][z] model, window
    (x0, x1, y0, y1), source metres (model coordinates), pad = (pd, ph, pw)."""
    x0, x1, y0, y1 = window
    wnx, wny = x1 - x0, y1 - y0
    sx, sy, sz = src[0] - x0 * h, src[1] - y0 * h, src[2]
    pd, ph, pw = pad
    d = np.minimum(np.arange(pd), wny - 1)
    hh = np.minimum(np.arange(ph), wnx - 1)
    w = np.minimum(np.arange(pw), nz - 1)
    s = slow[y0 + d][:, x0 + hh][:, :, w].astype(np.float64)
    isz, isx, isy = min(int(sz / h), nz - 1), min(int(sx / h), wnx - 1), min(int(sy / h), wny - 1)
    s_src = float(slow[y0 + isy, x0 + isx, isz])
    Y, X, Z = np.meshgrid(d * h, hh * h, w * h, indexing="ij")
    dist = np.sqrt((X - sx) ** 2 + (Y - sy) ** 2 + (Z - sz) ** 2)
    f = np.zeros((pd, ph, pw, 16))
    f[..., 0] = s / s_src - 1.0
    f[..., 1] = dist / (64.0 * h)
    inside = (np.arange(pd)[:, None, None] < wny) & (np.arange(ph)[None, :, None] < wnx) & \
        (np.arange(pw)[None, None, :] < nz)
    return f, dist, s_src, inside


def target(T, dist, s_src, inside, h):
    """tau target: T / (s_src * dist) inside the window where dist >= h, else 0."""
    t = np.zeros(dist.shape)
    pd, ph, pw = dist.shape
    wny, wnx, nz = T.shape
    m = inside & (dist >= h)
    Tp = np.zeros(dist.shape)
    Tp[:wny, :wnx, :nz] = T
    t[m] = Tp[m] / (s_src * dist[m])
    return t


def conv(x, w, b):
    B, D, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    y = np.zeros((B, D, H, W, w.shape[0]))
    for tap in range(27):
        dd, dh, dw = tap // 9, (tap // 3) % 3, tap % 3
        y += np.einsum("bdhwc,oc->bdhwo", xp[:, dd:dd + D, dh:dh + H, dw:dw + W, :], w[:, tap, :], optimize=True)
    return y + b


def conv_bwd(x, w, dy):
    B, D, H, W, C = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for tap in range(27):
        dd, dh, dw_ = tap // 9, (tap // 3) % 3, tap % 3
        xs = xp[:, dd:dd + D, dh:dh + H, dw_:dw_ + W, :]
        dw[:, tap, :] = np.einsum("bdhwo,bdhwc->oc", dy, xs, optimize=True)
        dxp[:, dd:dd + D, dh:dh + H, dw_:dw_ + W, :] += np.einsum("bdhwo,oc->bdhwc", dy, w[:, tap, :], optimize=True)
    return dxp[:, 1:-1, 1:-1, 1:-1, :], dw, dy.sum(axis=(0, 1, 2, 3))


def pool(x):
    B, D, H, W, C = x.shape
    return x.reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4, 6))


def pool_bwd(dy):
    return np.repeat(np.repeat(np.repeat(dy, 2, 1), 2, 2), 2, 3) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 1), 2, 2), 2, 3)


def up_bwd(dy):
    B, D, H, W, C = dy.shape
    return dy.reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4, 6))


def forward_backward(p, x, tgt, want_grad=True):
    """Loss (masked mean squared tau error, mask tgt > 0) and the flat FP64 gradient."""
    W, wh, bh = unpack(p)
    relu = lambda a: np.maximum(a, 0.0)  # noqa: E731
    acts = {}

    def c(i, a):
        z = conv(a, *W[i])
        y = relu(z)
        acts[i] = (a, y)
        return y

    e1 = c(1, c(0, x))
    e2 = c(3, c(2, pool(e1)))
    e3 = c(5, c(4, pool(e2)))
    bb = c(7, c(6, pool(e3)))
    d3 = c(9, c(8, np.concatenate([up(bb), e3], -1)))
    d2 = c(11, c(10, np.concatenate([up(d3), e2], -1)))
    d1 = c(13, c(12, np.concatenate([up(d2), e1], -1)))
    tau = 1.0 + d1 @ wh + bh
    m = tgt > 0
    cnt = float(m.sum())
    loss = float(((tau - tgt)[m] ** 2).sum() / cnt)
    if not want_grad:
        return loss, tau, None
    g_tau = np.where(m, 2.0 * (tau - tgt) / cnt, 0.0)
    grads = [None] * 14
    g_wh = np.einsum("bdhw,bdhwc->c", g_tau, d1)
    g_bh = g_tau.sum()

    def cb(i, dy):
        a, y = acts[i]
        dz = dy * (y > 0)
        da, dw, db = conv_bwd(a, W[i][0], dz)
        grads[i] = (dw, db)
        return da

    g = cb(12, cb(13, g_tau[..., None] * wh))
    g_up, g_e1 = g[..., :32], g[..., 32:]
    g = cb(10, cb(11, up_bwd(g_up)))
    g_up, g_e2 = g[..., :48], g[..., 48:]
    g = cb(8, cb(9, up_bwd(g_up)))
    g_up, g_e3 = g[..., :64], g[..., 64:]
    g = cb(6, cb(7, up_bwd(g_up)))
    g = cb(4, cb(5, g_e3 + pool_bwd(g)))
    g = cb(2, cb(3, g_e2 + pool_bwd(g)))
    cb(0, cb(1, g_e1 + pool_bwd(g)))
    flat = []
    for dw, db in grads:
        flat += [dw.ravel(), db.ravel()]
    flat += [g_wh, np.array([g_bh])]
    return loss, tau, np.concatenate(flat)


def init_params(seed):
    """He-uniform weights, zero biases, small head (the library's initialisation scheme)."""
    rng = np.random.default_rng(seed)
    convs, head, n = layout()
    p = np.zeros(n, np.float32)
    for w, b, ci, co in convs:
        bound = np.sqrt(6.0 / (27 * ci))
        p[w:w + 27 * ci * co] = rng.uniform(-bound, bound, 27 * ci * co)
    p[head:head + 16] = rng.uniform(-0.05, 0.05, 16)
    return p
