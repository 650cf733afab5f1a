"""CPU: the FP64 oracle of the traveltime surrogate against torch autograd (float64).

The oracle (oracle/unet.py) is the checker of the device network's gradients; here its
forward pass, loss and every parameter gradient are pinned to torch's conv3d / autograd
on the same parameters and inputs (agreement to 1e-9 relative)."""
import numpy as np
import pytest

from oracle import unet


def torch_reference(p, x, tgt):
    import torch
    import torch.nn.functional as F

    W, wh, bh = unet.unpack(p)
    params = []
    for w, b in W:
        # library layout w[co][tap][ci] -> torch [co][ci][kd][kh][kw]
        wt = torch.tensor(w.reshape(w.shape[0], 3, 3, 3, w.shape[2]).transpose(0, 4, 1, 2, 3).copy(),
                          dtype=torch.float64, requires_grad=True)
        bt = torch.tensor(b, dtype=torch.float64, requires_grad=True)
        params.append((wt, bt))
    wht = torch.tensor(wh, dtype=torch.float64, requires_grad=True)
    bht = torch.tensor([bh], dtype=torch.float64, requires_grad=True)
    xt = torch.tensor(x.transpose(0, 4, 1, 2, 3).copy(), dtype=torch.float64)

    def c(i, a):
        return F.relu(F.conv3d(a, params[i][0], params[i][1], padding=1))

    e1 = c(1, c(0, xt))
    e2 = c(3, c(2, F.avg_pool3d(e1, 2)))
    e3 = c(5, c(4, F.avg_pool3d(e2, 2)))
    bb = c(7, c(6, F.avg_pool3d(e3, 2)))
    up = lambda a: F.interpolate(a, scale_factor=2, mode="nearest")  # noqa: E731
    d3 = c(9, c(8, torch.cat([up(bb), e3], 1)))
    d2 = c(11, c(10, torch.cat([up(d3), e2], 1)))
    d1 = c(13, c(12, torch.cat([up(d2), e1], 1)))
    tau = 1.0 + torch.einsum("bcdhw,c->bdhw", d1, wht) + bht
    t = torch.tensor(tgt, dtype=torch.float64)
    m = t > 0
    loss = ((tau - t)[m] ** 2).sum() / m.sum()
    loss.backward()
    flat = []
    for wt, bt in params:
        g = wt.grad.numpy().transpose(0, 2, 3, 4, 1).reshape(wt.shape[0], 27, wt.shape[1])
        flat += [g.ravel(), bt.grad.numpy()]
    flat += [wht.grad.numpy(), bht.grad.numpy()]
    return float(loss), tau.detach().numpy(), np.concatenate(flat)


def test_layout_size():
    convs, head, n = unet.layout()
    assert len(convs) == 14 and n == head + 17


@pytest.mark.parametrize("shape", [(1, 8, 8, 8), (2, 8, 16, 8)])
def test_oracle_matches_torch_autograd(shape):
    pytest.importorskip("torch")
    rng = np.random.default_rng(sum(shape))
    B, D, H, W = shape
    p = unet.init_params(3)
    # biases non-zero so their gradients are exercised too
    convs, head, _ = unet.layout()
    for w, b, ci, co in convs:
        p[b:b + co] = rng.uniform(-0.05, 0.05, co)
    p[head + 16] = 0.02
    x = np.zeros((B, D, H, W, 16))
    x[..., :2] = rng.normal(0, 1, (B, D, H, W, 2))
    tgt = np.where(rng.random((B, D, H, W)) < 0.8, rng.uniform(0.8, 1.2, (B, D, H, W)), 0.0)
    loss, tau, g = unet.forward_backward(p, x, tgt)
    loss_t, tau_t, g_t = torch_reference(p, x, tgt)
    assert abs(loss - loss_t) <= 1e-9 * abs(loss_t)
    np.testing.assert_allclose(tau, tau_t, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(g, g_t, rtol=1e-8, atol=1e-12 * np.abs(g_t).max())


def test_features_and_target_geometry():
    """tau of a constant-velocity field is 1 wherever it is defined."""
    h, nz, nx, ny = 10.0, 12, 14, 10
    slow = np.full((ny, nx, nz), 1 / 2000.0, np.float32)
    src = (33.0, 41.0, 7.0)
    Y, X, Z = np.meshgrid(np.arange(ny) * h, np.arange(nx) * h, np.arange(nz) * h, indexing="ij")
    T = np.sqrt((X - src[0]) ** 2 + (Y - src[1]) ** 2 + (Z - src[2]) ** 2) / 2000.0
    f, dist, s_src, inside = unet.features(slow, (0, nx, 0, ny), nz, src, h, (16, 16, 16))
    t = unet.target(T, dist, s_src, inside, h)
    m = t > 0
    assert m.sum() > 0.8 * nx * ny * nz
    np.testing.assert_allclose(t[m], 1.0, rtol=1e-6)  # slowness is float32
    assert np.all(f[..., 0] == 0.0)
