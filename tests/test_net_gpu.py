"""The traveltime surrogate on the device, through the C ABI.

  * forward output and the gradients of every parameter (BF16 tensor-core convolutions,
    FP32 accumulation) against the FP64 oracle (oracle/unet.py, itself pinned to torch
    autograd), on a small odd-sized window and on the 64^3 training tile: loss within 1 %;
    the whole gradient within 3e-2 relative L2 error, the median parameter tensor within
    2e-2 and every tensor within 1e-1 (BF16 activations round to ~4e-3 relative through 14
    layers and back; the deepest level of the small window has 3 x 3 x 2 voxels, where a
    ReLU mask flipped by rounding moves a bias gradient by several per cent);
  * training on solver-generated fields lowers the loss;
  * the trained network's prediction, used as the ceiling of tomo_eik_solve_seeded, leaves
    the solution unchanged (the plain solve checks it) -- and the test reports what it saves.
"""
import numpy as np
import pytest

from oracle import unet
from seismic_tomography_3d_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def _case(tomo, seed=4, nx=20, ny=24, nz=14, h=20.0):
    """A layered model, one source, its plain-FIM traveltimes."""
    sv = wl.small(seed, nx, ny, nz, h=h, nshots=1)
    with tomo.Context(nx, ny, nz, h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots)
        T = ctx.eik_volume(0)
    slow = (1.0 / sv.velocity).astype(np.float32)
    return sv, slow, T


def _rel_l2(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / (np.linalg.norm(b) + 1e-300))


GRAD_REL = 3e-2         # the whole gradient (all parameters), relative L2
GRAD_REL_MEDIAN = 2e-2  # the median parameter tensor
GRAD_REL_TENSOR = 1e-1  # every parameter tensor
LOSS_REL = 1e-2


@pytest.mark.parametrize("shape", [(20, 24, 14, 20.0), (64, 64, 64, 12.5)], ids=["20x24x14", "64^3"])
def test_gradients_match_oracle(tomo, shape):
    nx, ny, nz, h = shape
    sv, slow, T = _case(tomo, nx=nx, ny=ny, nz=nz, h=h)
    net = tomo.Net(seed=11)
    p = unet.init_params(11)
    convs, head, _ = unet.layout()
    rng = np.random.default_rng(0)
    for w, b, ci, co in convs:
        p[b:b + co] = rng.uniform(-0.05, 0.05, co)
    net.set_params(p)
    p = net.get_params()
    slow_d, T_d = _dev(slow), _dev(T)
    win = (0, sv.nx, 0, sv.ny)
    sample = dict(slow=slow_d.data_ptr(), model_nx=sv.nx, model_ny=sv.ny, nz=sv.nz, window=win,
                  source=sv.shots[0], T=T_d.data_ptr())
    loss, g = net.gradients([sample], h)
    pad = tuple(-(-n // 8) * 8 for n in (sv.ny, sv.nx, sv.nz))
    f, dist, s_src, inside = unet.features(slow, win, sv.nz, sv.shots[0], h, pad)
    tgt = unet.target(T, dist, s_src, inside, h)
    loss_o, tau_o, g_o = unet.forward_backward(p, f[None], tgt[None])
    errs = {}
    for i, (w, b, ci, co) in enumerate(convs):
        gw, gw_o = g[w:w + 27 * ci * co], g_o[w:w + 27 * ci * co]
        if i == 0:  # input channels 2..15 are zero: only the first two carry gradient
            gw, gw_o = gw.reshape(co, 27, ci)[..., :2].ravel(), gw_o.reshape(co, 27, ci)[..., :2].ravel()
        errs[f"w{i}"] = _rel_l2(gw, gw_o)
        errs[f"b{i}"] = _rel_l2(g[b:b + co], g_o[b:b + co])
    errs["head"] = _rel_l2(g[head:head + 17], g_o[head:head + 17])
    worst = max(errs, key=errs.get)
    med = float(np.median(list(errs.values())))
    whole = _rel_l2(g, g_o)
    print(f"\n{shape}: loss {loss:.6f} vs oracle {loss_o:.6f} ({abs(loss - loss_o) / loss_o:.2e}); gradient rel L2 "
          f"{whole:.3e}; per tensor worst {errs[worst]:.3e} ({worst}), median {med:.3e}")
    assert abs(loss - loss_o) <= LOSS_REL * loss_o, (loss, loss_o)
    assert whole <= GRAD_REL
    assert med <= GRAD_REL_MEDIAN, errs
    assert errs[worst] <= GRAD_REL_TENSOR, errs
    # prediction = oracle tau * s_src * distance on the window
    import torch

    out = torch.zeros(sv.nx * sv.ny * sv.nz, dtype=torch.float32, device="cuda")
    net.predict([sample], h, out.data_ptr())
    t_pred = out.cpu().numpy().reshape(sv.ny, sv.nx, sv.nz)
    t_o = (tau_o[0] * s_src * dist)[:sv.ny, :sv.nx, :sv.nz]
    m = dist[:sv.ny, :sv.nx, :sv.nz] >= h
    assert np.max(np.abs(t_pred[m] - t_o[m]) / t_o[m]) < 0.02
    assert np.all(t_pred[~m] == 0.0)
    net.close()


def test_strided_prediction_equals_prediction_on_the_subsampled_model(tomo):
    """tomo_net_predict_strided with stride 2 on a model feeds the network exactly the
    features the plain prediction gets on that model subsampled by 2 at spacing 2h (same
    slowness samples, same distances, distance channel / (64 h stride)), so at the sampled
    nodes both predictions agree; between them the strided one interpolates tau."""
    import torch

    nx, ny, nz, h, k = 33, 29, 17, 20.0, 2
    sv = wl.small(6, nx, ny, nz, h=h, nshots=1)
    slow = (1.0 / sv.velocity).astype(np.float32)
    src = (8 * h, 12 * h, 2 * h)  # on a node of both grids
    net = tomo.Net(seed=3)
    fine_d = _dev(slow)
    coarse = np.ascontiguousarray(slow[::k, ::k, ::k])
    coarse_d = _dev(coarse)
    cy, cx, cz = coarse.shape
    out_f = torch.zeros(nx * ny * nz, dtype=torch.float32, device="cuda")
    out_c = torch.zeros(cx * cy * cz, dtype=torch.float32, device="cuda")
    net.predict([dict(slow=fine_d.data_ptr(), model_nx=nx, model_ny=ny, nz=nz, window=(0, nx, 0, ny), source=src,
                      T=0)], h, out_f.data_ptr(), stride=k)
    net.predict([dict(slow=coarse_d.data_ptr(), model_nx=cx, model_ny=cy, nz=cz, window=(0, cx, 0, cy), source=src,
                      T=0)], k * h, out_c.data_ptr())
    tf = out_f.cpu().numpy().reshape(ny, nx, nz)
    tc = out_c.cpu().numpy().reshape(cy, cx, cz)
    np.testing.assert_allclose(tf[::k, ::k, ::k], tc, rtol=1e-6, atol=0)
    assert np.all(np.isfinite(tf)) and (tf > 0).mean() > 0.99
    net.close()


def _tiles(tomo, ctx, tile, nz, h, seed):
    """Random tiles as the model, one surface source per tile; returns net samples."""
    import torch

    ctx.random_tiles(tile, seed)
    rng = np.random.default_rng(seed)
    tx, ty = ctx.grid.nx // tile, ctx.grid.ny // tile
    wins, shots = [], []
    for j in range(ty):
        for i in range(tx):
            wins.append((i * tile, (i + 1) * tile, j * tile, (j + 1) * tile))
            shots.append(((i * tile + rng.integers(0, tile)) * h, (j * tile + rng.integers(0, tile)) * h, 0.0))
    wins, shots = np.array(wins, np.int32), np.array(shots, np.float32)
    ctx.eik_solve(shots, windows=wins)
    T = torch.empty(len(shots) * tile * tile * nz, dtype=torch.float32, device="cuda")
    ctx.eik_volumes_to(T.data_ptr())
    # the model is rewritten by the next random_tiles call: keep a copy
    slow = torch.from_numpy(ctx.get_slowness().ravel()).cuda()
    vol = tile * tile * nz
    samples = [dict(slow=slow.data_ptr(), model_nx=ctx.grid.nx, model_ny=ctx.grid.ny, nz=nz, window=tuple(wins[k]),
                    source=shots[k], T=T.data_ptr() + 4 * k * vol) for k in range(len(shots))]
    return samples, (slow, T), wins, shots


def test_training_lowers_loss_and_warm_start_keeps_the_solution(tomo):
    import torch

    tile, nz, h = 32, 32, 20.0
    ctx = tomo.Context(4 * tile, 4 * tile, nz, h)
    train, keep, _, _ = _tiles(tomo, ctx, tile, nz, h, seed=1)
    net = tomo.Net(seed=5)
    first = net.evaluate(train, h)
    for it in range(60):
        k = (4 * it) % len(train)
        net.train_step(train[k:k + 4], h, 2e-3)
    last = net.evaluate(train, h)
    assert last < 0.5 * first, (first, last)

    # warm start on a fresh set of tiles: prediction -> ceiling -> seeded solve
    test, keep2, wins, shots = _tiles(tomo, ctx, tile, nz, h, seed=99)
    _, st_plain = ctx.eik_solve(shots, windows=wins)
    plain = [ctx.eik_volume(i) for i in range(len(shots))]
    pred = torch.zeros(len(shots) * tile * tile * nz, dtype=torch.float32, device="cuda")
    net.predict(test, h, pred.data_ptr())
    torch.cuda.synchronize()
    _, st, ss = ctx.eik_solve_seeded(shots, pred.data_ptr(), 0.02, windows=wins)
    vmax = 4500.0 * 1.15
    for i in range(len(shots)):
        T = ctx.eik_volume(i)
        m = plain[i] >= 2 * h / vmax
        assert np.max(np.abs(T[m] - plain[i][m]) / plain[i][m]) < 1e-5
    print(f"\nwarm start with the trained surrogate: activations {st['activations']} vs plain "
          f"{st_plain['activations']}, fallback shots {ss['shots_fallback']}/{len(shots)}")
    net.close()
    ctx.close()
