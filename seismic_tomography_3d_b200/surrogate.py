"""Learned warm start: training data, training loop and the warm-started solve, all on the
device through the C ABI (tomo_random_tiles, tomo_eik_solve, tomo_net_*,
tomo_eik_solve_seeded).  torch only holds device buffers.

Training data are fields of this solver on seeded random models: a context whose model is
a mosaic of tile x tile x nz random layered tiles (3-6 dipping layers, 1500-4500 m/s, 0-12
Gaussian anomalies of up to +-15 %), one surface source per tile and each tile solved as
the shot's window -- a windowed solve equals the solve on the tile alone, so one batched
launch yields a whole chunk of independent training fields.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np

from . import Context, Net


def conv_flops_per_voxel():
    """Forward FLOPs of the network per full-resolution voxel (2 x 27 x Cin x Cout per
    convolution, deeper levels at 1/8 of the voxels per level)."""
    levels = {0: [(16, 16), (16, 16), (48, 16), (16, 16)], 1: [(16, 32), (32, 32), (80, 32), (32, 32)],
              2: [(32, 48), (48, 48), (112, 48), (48, 48)], 3: [(48, 64), (64, 64)]}
    return sum(54.0 * ci * co / 8 ** lv for lv, convs in levels.items() for ci, co in convs)


@dataclasses.dataclass
class Dataset:
    samples: list          # tomo_net_sample dicts
    keep: list             # device tensors the samples point into
    tile: int
    nz: int
    h: float
    gen_s: float
    solve_ms: float


def make_dataset(nfields=20000, tile=64, nz=64, h=12.5, tiles_per_side=16, seed=0, device=0):
    """nfields solver-generated (slowness, traveltime) fields on tile^2 x nz windows."""
    import torch

    per = tiles_per_side * tiles_per_side
    ctx = Context(tiles_per_side * tile, tiles_per_side * tile, nz, h, device=device)
    rng = np.random.default_rng(seed)
    samples, keep = [], []
    t0 = time.perf_counter()
    solve_ms = 0.0
    vol = tile * tile * nz
    chunk = 0
    while len(samples) < nfields:
        ctx.random_tiles(tile, seed * 1_000_003 + chunk)
        wins, shots = [], []
        for j in range(tiles_per_side):
            for i in range(tiles_per_side):
                wins.append((i * tile, (i + 1) * tile, j * tile, (j + 1) * tile))
                shots.append(((i * tile + rng.integers(0, tile)) * h, (j * tile + rng.integers(0, tile)) * h,
                              float(rng.integers(0, max(nz // 8, 1))) * h))
        wins, shots = np.array(wins, np.int32), np.array(shots, np.float32)
        _, st = ctx.eik_solve(shots, windows=wins)
        solve_ms += st["total_ms"]
        T = torch.empty(per * vol, dtype=torch.float32, device=f"cuda:{device}")
        ctx.eik_volumes_to(T.data_ptr())
        slow = device_view(ctx.slowness_device(), ctx.grid.nx * ctx.grid.ny * nz).clone()
        keep += [T, slow]
        for k in range(per):
            if len(samples) >= nfields:
                break
            samples.append(dict(slow=slow.data_ptr(), model_nx=ctx.grid.nx, model_ny=ctx.grid.ny, nz=nz,
                                window=tuple(int(v) for v in wins[k]), source=tuple(float(v) for v in shots[k]),
                                T=T.data_ptr() + 4 * k * vol))
        chunk += 1
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    ctx.close()
    return Dataset(samples, keep, tile, nz, h, gen_s, solve_ms)


class _DeviceArray:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (int(ptr), False), "version": 3}


def device_view(ptr, n):
    """torch view (no copy) of n float32 at a raw device address owned by the library."""
    import torch

    return torch.as_tensor(_DeviceArray(ptr, n), device="cuda")


def train(net: Net, ds: Dataset, epochs=3, batch=8, lr=1e-3, val_frac=0.02, seed=0, log=None):
    """Adam over shuffled batches; lr halves every epoch.  Returns a summary dict."""
    import torch

    n = len(ds.samples)
    nval = max(batch, int(n * val_frac))
    idx = np.random.default_rng(seed).permutation(n)
    val, tr = [ds.samples[i] for i in idx[:nval]], idx[nval:]
    val_loss = lambda: float(np.mean([net.evaluate(val[k:k + batch], ds.h)  # noqa: E731
                                      for k in range(0, len(val), batch)]))
    v0 = val_loss()
    steps, t_train = 0, 0.0
    hist = []
    rng = np.random.default_rng(seed + 1)
    for ep in range(epochs):
        order = rng.permutation(tr)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        losses = []
        for k in range(0, len(order) - batch + 1, batch):
            losses.append(net.train_step([ds.samples[i] for i in order[k:k + batch]], ds.h, lr))
            steps += 1
        torch.cuda.synchronize()
        t_train += time.perf_counter() - t0
        hist.append({"epoch": ep, "train_loss": float(np.mean(losses[-50:])), "val_loss": val_loss(), "lr": lr})
        if log:
            log(hist[-1])
        lr *= 0.5
    vox = ds.tile * ds.tile * ds.nz
    flops = 3.0 * conv_flops_per_voxel() * vox * steps * batch
    return {"steps": steps, "batch": batch, "epochs": epochs, "train_s": t_train,
            "samples_per_s": steps * batch / t_train, "tflops": flops / t_train / 1e12,
            "val_loss_initial": v0, "val_loss": hist[-1]["val_loss"], "val_tau_rms": float(np.sqrt(hist[-1]["val_loss"])),
            "history": hist}


def predict_ceiling(net: Net, ctx: Context, shots, windows, stride=1):
    """Predicted traveltimes of every shot's window (back to back, z fastest) on the device,
    from the context's current model; stride > 1: the network on every stride-th node, tau
    interpolated back.  Returns (tensor, device ms)."""
    import torch

    g = ctx.grid
    n = len(shots)
    if windows is None:
        windows = np.tile(np.array([0, g.nx, 0, g.ny], np.int32), (n, 1))
    sizes = ctx.volume_sizes(n, windows)
    out = torch.zeros(sum(sizes), dtype=torch.float32, device="cuda")
    sp = ctx.slowness_device()
    samples = [dict(slow=sp, model_nx=g.nx, model_ny=g.ny, nz=g.nz, window=tuple(int(v) for v in windows[k]),
                    source=tuple(float(v) for v in shots[k]), T=0) for k in range(n)]
    ms = net.predict(samples, g.dx, out.data_ptr(), stride=stride)
    return out, ms
