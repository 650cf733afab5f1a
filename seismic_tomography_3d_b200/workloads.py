"""Seeded synthetic workloads (numpy ``default_rng(seed)``).

The reference ships no data (its .gitignore drops every .bin/.txt), so the benchmark and
test inputs are generated here with the shapes, spacings and value ranges of the five
tomography configurations:

1. single shot, 101x101x51 nodes at 25 m, v(z) = 1500 + 0.6 z plus two +-10 % Gaussian
   anomalies (sigma 150 m), a surface source and 200 surface receivers;
2. 64 shots on a jittered 8x8 surface grid over a 201x201x101 model at 12.5 m (three layers
   1500/2500/3500 m/s with dipping interfaces plus eight +-10 % anomalies), each shot on a
   brick-aligned window covering 60-100 % of the lateral extent;
3. one tomography iteration on the config-2 model: start model v(z) = 1500 + z, 64 shots x
   2500 receivers (50x50 surface grid, 25..2475 m), picks = traveltimes + N(0, 2 ms),
   inversion cells 51 x 51 x 52 m (50x50x25), lambda 0.1, order 2, 30 CGLS iterations;
5. 401x401x201 nodes at 10 m, 256 shots (16x16) x 10,000 receivers (100x100).

Velocities are float32 arrays of shape (ny, nx, nz) (the reference's z-fastest layout).
Shots and receivers sit on grid nodes (surface z = 0).
"""
from __future__ import annotations

import dataclasses

import numpy as np

BRICK = 4

# Solver tolerances of the timed runs.  The metric is quoted at 1e-4 relative traveltime
# error, so the face-change and in-brick tolerances are loosened until the error against
# the FP64 fixed point sits well inside that budget (tests/test_fullsize_gpu.py checks the
# whole config-2 batch at these settings).  The library default is the exact fixed point.
TIMED_TOLERANCES = dict(change_tol=1e-5, inner_tol=1e-6)
# Full-grid solves on the smooth starting models of configs 3 and 5 add the time-band
# ordering (0.2 s): it removes most re-activation cascades of those models.
TIMED_TOLERANCES_BANDED = dict(TIMED_TOLERANCES, time_band=0.2)


@dataclasses.dataclass
class Survey:
    name: str
    nx: int
    ny: int
    nz: int
    h: float
    velocity: np.ndarray            # (ny, nx, nz) float32
    shots: np.ndarray               # (ns, 3) float32 metres
    windows: np.ndarray | None      # (ns, 4) int32 [x0, x1, y0, y1] or None
    receivers: np.ndarray | None    # (nr, 3) float32

    @property
    def nodes(self):
        return self.nx * self.ny * self.nz


def _coords(nx, ny, nz, h):
    y = np.arange(ny, dtype=np.float64)[:, None, None] * h
    x = np.arange(nx, dtype=np.float64)[None, :, None] * h
    z = np.arange(nz, dtype=np.float64)[None, None, :] * h
    return x, y, z


def _anomalies(rng, nx, ny, nz, h, count, amp=0.10, sigma=150.0):
    x, y, z = _coords(nx, ny, nz, h)
    f = np.ones((ny, nx, nz), np.float64)
    lx, ly, lz = (nx - 1) * h, (ny - 1) * h, (nz - 1) * h
    for i in range(count):
        cx, cy = rng.uniform(0.15, 0.85) * lx, rng.uniform(0.15, 0.85) * ly
        cz = rng.uniform(0.2, 0.8) * lz
        a = amp if i % 2 == 0 else -amp
        f *= 1.0 + a * np.exp(-((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) / (2 * sigma ** 2))
    return f


def gradient_model(nx, ny, nz, h, v0=1500.0, g=0.6):
    _, _, z = _coords(nx, ny, nz, h)
    return np.broadcast_to(v0 + g * z, (ny, nx, nz)).astype(np.float32)


def layered_model(rng, nx, ny, nz, h, speeds=(1500.0, 2500.0, 3500.0)):
    x, y, z = _coords(nx, ny, nz, h)
    lz = (nz - 1) * h
    v = np.full((ny, nx, nz), speeds[0], np.float64)
    depths = np.sort(rng.uniform(0.25, 0.75, len(speeds) - 1)) * lz
    for i, d in enumerate(depths):
        ax, ay = rng.uniform(-0.08, 0.08, 2)  # dips (m/m)
        iface = d + ax * (x - (nx - 1) * h / 2) + ay * (y - (ny - 1) * h / 2)
        v = np.where(z >= iface, speeds[i + 1], v)
    return v


def surface_nodes(rng, nx, ny, h, count):
    idx = rng.choice(nx * ny, size=count, replace=False)
    return np.stack([(idx % nx) * h, (idx // nx) * h, np.zeros(count)], 1).astype(np.float32)


def jittered_shots(rng, nx, ny, h, n_side):
    """n_side x n_side surface shots on a jittered regular grid, snapped to nodes."""
    out = []
    for j in range(n_side):
        for i in range(n_side):
            fx = (i + 0.5 + rng.uniform(-0.3, 0.3)) / n_side
            fy = (j + 0.5 + rng.uniform(-0.3, 0.3)) / n_side
            ix = int(np.clip(round(fx * (nx - 1)), 0, nx - 1))
            iy = int(np.clip(round(fy * (ny - 1)), 0, ny - 1))
            out.append((ix * h, iy * h, 0.0))
    return np.asarray(out, np.float32)


def brick_window(rng, n, center, frac_lo=0.6, frac_hi=1.0):
    """A window [a, b) of about frac*n nodes around `center`, a multiple of BRICK at the
    start and at the end (or reaching n)."""
    width = int(round(rng.uniform(frac_lo, frac_hi) * n))
    a = int(np.clip(center - width // 2, 0, max(n - width, 0)))
    b = min(a + width, n)
    a -= a % BRICK
    if b % BRICK and b != n:
        b = min(b + (BRICK - b % BRICK), n)
    return a, b


def crop_window(rng, n, center, frac_lo=0.6, frac_hi=1.0):
    """A window [a, b) of about frac*n nodes around `center`, at any origin."""
    width = max(2, int(round(rng.uniform(frac_lo, frac_hi) * n)))
    a = int(np.clip(center - width // 2, 0, max(n - width, 0)))
    return a, min(a + width, n)


def regular_receivers(n_side, lo, hi):
    c = np.linspace(lo, hi, n_side, dtype=np.float64)
    yy, xx = np.meshgrid(c, c, indexing="ij")
    return np.stack([xx.ravel(), yy.ravel(), np.zeros(xx.size)], 1).astype(np.float32)


def config1(seed=1) -> Survey:
    rng = np.random.default_rng(seed)
    nx, ny, nz, h = 101, 101, 51, 25.0
    v = gradient_model(nx, ny, nz, h).astype(np.float64) * _anomalies(rng, nx, ny, nz, h, 2)
    shot = surface_nodes(rng, nx, ny, h, 1)
    rec = surface_nodes(rng, nx, ny, h, 200)
    return Survey("config1", nx, ny, nz, h, v.astype(np.float32), shot, None, rec)


def config2_model(seed=2, nx=201, ny=201, nz=101, h=12.5):
    rng = np.random.default_rng(seed)
    v = layered_model(rng, nx, ny, nz, h) * _anomalies(rng, nx, ny, nz, h, 8)
    return v.astype(np.float32), rng


def config2(seed=2, nx=201, ny=201, nz=101, h=12.5, n_side=8, aligned=True) -> Survey:
    """aligned=False: each window is the seeded crop itself, at any origin (the solver then
    gathers those windows' slowness node by node); aligned=True rounds the same crops out
    to bricks."""
    v, rng = config2_model(seed, nx, ny, nz, h)
    shots = jittered_shots(rng, nx, ny, h, n_side)
    wins = []
    for sx, sy, _ in shots:
        ix, iy = int(round(sx / h)), int(round(sy / h))
        if not aligned:
            x0, x1 = crop_window(rng, nx, ix)
            y0, y1 = crop_window(rng, ny, iy)
            wins.append((x0, x1, y0, y1))
            continue
        x0, x1 = brick_window(rng, nx, ix)
        y0, y1 = brick_window(rng, ny, iy)
        # the window must contain its shot
        x0 = min(x0, ix - ix % BRICK)
        y0 = min(y0, iy - iy % BRICK)
        x1 = max(x1, min(ix + 1 + (BRICK - (ix + 1) % BRICK) % BRICK, nx))
        y1 = max(y1, min(iy + 1 + (BRICK - (iy + 1) % BRICK) % BRICK, ny))
        wins.append((x0, x1, y0, y1))
    rec = regular_receivers(50, 25.0, 2475.0) if (nx, h) == (201, 12.5) else None
    return Survey("config2", nx, ny, nz, h, v, shots, np.asarray(wins, np.int32), rec)


def config3(seed=2):
    """(true Survey with full windows, starting velocity, inversion settings)."""
    s = config2(seed)
    s = dataclasses.replace(s, name="config3", windows=None, receivers=regular_receivers(50, 25.0, 2475.0))
    start = gradient_model(s.nx, s.ny, s.nz, s.h, 1500.0, 1.0)
    inv = dict(d_tomo=(51.0, 51.0, 52.0), tk_order=2, tk_param=0.1, cg_iterations=30,
               smooth=True, filter_samples=5, standard_deviation=2.0, pick_noise=0.002)
    return s, start, inv


def config5(seed=5) -> Survey:
    rng = np.random.default_rng(seed)
    nx, ny, nz, h = 401, 401, 201, 10.0
    v = layered_model(rng, nx, ny, nz, h) * _anomalies(rng, nx, ny, nz, h, 8)
    shots = jittered_shots(rng, nx, ny, h, 16)
    rec = regular_receivers(100, 20.0, 3980.0)
    return Survey("config5", nx, ny, nz, h, v.astype(np.float32), shots, None, rec)


def config5_inversion(seed=5):
    """(true Survey, starting velocity, inversion settings) of the large device-resident
    inversion: 401x401x201 @10 m, 256 shots x 10,000 receivers, 5 iterations."""
    s = config5(seed)
    start = gradient_model(s.nx, s.ny, s.nz, s.h, 1500.0, 1.0)
    inv = dict(d_tomo=(50.0, 50.0, 50.0), tk_order=2, tk_param=0.1, cg_iterations=30, iterations=5,
               smooth=True, filter_samples=5, standard_deviation=2.0, pick_noise=0.002)
    return s, start, inv


def small(seed, nx, ny, nz, h=25.0, nshots=1, windows=False, layered=True, nrec=16):
    """Small seeded case for parity tests."""
    rng = np.random.default_rng(seed)
    if layered:
        v = layered_model(rng, nx, ny, nz, h) * _anomalies(rng, nx, ny, nz, h, 2, sigma=2.5 * h)
    else:
        v = gradient_model(nx, ny, nz, h).astype(np.float64) * _anomalies(rng, nx, ny, nz, h, 2, sigma=2.5 * h)
    shots = []
    for _ in range(nshots):
        ix, iy = rng.integers(0, nx), rng.integers(0, ny)
        iz = rng.integers(0, max(nz // 3, 1))
        shots.append((ix * h, iy * h, iz * h))
    shots = np.asarray(shots, np.float32)
    wins = None
    if windows:
        wins = []
        for sx, sy, _ in shots:
            ix, iy = int(round(sx / h)), int(round(sy / h))
            x0 = ix - ix % BRICK - BRICK * int(rng.integers(0, 3))
            x1 = ix + 1 + BRICK * int(rng.integers(0, 3))
            y0 = iy - iy % BRICK - BRICK * int(rng.integers(0, 3))
            y1 = iy + 1 + BRICK * int(rng.integers(0, 3))
            x0, y0 = max(x0, 0), max(y0, 0)
            x1 = nx if x1 >= nx else x1 + (BRICK - x1 % BRICK) % BRICK
            y1 = ny if y1 >= ny else y1 + (BRICK - y1 % BRICK) % BRICK
            x1, y1 = min(x1, nx), min(y1, ny)
            if x1 - x0 < 2:
                x1 = min(x0 + BRICK, nx)
            if y1 - y0 < 2:
                y1 = min(y0 + BRICK, ny)
            wins.append((x0, x1, y0, y1))
        wins = np.asarray(wins, np.int32)
    rec = surface_nodes(rng, nx, ny, h, nrec)
    return Survey(f"small{seed}", nx, ny, nz, h, v.astype(np.float32), shots, wins, rec)
