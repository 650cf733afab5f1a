"""TOMO_OP_NGB: the reference's Accurate_FSM (Noble, Gesret & Belayouni 2014 fast sweeping)
on the device, compared BIT FOR BIT with the reference's own CPU solver (golden volumes
from oracle/_ref, tests/golden/eik_ref.npz) and with the oracle's FP32 restatement."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden as mg  # noqa: E402

from seismic_tomography_3d_b200 import workloads as wl  # noqa: E402

pytestmark = pytest.mark.gpu
NGB = 1


def test_matches_reference_fsm_golden(tomo):
    """Default schedule (tiled where every source lies off its window's far faces, plane
    otherwise) against the reference's own FSM volumes."""
    g = np.load(os.path.join(HERE, "golden", "eik_ref.npz"))
    for seed, nx, ny, nz, h, shots in mg.EIK_CASES:
        v, sh = g[f"v_{seed}"], g[f"shots_{seed}"]
        with tomo.Context(nx, ny, nz, h) as ctx:
            ctx.set_velocity(v)
            ctx.eik_solve(sh, op=NGB)
            for i in range(len(sh)):
                np.testing.assert_array_equal(ctx.eik_volume(i), g[f"fsm_{seed}"][i])


def test_matches_oracle_on_config1_and_receivers(tomo, oracle_mod):
    sv = wl.config1()
    s = (np.float32(1.0) / sv.velocity).astype(np.float32)
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        t_recv, _ = ctx.eik_solve(sv.shots, receivers=sv.receivers, op=NGB)
        T = ctx.eik_volume(0)
    T_ref, _ = oracle_mod.fsm_ngb(s, sv.h, tuple(map(float, sv.shots[0])), 0)
    np.testing.assert_array_equal(T, T_ref)
    np.testing.assert_array_equal(t_recv[0], oracle_mod.first_arrival(T_ref, sv.h, *sv.receivers.T))


@pytest.mark.parametrize("groups", [0, 1, 3])
def test_windowed_batch_matches_cropped_oracle(tomo, oracle_mod, groups):
    """groups 0: the tile-wavefront schedule (default); 1, 3: the plane schedule with that
    many independent block groups.  Both reproduce the sequential sweeps bit for bit."""
    nx, ny, nz = 37, 30, 14
    sv = wl.small(11, nx, ny, nz, nshots=6, windows=True)
    s = (np.float32(1.0) / sv.velocity).astype(np.float32)
    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots, windows=sv.windows, op=NGB, sweep_groups=groups)
        for i in range(len(sv.shots)):
            x0, x1, y0, y1 = sv.windows[i]
            sx = float(np.float32(sv.shots[i][0]) - np.float32(x0) * np.float32(sv.h))
            sy = float(np.float32(sv.shots[i][1]) - np.float32(y0) * np.float32(sv.h))
            T_ref, _ = oracle_mod.fsm_ngb(np.ascontiguousarray(s[y0:y1, x0:x1, :]), sv.h, (sx, sy, float(sv.shots[i][2])), 0)
            np.testing.assert_array_equal(ctx.eik_volume(i), T_ref)


def test_ngb_batch_feeds_ray_tracing(tomo, oracle_mod):
    """The sweep result lands in the same device pool the ray tracer reads."""
    nx, ny, nz, h = 33, 29, 15, 25.0
    sv = wl.small(4, nx, ny, nz, h=h, nshots=2, nrec=12)
    with tomo.Context(nx, ny, nz, h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots, receivers=sv.receivers, op=NGB)
        vols = [ctx.eik_volume(i) for i in range(2)]
        st = ctx.build_jacobian((100.0, 100.0, 100.0), 2, 0.1, max_ray_steps=6000)
        rp, cols, vals = ctx.jacobian()
    nt = [int(np.float32((n - 1) * np.float32(h)) / np.float32(100.0)) + 1 for n in (nx, ny, nz)]
    got = []
    for i in range(2):
        rt = oracle_mod.raytrace(vols[i], h, sv.shots[i], *sv.receivers.T, (100.0,) * 3, nt, max_steps=6000)
        got.append(rt["cols"])
    np.testing.assert_array_equal(cols[:st["nnz_rays"]], np.concatenate(got))



def test_unaligned_windows_bit_exact(tomo, oracle_mod):
    """NGB sweeps on windows of any origin and end (sources off the far faces): the tile
    schedule, bit for bit against the oracle's sequential sweeps on the cropped model."""
    nx, ny, nz, h = 37, 30, 14, 25.0
    sv = wl.small(23, nx, ny, nz, h=h, nshots=5)  # no source on the last node of an axis
    rng = np.random.default_rng(29)
    wins = []
    for sx, sy, _ in sv.shots:
        ix, iy = int(round(sx / h)), int(round(sy / h))
        x0, y0 = int(rng.integers(max(0, ix - 7), ix + 1)), int(rng.integers(max(0, iy - 7), iy + 1))
        x1 = min(nx, ix + 2 + int(rng.integers(0, 8)))
        y1 = min(ny, iy + 2 + int(rng.integers(0, 8)))
        wins.append((x0, x1, y0, y1))
    wins = np.asarray(wins, np.int32)
    # every source off the far faces of its window: the tile schedule runs
    assert np.all(np.round(sv.shots[:, 0] / h) < wins[:, 1] - 1) and np.all(np.round(sv.shots[:, 1] / h) < wins[:, 3] - 1)
    s = (np.float32(1.0) / sv.velocity).astype(np.float32)
    with tomo.Context(nx, ny, nz, h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots, windows=wins, op=NGB)
        for i in range(len(sv.shots)):
            x0, x1, y0, y1 = wins[i]
            sx = float(np.float32(sv.shots[i][0]) - np.float32(x0) * np.float32(h))
            sy = float(np.float32(sv.shots[i][1]) - np.float32(y0) * np.float32(h))
            T_ref, _ = oracle_mod.fsm_ngb(np.ascontiguousarray(s[y0:y1, x0:x1, :]), h, (sx, sy, float(sv.shots[i][2])), 0)
            np.testing.assert_array_equal(ctx.eik_volume(i), T_ref)


def test_ngb_wait_limit_returns_timeout(tomo):
    """The tile schedule's bounded waits -- grid barriers, upwind-tile flags and the per-shot
    sweep counts of a batch: with a limit of one poll they give up, the call returns
    TOMO_ERR_TIMEOUT, and the context then solves the batch to the same bits as before."""
    sv = wl.small(45, 24, 20, 12, nshots=3)  # every source off the far faces: tile schedule
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots, op=1)
        ref = [ctx.eik_volume(i) for i in range(len(sv.shots))]
        with pytest.raises(tomo.TomoError) as e:
            ctx.eik_solve(sv.shots, op=1, spin_limit=1)
        assert e.value.status == -5  # TOMO_ERR_TIMEOUT
        ctx.eik_solve(sv.shots, op=1)
        for i in range(len(sv.shots)):
            np.testing.assert_array_equal(ctx.eik_volume(i), ref[i])
