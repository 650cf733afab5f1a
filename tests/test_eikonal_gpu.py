"""Parity of the batched persistent FIM (through the C ABI) against the CPU oracle.

The oracle is the FP64 fixed point of the reference Block_FIM operator
(src/eikonal/block_FIM/cuda_kernel.cu:217-248) with Block_FIM's padding and single-node
source seed (src/eikonal/block_FIM/block_FIM.cpp:142-157, 305-317).  Tolerance: 1e-4
relative traveltime error on nodes with T >= 2h/v_max (the error target of the task); the
measured error is ~1e-6 (FP32 rounding only).  Receiver sampling is checked bit-exact.
"""
import numpy as np
import pytest

from seismic_tomography_3d_b200 import workloads as wl

pytestmark = pytest.mark.gpu

REL_TOL = 1e-4


def rel_err(T, Tref, h, vmax):
    m = Tref >= 2.0 * h / vmax
    return float(np.max(np.abs(T[m] - Tref[m]) / Tref[m])) if m.any() else 0.0


def solve_oracle(oracle_mod, v, h, shot, window=None):
    s = (1.0 / v).astype(np.float32)
    sx, sy, sz = map(float, shot)
    if window is not None:
        x0, x1, y0, y1 = window
        s = s[y0:y1, x0:x1, :]
        sx -= np.float32(x0) * np.float32(h)
        sy -= np.float32(y0) * np.float32(h)
    T, _ = oracle_mod.fim_jw(s, h, (sx, sy, sz))
    return T


BRICKS = {"4^3": 1, "8^3": 2}  # TOMO_BRICK_4, TOMO_BRICK_8


@pytest.mark.parametrize("brick", sorted(BRICKS))
@pytest.mark.parametrize("dims", [(13, 11, 9), (16, 16, 16), (21, 17, 10), (33, 29, 18)])
def test_single_shot_matches_oracle(tomo, oracle_mod, dims, brick):
    """Both brick shapes; odd brick counts (13 x 11 x 9 pads to 4 x 3 x 3 bricks) leave
    partial 8^3 groups at the far edges."""
    nx, ny, nz = dims
    sv = wl.small(sum(dims), nx, ny, nz, nshots=1)
    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        _, st = ctx.eik_solve(sv.shots, brick=BRICKS[brick])
        assert st["nodes_per_brick"] == (64 if brick == "4^3" else 512)
        T = ctx.eik_volume(0)
    Tref = solve_oracle(oracle_mod, sv.velocity, sv.h, sv.shots[0])
    assert T.shape == Tref.shape
    assert rel_err(T, Tref, sv.h, sv.velocity.max()) < REL_TOL


def test_constant_velocity_corner_and_interior(tomo, oracle_mod):
    nx, ny, nz, h = 24, 20, 12, 10.0
    v = np.full((ny, nx, nz), 2000.0, np.float32)
    shots = np.array([[0, 0, 0], [110.0, 90.0, 40.0], [230.0, 190.0, 110.0]], np.float32)
    with tomo.Context(nx, ny, nz, h) as ctx:
        ctx.set_velocity(v)
        ctx.eik_solve(shots)
        for i, sh in enumerate(shots):
            T = ctx.eik_volume(i)
            Tref = solve_oracle(oracle_mod, v, h, sh)
            assert rel_err(T, Tref, h, 2000.0) < REL_TOL
            # the axis through the source is exactly |x - xs| * s (1D operator)
            ix, iy, iz = (int(round(c / h)) for c in sh)
            line = T[iy, :, iz].astype(np.float64)
            exact = np.abs(np.arange(nx) * h - sh[0]) / 2000.0
            assert np.max(np.abs(line - exact)) < 1e-5


def test_off_node_source(tomo, oracle_mod):
    nx, ny, nz, h = 18, 18, 10, 20.0
    sv = wl.small(7, nx, ny, nz, h=h)
    shot = np.array([[101.3, 77.7, 13.1]], np.float32)
    with tomo.Context(nx, ny, nz, h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(shot)
        T = ctx.eik_volume(0)
    Tref = solve_oracle(oracle_mod, sv.velocity, h, shot[0])
    assert rel_err(T, Tref, h, sv.velocity.max()) < REL_TOL


def test_batched_windows_match_cropped_oracle(tomo, oracle_mod):
    nx, ny, nz = 37, 30, 14
    sv = wl.small(11, nx, ny, nz, nshots=6, windows=True)
    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots, windows=sv.windows)
        for i in range(len(sv.shots)):
            assert ctx.eik_window(i) == tuple(sv.windows[i])
            T = ctx.eik_volume(i)
            Tref = solve_oracle(oracle_mod, sv.velocity, sv.h, sv.shots[i], sv.windows[i])
            assert T.shape == Tref.shape
            assert rel_err(T, Tref, sv.h, sv.velocity.max()) < REL_TOL


def _any_windows(rng, sv, n):
    """Windows of any origin and end (not brick-aligned) around each shot."""
    wins = []
    for sx, sy, _ in sv.shots[:n]:
        ix, iy = int(round(sx / sv.h)), int(round(sy / sv.h))
        x0 = int(rng.integers(max(0, ix - 9), ix + 1))
        y0 = int(rng.integers(max(0, iy - 9), iy + 1))
        x1 = int(rng.integers(ix + 1, min(sv.nx, ix + 10) + 1))
        y1 = int(rng.integers(iy + 1, min(sv.ny, iy + 10) + 1))
        wins.append((x0, max(x1, x0 + 2), y0, max(y1, y0 + 2)))
    return np.asarray(wins, np.int32)


@pytest.mark.parametrize("brick", sorted(BRICKS))
def test_unaligned_windows_match_cropped_oracle(tomo, oracle_mod, brick):
    """Windows of any origin and end: each reads its slowness node by node from the shared
    model, its padding replicating the window's edge (the cropped model padded as the
    reference pads a model), so each windowed solve equals the oracle on the cropped model;
    the receivers follow the window's offset."""
    nx, ny, nz = 37, 30, 14
    sv = wl.small(23, nx, ny, nz, nshots=6, nrec=30)
    wins = _any_windows(np.random.default_rng(23), sv, 6)
    assert np.any(wins[:, 0] % 4) and np.any(wins[:, 1] % 4)
    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        t_recv, _ = ctx.eik_solve(sv.shots, windows=wins, receivers=sv.receivers, brick=BRICKS[brick])
        for i in range(len(sv.shots)):
            assert ctx.eik_window(i) == tuple(wins[i])
            T = ctx.eik_volume(i)
            Tref = solve_oracle(oracle_mod, sv.velocity, sv.h, sv.shots[i], wins[i])
            assert T.shape == Tref.shape
            assert rel_err(T, Tref, sv.h, sv.velocity.max()) < REL_TOL
            # receivers inside the window: sampled from the window's own field
            x0, x1, y0, y1 = (int(a) for a in wins[i])
            rx = sv.receivers[:, 0] - np.float32(x0) * np.float32(sv.h)
            ry = sv.receivers[:, 1] - np.float32(y0) * np.float32(sv.h)
            inside = (rx >= 0) & (ry >= 0) & (rx <= (x1 - x0 - 1) * sv.h) & (ry <= (y1 - y0 - 1) * sv.h)
            ref = oracle_mod.first_arrival(T, sv.h, rx[inside], ry[inside], sv.receivers[inside, 2])
            np.testing.assert_array_equal(t_recv[i][inside], ref)
            assert np.all(t_recv[i][~inside] >= 1e5)


@pytest.mark.parametrize("brick", sorted(BRICKS))
def test_unaligned_window_edge_cases(tomo, oracle_mod, brick):
    """Unaligned origins against the model's far edges (37 x 30 is not a multiple of 4, so
    the model's own padding and the window's meet), a 2-node-wide window, and a window whose
    padding is all replicated edge, in one batch with an aligned one."""
    nx, ny, nz = 37, 30, 14
    sv = wl.small(31, nx, ny, nz, nshots=1)
    wins = np.array([[33, 37, 0, 30], [1, 3, 27, 30], [5, 37, 2, 29], [9, 15, 6, 7 + 2], [0, 36, 0, 28]],
                    np.int32)
    shots = np.array([[(w[0] + (w[1] - w[0]) // 2) * sv.h, (w[2] + (w[3] - w[2]) // 2) * sv.h, 2 * sv.h]
                      for w in wins], np.float32)
    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(shots, windows=wins, brick=BRICKS[brick])
        for i in range(len(wins)):
            T = ctx.eik_volume(i)
            Tref = solve_oracle(oracle_mod, sv.velocity, sv.h, shots[i], wins[i])
            assert T.shape == Tref.shape
            assert rel_err(T, Tref, sv.h, sv.velocity.max()) < REL_TOL, i


def test_batch_equals_single_solves(tomo):
    nx, ny, nz = 29, 26, 13
    sv = wl.small(5, nx, ny, nz, nshots=5)
    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots)
        batch = [ctx.eik_volume(i) for i in range(len(sv.shots))]
        for i in range(len(sv.shots)):
            ctx.eik_solve(sv.shots[i:i + 1])
            one = ctx.eik_volume(0)
            assert rel_err(batch[i], one, sv.h, sv.velocity.max()) < 1e-5


def test_receivers_bit_exact_vs_oracle_trilinear(tomo, oracle_mod):
    nx, ny, nz = 25, 23, 11
    sv = wl.small(3, nx, ny, nz, nshots=2, nrec=40)
    rec = sv.receivers.copy()
    rng = np.random.default_rng(0)
    rec[:20, 0] += rng.uniform(0, sv.h, 20).astype(np.float32)  # off-node receivers
    rec[:20, 1] += rng.uniform(0, sv.h, 20).astype(np.float32)
    rec[:, 0] = np.minimum(rec[:, 0], (nx - 1) * sv.h)
    rec[:, 1] = np.minimum(rec[:, 1], (ny - 1) * sv.h)
    rec[:10, 2] = rng.uniform(0, (nz - 1) * sv.h, 10).astype(np.float32)
    rec[-1] = ((nx - 1) * sv.h, (ny - 1) * sv.h, (nz - 1) * sv.h)  # last node: the reference's wrap case
    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        t_recv, _ = ctx.eik_solve(sv.shots, receivers=rec)
        for i in range(len(sv.shots)):
            T = ctx.eik_volume(i)
            ref = oracle_mod.first_arrival(T, sv.h, rec[:, 0], rec[:, 1], rec[:, 2])
            np.testing.assert_array_equal(t_recv[i], ref)


@pytest.mark.parametrize("tol", [{}, dict(change_tol=1e-5, inner_tol=1e-6)], ids=["default", "timed"])
def test_brick8_windowed_batch_matches_oracle(tomo, oracle_mod, tol):
    """8^3 bricks on a windowed batch (windows of any brick-aligned origin, so groups start
    at odd bricks of the model) with receivers: every shot against the oracle on its cropped
    window, and the receiver times against the 4^3 solve's at the same tolerances."""
    sv = wl.small(57, 52, 44, 26, nshots=6, windows=True, nrec=24)
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        t4, _ = ctx.eik_solve(sv.shots, windows=sv.windows, receivers=sv.receivers, brick=1, **tol)
        t8, st = ctx.eik_solve(sv.shots, windows=sv.windows, receivers=sv.receivers, brick=2, **tol)
        assert st["activations"] > 0 and st["nodes_per_brick"] == 512
        for i, sh in enumerate(sv.shots):
            Tref = solve_oracle(oracle_mod, sv.velocity, sv.h, sh, sv.windows[i])
            assert rel_err(ctx.eik_volume(i), Tref, sv.h, sv.velocity.max()) < REL_TOL
    fin = t4 < 1e5
    assert np.array_equal(fin, t8 < 1e5)
    m = fin & (t4 >= 2.0 * sv.h / float(sv.velocity.max()))
    np.testing.assert_allclose(t8[m], t4[m], rtol=REL_TOL)


def test_repeat_runs_agree(tomo):
    nx, ny, nz = 40, 36, 20
    sv = wl.small(9, nx, ny, nz, nshots=4)
    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots)
        a = [ctx.eik_volume(i) for i in range(4)]
        ctx.eik_solve(sv.shots)
        b = [ctx.eik_volume(i) for i in range(4)]
    for x, y in zip(a, b):
        assert rel_err(x, y, sv.h, sv.velocity.max()) < 1e-5


def test_errors_are_status_codes(tomo):
    nx, ny, nz, h = 12, 12, 8, 10.0
    v = np.full((ny, nx, nz), 1500.0, np.float32)
    with tomo.Context(nx, ny, nz, h) as ctx:
        with pytest.raises(tomo.TomoError) as e:
            ctx.eik_solve([[5.0, 5.0, 0.0]])  # no model yet
        assert e.value.status == -6
        ctx.set_velocity(v)
        with pytest.raises(tomo.TomoError) as e:
            ctx.eik_solve([[500.0, 5.0, 0.0]])  # outside
        assert e.value.status == -1
        with pytest.raises(tomo.TomoError) as e:
            ctx.eik_solve([[5.0, 5.0, 0.0]], windows=[[0, 13, 0, 12]])  # window beyond the model
        assert e.value.status == -1
        with pytest.raises(tomo.TomoError) as e:
            ctx.eik_solve([[5.0, 5.0, 0.0]], windows=[[1, 12, 0, 12]])  # shot outside its window
        assert e.value.status == -1
        with pytest.raises(tomo.TomoError) as e:
            ctx.eik_solve([[50.0, 50.0, 0.0]], max_rounds=2, schedule=1)  # round cap
        assert e.value.status == -4
        t, st = ctx.eik_solve([[50.0, 50.0, 0.0]], schedule=1)  # context still usable
        assert st["rounds"] > 2
        with pytest.raises(tomo.TomoError) as e:  # asynchronous schedule: activation cap
            ctx.eik_solve([[50.0, 50.0, 0.0]], max_rounds=1, max_inner=1, schedule=2)
        assert e.value.status == -4
        ctx.eik_solve([[50.0, 50.0, 0.0]], schedule=2)


def test_barrier_wait_limit_returns_timeout(tomo, oracle_mod):
    """tomo_eik_opts.spin_limit bounds the round barrier's wait.  With a limit of one poll
    the blocks waiting at the first barrier (for the one warp relaxing the source brick)
    give up: every block leaves the launch, the call returns TOMO_ERR_TIMEOUT, and the
    context solves the batch correctly afterwards.  A bounded wait on the device, no fault:
    the reference waits without bound (cuda_kernel.cu:91)."""
    sv = wl.small(44, 24, 20, 12, nshots=2)
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        with pytest.raises(tomo.TomoError) as e:
            ctx.eik_solve(sv.shots, spin_limit=1)
        assert e.value.status == -5  # TOMO_ERR_TIMEOUT
        with pytest.raises(tomo.TomoError) as e:  # no solve to read after the timeout
            ctx.eik_volume(0)
        assert e.value.status == -6
        ctx.eik_solve(sv.shots)
        for i, sh in enumerate(sv.shots):
            Tref = solve_oracle(oracle_mod, sv.velocity, sv.h, sh)
            assert rel_err(ctx.eik_volume(i), Tref, sv.h, sv.velocity.max()) < REL_TOL


@pytest.mark.slow
def test_config1_full_size(tomo, oracle_mod):
    sv = wl.config1()
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        t_recv, st = ctx.eik_solve(sv.shots, receivers=sv.receivers)
        T = ctx.eik_volume(0)
    Tref = solve_oracle(oracle_mod, sv.velocity, sv.h, sv.shots[0])
    assert rel_err(T, Tref, sv.h, sv.velocity.max()) < REL_TOL
    ref_recv = oracle_mod.first_arrival(Tref.astype(np.float32), sv.h, *sv.receivers.T)
    m = ref_recv >= 2 * sv.h / sv.velocity.max()
    assert np.max(np.abs(t_recv[0][m] - ref_recv[m]) / ref_recv[m]) < REL_TOL


def test_autotune_picks_a_shape_and_keeps_results(tomo):
    """tomo_eik_autotune times the launch shapes, keeps the fastest in the context, and the
    tuned solve converges to the same field as the default one."""
    sv = wl.small(5, 48, 40, 24, nshots=4, windows=True)
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots, windows=sv.windows)
        ref = [ctx.eik_volume(i) for i in range(len(sv.shots))]
        shape, st = ctx.eik_autotune(sv.shots, windows=sv.windows, repeats=1)
        # 36 + 6 + 8 launch shapes (4^3, two 4^3 bricks per warp, 8^3), 4 time bands, and the
        # 12 warps x occupancy shapes again if a band won
        assert st["trials"] in (54, 66)
        assert shape["brick"] in (1, 2)
        assert shape["schedule"] in (0, 3)
        assert shape["schedule"] == 0 or (shape["brick"] == 1 and shape["time_band"] == 0.0)
        assert shape["block_warps"] in (4, 8, 16) and shape["occupancy"] in (2, 3, 4, 5, 6)
        assert shape["max_inner"] in (8, 16, 32)
        assert shape["time_band"] >= 0.0
        assert 0 < st["best_ms"] <= st["default_ms"]
        ctx.eik_solve(sv.shots, windows=sv.windows)
        for i in range(len(sv.shots)):
            assert rel_err(ctx.eik_volume(i), ref[i], sv.h, float(sv.velocity.max())) < 1e-5


@pytest.mark.parametrize("windows", [False, True])
def test_async_and_round_schedules_agree(tomo, windows):
    """The asynchronous schedule and the round-synchronous one (default) relax the bricks in
    different orders towards the same fixed point."""
    sv = wl.small(31, 52, 44, 26, nshots=6, windows=windows)
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots, windows=sv.windows, schedule=1, change_tol=-1.0)
        ref = [ctx.eik_volume(i) for i in range(len(sv.shots))]
        _, st = ctx.eik_solve(sv.shots, windows=sv.windows, change_tol=-1.0, schedule=2)
        assert st["rounds"] == 0 and st["activations"] > 0
        for i in range(len(sv.shots)):
            assert rel_err(ctx.eik_volume(i), ref[i], sv.h, float(sv.velocity.max())) < 1e-6


@pytest.mark.parametrize("band", [0.01, 0.2])
def test_time_band_ordering_same_fixed_point(tomo, oracle_mod, band):
    """Time-band ordering (tomo_eik_opts.time_band) only changes when queued bricks are
    relaxed.  On a smooth v(z) model, where a surface path reaches bricks before the
    diving one and many bricks are put off, the solve reaches the oracle's fixed point and,
    with every drop re-queued, the unordered solve's field."""
    nx, ny, nz, h = 48, 44, 28, 25.0
    v = np.ascontiguousarray(wl.gradient_model(nx, ny, nz, h, 1500.0, 1.0))
    shots = np.array([[0.0, 0.0, 0.0], [600.0, 500.0, 0.0], [1175.0, 1075.0, 100.0]], np.float32)
    with tomo.Context(nx, ny, nz, h) as ctx:
        ctx.set_velocity(v)
        _, st0 = ctx.eik_solve(shots, want_recv=False, change_tol=-1.0)
        T0 = [ctx.eik_volume(i) for i in range(len(shots))]
        _, st1 = ctx.eik_solve(shots, want_recv=False, change_tol=-1.0, time_band=band)
        T1 = [ctx.eik_volume(i) for i in range(len(shots))]
        # the bench tolerances with the band
        ctx.eik_solve(shots, want_recv=False, change_tol=1e-5, inner_tol=1e-6, time_band=band)
        T2 = [ctx.eik_volume(i) for i in range(len(shots))]
    assert st0["deferred"] == 0
    if band < 0.05:
        assert st1["deferred"] > 0
    for i, sh in enumerate(shots):
        Tref = solve_oracle(oracle_mod, v, h, sh)
        assert rel_err(T1[i], Tref, h, float(v.max())) < REL_TOL
        assert rel_err(T2[i], Tref, h, float(v.max())) < REL_TOL
        assert rel_err(T1[i], T0[i], h, float(v.max())) < 1e-6


def test_time_band_values(tomo):
    """A negative band switches the ordering off (even after autotuning); non-finite bands
    are rejected."""
    sv = wl.small(5, 16, 16, 12)
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        _, st = ctx.eik_solve(sv.shots, time_band=-1.0)
        assert st["deferred"] == 0
        for bad in (float("nan"), float("inf"), -float("inf")):
            with pytest.raises(tomo.TomoError):
                ctx.eik_solve(sv.shots, time_band=bad)


def test_staged_velocity_upload(tomo):
    """tomo_stage_velocity / tomo_commit_velocity: the next model is copied while the current
    one is solved; each solve sees the model committed before it, as with tomo_set_velocity."""
    nx, ny, nz = 37, 30, 14
    sv = wl.small(41, nx, ny, nz, nshots=3, nrec=20)
    v1 = sv.velocity
    v2 = (sv.velocity * np.float32(1.1)).astype(np.float32)
    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        with pytest.raises(tomo.TomoError):
            ctx.commit_velocity()  # nothing staged
        ctx.set_velocity(v1)
        r1, _ = ctx.eik_solve(sv.shots, receivers=sv.receivers)
        s1 = ctx.get_slowness()
        ctx.set_velocity(v2)
        r2, _ = ctx.eik_solve(sv.shots, receivers=sv.receivers)
        s2 = ctx.get_slowness()
        ctx.stage_velocity(v1)
        ctx.commit_velocity()
        ctx.stage_velocity(v2)  # copied while the next solve runs
        q1, _ = ctx.eik_solve(sv.shots, receivers=sv.receivers)
        np.testing.assert_array_equal(ctx.get_slowness(), s1)
        ctx.commit_velocity()
        q2, _ = ctx.eik_solve(sv.shots, receivers=sv.receivers)
        np.testing.assert_array_equal(ctx.get_slowness(), s2)
        with pytest.raises(tomo.TomoError):
            ctx.commit_velocity()  # the staged model was used
    np.testing.assert_allclose(q1, r1, rtol=1e-5)
    np.testing.assert_allclose(q2, r2, rtol=1e-5)
    m = r1 > 0
    assert np.min(r1[m] / r2[m]) > 1.09  # the models differ: times scale by 1 / 1.1
    assert np.max(np.abs(r2[m] * 1.1 - r1[m]) / r1[m]) < 1e-4


@pytest.mark.parametrize("dims", [(13, 11, 9), (33, 29, 18)])
def test_pair_schedule_matches_oracle(tomo, oracle_mod, dims):
    """TOMO_SCHED_PAIR (two bricks per warp, a y-column of four nodes per lane) at the
    launch shapes the autotuner tries, single shots and a windowed batch (odd brick counts
    leave the last warp with one brick), against the oracle on the cropped windows."""
    nx, ny, nz = dims
    sv = wl.small(sum(dims) + 7, nx, ny, nz, nshots=5, windows=True)
    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        for bw, occ in ((8, 3), (4, 3), (16, 4)):
            ctx.eik_solve(sv.shots, windows=sv.windows, schedule=3, block_warps=bw, occupancy=occ)
            for i in range(len(sv.shots)):
                Tref = solve_oracle(oracle_mod, sv.velocity, sv.h, sv.shots[i], sv.windows[i])
                assert rel_err(ctx.eik_volume(i), Tref, sv.h, sv.velocity.max()) < REL_TOL, (bw, occ, i)


def test_pair_schedule_unaligned_windows(tomo, oracle_mod):
    """Two bricks per warp on windows of any origin (slowness gathered node by node)."""
    nx, ny, nz = 37, 30, 14
    sv = wl.small(23, nx, ny, nz, nshots=6, nrec=30)
    wins = _any_windows(np.random.default_rng(23), sv, 6)
    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots, windows=wins, schedule=3, block_warps=8, occupancy=3)
        for i in range(len(sv.shots)):
            Tref = solve_oracle(oracle_mod, sv.velocity, sv.h, sv.shots[i], wins[i])
            assert rel_err(ctx.eik_volume(i), Tref, sv.h, sv.velocity.max()) < REL_TOL, i


def test_repeated_batches_change_receivers_and_shots(tomo):
    """A context keeps the receivers and shot descriptors of the last batch on the device and
    uploads a batch's only when they differ: after solves with other receivers, other shots
    and other windows (same counts), each result equals the same solve in a fresh context."""
    nx, ny, nz, h = 29, 27, 14, 25.0
    sv_a = wl.small(61, nx, ny, nz, h=h, nshots=4, windows=True, nrec=20)
    sv_b = wl.small(62, nx, ny, nz, h=h, nshots=4, windows=True, nrec=20)
    rec_a = sv_a.receivers
    rec_b = rec_a.copy()
    rec_b[:, 0] = np.minimum(rec_b[:, 0] + np.float32(h / 3), np.float32((nx - 1) * h))
    steps = [(sv_a.shots, sv_a.windows, rec_a), (sv_a.shots, sv_a.windows, rec_b),
             (sv_b.shots, sv_b.windows, rec_b), (sv_b.shots, None, rec_b), (sv_a.shots, sv_a.windows, rec_a)]
    kw = dict(change_tol=-1.0, inner_tol=0.0)  # converged fields: no schedule-level rounding
    with tomo.Context(nx, ny, nz, h) as ctx:
        ctx.set_velocity(sv_a.velocity)
        for shots, wins, rec in steps:
            t, _ = ctx.eik_solve(shots, windows=wins, receivers=rec, **kw)
            with tomo.Context(nx, ny, nz, h) as fresh:
                fresh.set_velocity(sv_a.velocity)
                t_ref, _ = fresh.eik_solve(shots, windows=wins, receivers=rec, **kw)
            np.testing.assert_allclose(t, t_ref, rtol=1e-5, atol=0)
