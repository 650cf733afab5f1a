"""Parity at the configured sizes, in the settings the benchmark times.

* Config 2 (201 x 201 x 101 at 12.5 m, 64 shots on brick-aligned windows of 60-100 % of
  the lateral extent) solved in one batch at the timed tolerances
  (workloads.TIMED_TOLERANCES): every shot's field against the FP64 fixed point of the
  Block_FIM operator on its cropped window (src/eikonal/block_FIM/cuda_kernel.cu:217-248,
  block_FIM.cpp:142-157, 305-317), <= 1e-4 relative on nodes with T >= 2h/v_max, and the
  receiver times sampled from it.
* One config-2 shot on the NGB operator, bit for bit against the reference's own
  Accurate_FSM (src/eikonal/accurate_FSM/accurate_FSM.cpp:577-650, oracle/_ref).
* Config 3 (64 shots x 2,500 receivers, 50 x 50 x 25 cells): the whole Jacobian built
  from the device's fields, bit for bit against the oracle's ray tracer
  (least_squares.cpp:192-280) for every shot; and one full iteration (eikonal at the timed
  banded tolerances, rays, Tikhonov, CGLS with the reference's 10 iterations, model update
  with smoothing) against the oracle pipeline run from its own FP64 fields
  (least_squares.cpp:163-570): recovered models within 0.5 % RMS.
* Config 5 (401 x 401 x 201, 256 shots x 10,000 receivers): all shots solved and
  ray-traced in one context; the first and the last shot's fields against the FP64
  oracle and their Jacobian rows bit for bit against the oracle's ray tracer.  The
  oracle pipeline over all 256 shots (hours on the host) is left to config 3.

The oracle runs on the host's cores in threads (its C routines release the GIL).
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

from seismic_tomography_3d_b200 import workloads as wl

pytestmark = pytest.mark.gpu

REL_TOL = 1e-4
THREADS = max(1, min(32, os.cpu_count() or 1))


def _crop(v, window, shot, h):
    x0, x1, y0, y1 = (int(a) for a in window)
    s = np.ascontiguousarray((np.float32(1.0) / v[y0:y1, x0:x1, :]).astype(np.float32))
    sx = float(np.float32(shot[0]) - np.float32(x0) * np.float32(h))
    sy = float(np.float32(shot[1]) - np.float32(y0) * np.float32(h))
    return s, (sx, sy, float(shot[2]))


def test_config2_batch_at_timed_tolerances_vs_fp64_oracle(tomo, oracle_mod):
    sv = wl.config2()
    vmax = float(sv.velocity.max())
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        t_recv, st = ctx.eik_solve(sv.shots, windows=sv.windows, receivers=sv.receivers, **wl.TIMED_TOLERANCES)
        vols = [ctx.eik_volume(i) for i in range(len(sv.shots))]

    def check(i):
        s, src = _crop(sv.velocity, sv.windows[i], sv.shots[i], sv.h)
        Tref, _ = oracle_mod.fim_jw(s, sv.h, src)
        m = Tref >= 2.0 * sv.h / vmax
        err = float(np.max(np.abs(vols[i][m] - Tref[m]) / Tref[m]))
        # receivers inside the window, sampled from the oracle field
        x0, x1, y0, y1 = (int(a) for a in sv.windows[i])
        rx = sv.receivers[:, 0] - np.float32(x0) * np.float32(sv.h)
        ry = sv.receivers[:, 1] - np.float32(y0) * np.float32(sv.h)
        inside = (rx >= 0) & (ry >= 0) & (rx <= (x1 - x0 - 1) * sv.h) & (ry <= (y1 - y0 - 1) * sv.h)
        r_ref = oracle_mod.first_arrival(Tref.astype(np.float32), sv.h, rx[inside], ry[inside],
                                         sv.receivers[inside, 2])
        got = t_recv[i][inside]
        mr = r_ref >= 2.0 * sv.h / vmax
        rerr = float(np.max(np.abs(got[mr] - r_ref[mr]) / r_ref[mr])) if mr.any() else 0.0
        outside_inf = bool(np.all(t_recv[i][~inside] >= 1e5))
        return err, rerr, outside_inf

    with cf.ThreadPoolExecutor(THREADS) as ex:
        res = list(ex.map(check, range(len(sv.shots))))
    errs = np.array([r[0] for r in res])
    rerrs = np.array([r[1] for r in res])
    print(f"config 2, 64 shots at {wl.TIMED_TOLERANCES}: field max rel err {errs.max():.3e} "
          f"(median {np.median(errs):.3e}); receivers {rerrs.max():.3e}; activations {st['activations']}")
    assert errs.max() < REL_TOL
    assert rerrs.max() < REL_TOL
    assert all(r[2] for r in res)


def test_config2_shot_ngb_bit_exact_vs_reference_fsm(tomo, oracle_mod):
    if not oracle_mod.have_ref():
        pytest.skip("oracle/_ref (the reference's own solvers) not built")
    sv = wl.config2()
    areas = [(w[1] - w[0]) * (w[3] - w[2]) for w in sv.windows]
    picks = [int(np.argmax(areas)), int(np.argmin(areas))]  # the largest and the smallest window
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots[picks], windows=sv.windows[picks], op=1)
        got = [ctx.eik_volume(i) for i in range(len(picks))]
    for k, i in enumerate(picks):
        x0, x1, y0, y1 = (int(a) for a in sv.windows[i])
        v = np.ascontiguousarray(sv.velocity[y0:y1, x0:x1, :])
        shot = np.array([[np.float32(sv.shots[i][0]) - np.float32(x0) * np.float32(sv.h),
                          np.float32(sv.shots[i][1]) - np.float32(y0) * np.float32(sv.h), sv.shots[i][2]]], np.float32)
        T_ref, _ = oracle_mod.ref_solve(oracle_mod.REF_FSM, v, sv.h, shot)
        np.testing.assert_array_equal(got[k], T_ref[0])


def _n_tomo(sv, d):
    return [int(np.float32((n - 1) * np.float32(sv.h)) / np.float32(dd)) + 1 for n, dd in zip((sv.nx, sv.ny, sv.nz), d)]


def _oracle_rows(rt, shot, nrec):
    rp = rt["row_ptr"]
    return np.repeat(np.arange(nrec, dtype=np.int64), np.diff(rp)) + shot * nrec


@pytest.fixture(scope="module")
def config3():
    sv, start, inv = wl.config3()
    return sv, start, inv


def test_config3_jacobian_bit_exact_full_size(tomo, oracle_mod, config3):
    sv, start, inv = config3
    nrec = len(sv.receivers)
    d = inv["d_tomo"]
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(start)
        ctx.eik_solve(sv.shots, receivers=sv.receivers, want_recv=False, **wl.TIMED_TOLERANCES_BANDED)
        jst = ctx.build_jacobian(d, inv["tk_order"], inv["tk_param"])
        rp, cols, vals = ctx.jacobian()
        status = ctx.ray_status()
        # fields of every shot, fetched one at a time into the oracle's threads
        nt = _n_tomo(sv, d)
        futs = []
        with cf.ThreadPoolExecutor(THREADS) as ex:
            for i, sh in enumerate(sv.shots):
                T = ctx.eik_volume(i)
                futs.append(ex.submit(oracle_mod.raytrace, T, sv.h, sh, *sv.receivers.T, d, nt, 20000))
            rts = [f.result() for f in futs]
    assert jst["rays"] == len(sv.shots) * nrec
    print(f"config 3 Jacobian: {jst['nnz_rays']} ray non-zeros, rays ok {jst['rays_ok']} stalled "
          f"{jst['rays_stalled']} capped {jst['rays_capped']}")
    np.testing.assert_array_equal(status, np.concatenate([rt["status"] for rt in rts]))
    ng = jst["nnz_rays"]
    assert ng == sum(len(rt["cols"]) for rt in rts)
    rows = np.repeat(np.arange(len(rp) - 1, dtype=np.int64), np.diff(rp))[:ng]
    np.testing.assert_array_equal(rows, np.concatenate([_oracle_rows(rt, i, nrec) for i, rt in enumerate(rts)]))
    np.testing.assert_array_equal(cols[:ng], np.concatenate([rt["cols"] for rt in rts]))
    np.testing.assert_array_equal(vals[:ng], np.concatenate([rt["vals"] for rt in rts]))


def test_config3_iteration_vs_oracle_pipeline(tomo, oracle_mod, config3):
    """One tomography iteration on the device against the oracle pipeline, the reference's
    loop body (tomography_main.cpp:19-30) restated on the CPU from its own FP64 fields."""
    sv, start, inv = config3
    nrec, ns = len(sv.receivers), len(sv.shots)
    d, nt = inv["d_tomo"], _n_tomo(sv, inv["d_tomo"])
    M = nt[0] * nt[1] * nt[2]
    cg = 10  # the reference's hard-coded count (least_squares.cpp:424-496)
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        dobs, _ = ctx.eik_solve(sv.shots, receivers=sv.receivers)
        dobs = (dobs + np.random.default_rng(3).normal(0.0, inv["pick_noise"], dobs.shape)).astype(np.float32)
        ctx.set_velocity(start)
        ctx.eik_solve(sv.shots, receivers=sv.receivers, want_recv=False, **wl.TIMED_TOLERANCES_BANDED)
        ctx.build_jacobian(d, inv["tk_order"], inv["tk_param"])
        ctx.set_observed(dobs)
        x_dev, _, _ = ctx.cgls(cg)
        vel_dev = ctx.model_update(inv["smooth"], inv["filter_samples"], inv["standard_deviation"])

    # the oracle pipeline: FP64 fields -> receiver times and rays -> [G; lambda L] -> FP64 CGLS
    s_start = (np.float32(1.0) / start).astype(np.float32)

    def shot_rows(i):
        T, _ = oracle_mod.fim_jw(s_start, sv.h, tuple(map(float, sv.shots[i])))
        T = T.astype(np.float32)
        dcal = oracle_mod.first_arrival(T, sv.h, *sv.receivers.T)
        rt = oracle_mod.raytrace(T, sv.h, sv.shots[i], *sv.receivers.T, d, nt, 20000)
        return dcal, _oracle_rows(rt, i, nrec), rt["cols"], rt["vals"]

    with cf.ThreadPoolExecutor(THREADS) as ex:
        parts = list(ex.map(shot_rows, range(ns)))
    dcal = np.concatenate([p[0] for p in parts])
    order = inv["tk_order"]
    coef = (np.float32(inv["tk_param"]) * oracle_mod.tk_coeffs(order).astype(np.float32)).astype(np.float32)
    nL = M - order
    tk_rows = np.repeat(np.arange(nL, dtype=np.int64), order + 1) + ns * nrec
    tk_cols = (np.arange(nL)[:, None] + np.arange(order + 1)[None, :]).ravel().astype(np.int32)
    tk_vals = np.tile(coef, nL)
    iA = np.concatenate([p[1] for p in parts] + [tk_rows]).astype(np.int32)
    jA = np.concatenate([p[2] for p in parts] + [tk_cols]).astype(np.int32)
    vA = np.concatenate([p[3] for p in parts] + [tk_vals]).astype(np.float32)
    N = ns * nrec + nL
    B = np.zeros(N, np.float32)
    B[:ns * nrec] = dobs.ravel() - dcal
    x_or, _ = oracle_mod.cgls_f64(N, M, iA, jA, vA, B, cg)
    s_or, vel_or = oracle_mod.model_update(s_start, sv.h, d, nt, x_or.astype(np.float32), inv["smooth"],
                                           inv["filter_samples"], inv["standard_deviation"])
    rms_model = float(np.sqrt(np.mean(((vel_dev.astype(np.float64) - vel_or) / vel_or) ** 2)))
    dv_or = vel_or.astype(np.float64) - start
    dv_dev = vel_dev.astype(np.float64) - start
    upd = float(np.linalg.norm(dv_dev - dv_or) / np.linalg.norm(dv_or))
    xrel = float(np.linalg.norm(x_dev - x_or) / np.linalg.norm(x_or))
    print(f"config 3 iteration vs oracle pipeline: model RMS {rms_model:.3e}, update rel L2 {upd:.3e}, "
          f"CGLS x rel L2 {xrel:.3e}; update RMS {np.sqrt(np.mean((dv_or / start) ** 2)):.3e}")
    assert rms_model < 5e-3  # recovered models within 0.5 % RMS
    assert upd < 0.1


def test_config5_first_and_last_shot_vs_oracle(tomo, oracle_mod):
    """Config 5 (401 x 401 x 201 at 10 m, 256 full-window shots x 10,000 receivers, 50 m
    cells) solved and ray-traced in one context, as the inversion does: all 256 shots at the
    banded timed tolerances on the layered true model, then the whole Jacobian.  The first
    and the last shot are checked against the oracle.  The last shot's field starts
    8.5 G nodes into the traveltime pool, past 32-bit offsets.
      * fields: the FP64 fixed point of the Block_FIM operator on the whole grid
        (cuda_kernel.cu:217-248), <= 1e-4 relative on nodes with T >= 2h/v_max;
      * rays: status and every row of G bit for bit against the oracle's ray tracer on the
        device's own field (least_squares.cpp:192-280), with one explicit step cap on both
        sides (the device's default cap follows each ray's traveltime instead)."""
    sv, _, inv = wl.config5_inversion()
    nrec, ns = len(sv.receivers), len(sv.shots)
    d = inv["d_tomo"]
    nt = _n_tomo(sv, d)
    cap = 20000
    picks = (0, ns - 1)
    with tomo.Context(sv.nx, sv.ny, sv.nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(sv.shots, receivers=sv.receivers, want_recv=False, **wl.TIMED_TOLERANCES_BANDED)
        jst = ctx.build_jacobian(d, inv["tk_order"], inv["tk_param"], max_ray_steps=cap)
        rp, cols, vals = ctx.jacobian()
        status = ctx.ray_status()
        vols = [ctx.eik_volume(i) for i in picks]
    assert jst["rays"] == ns * nrec
    vmax = float(sv.velocity.max())
    s = (np.float32(1.0) / sv.velocity).astype(np.float32)

    def check(k):
        i = picks[k]
        T = vols[k]
        Tref, _ = oracle_mod.fim_jw(s, sv.h, tuple(map(float, sv.shots[i])))
        m = Tref >= 2.0 * sv.h / vmax
        err = float(np.max(np.abs(T[m] - Tref[m]) / Tref[m]))
        rt = oracle_mod.raytrace(T, sv.h, sv.shots[i], *sv.receivers.T, d, nt, cap)
        return err, rt

    with cf.ThreadPoolExecutor(len(picks)) as ex:
        res = list(ex.map(check, range(len(picks))))
    for (err, rt), i in zip(res, picks):
        lo, hi = i * nrec, (i + 1) * nrec
        print(f"config 5 shot {i}: field max rel err {err:.2e} vs FP64 oracle; "
              f"{int(rp[hi] - rp[lo])} ray non-zeros")
        assert err <= REL_TOL, (i, err)
        np.testing.assert_array_equal(status[lo:hi], rt["status"])
        np.testing.assert_array_equal(np.diff(rp[lo:hi + 1]), np.diff(rt["row_ptr"]))
        np.testing.assert_array_equal(cols[rp[lo]:rp[hi]], rt["cols"])
        np.testing.assert_array_equal(vals[rp[lo]:rp[hi]], rt["vals"])
