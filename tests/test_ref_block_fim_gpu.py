"""The reference's own GPU solver beside this library on the config-1 and config-2 grids.

The reference Block_FIM (src/eikonal/block_FIM/block_FIM.cpp + cuda_kernel.cu, built
unmodified for sm_100a into oracle/_ref/libref_fim.so and driven through its public
`Eikonal` API) solves the shot of config 1 (101 x 101 x 51 @ 25 m, gradient model with two
anomalies) and the first shots of config 2 (201 x 201 x 101 @ 12.5 m, layered model with
anomalies) over the full grid, one shot per `eikonal_equation()` call as the reference
does.  The same shots go through `tomo_eik_solve` as one batch.

Checked: the two traveltime volumes agree within the 1e-4 relative traveltime budget on
nodes with T >= 2h/v_max (same Jeong-Whitaker operator and source seed; the two differ only
in convergence control and FP32 rounding order), and the batched solve is faster per shot.
The measured times (the reference's per-shot wall time of `eikonal_equation()`, which
includes its per-shot allocations, host bricking and copies; this library's per-shot time
of the batch) are printed and, when TOMO_REF_GPU_JSON names a file, added to it under the
case's name.
"""
import json
import os
import time

import numpy as np
import pytest

from seismic_tomography_3d_b200 import workloads as wl

pytestmark = pytest.mark.gpu

REL_TOL = 1e-4
NSHOTS = int(os.environ.get("TOMO_REF_GPU_SHOTS", "4"))


def rel_err(T, Tref, h, vmax):
    m = Tref >= 2.0 * h / vmax
    return float(np.max(np.abs(T[m] - Tref[m]) / Tref[m]))


@pytest.mark.parametrize("case", ["config1", "config2"])
def test_block_fim_reference(tomo, oracle_mod, case):
    if not os.path.exists(os.path.join(os.path.dirname(oracle_mod.__file__), "_ref", "libref_fim.so")):
        pytest.skip("oracle/_ref/libref_fim.so not built (needs the reference sources)")
    sv = wl.config1(seed=1) if case == "config1" else wl.config2(seed=2)
    nshots = min(NSHOTS, len(sv.shots))
    shots = np.asarray(sv.shots[:nshots], np.float32)
    ny, nx, nz = sv.velocity.shape
    # the reference: one eikonal_equation() per shot (first call also warms its CUDA context)
    oracle_mod.ref_solve(oracle_mod.REF_BLOCK_FIM, sv.velocity, sv.h, shots[:1], want_T=False)
    T_ref, secs = oracle_mod.ref_solve(oracle_mod.REF_BLOCK_FIM, sv.velocity, sv.h, shots)

    with tomo.Context(nx, ny, nz, sv.h) as ctx:
        ctx.set_velocity(sv.velocity)
        ctx.eik_solve(shots, want_recv=False)              # warm-up
        reps, t0 = 5, time.perf_counter()
        for _ in range(reps):
            _, st = ctx.eik_solve(shots, want_recv=False)  # returns after the solve's stats read
        ours_batch = (time.perf_counter() - t0) / reps
        t0 = time.perf_counter()
        for i in range(nshots):
            ctx.eik_solve(shots[i:i + 1], want_recv=False)
        ours_single = (time.perf_counter() - t0) / nshots
        ctx.eik_solve(shots, want_recv=False)
        errs = [rel_err(ctx.eik_volume(i), T_ref[i], sv.h, float(sv.velocity.max())) for i in range(nshots)]

    rec = {
        "case": case, "grid": [nx, ny, nz], "h_m": sv.h, "shots": nshots, "windows": "full grid",
        "reference_block_fim_s_per_shot": [float(s) for s in secs],
        "reference_block_fim_s_per_shot_median": float(np.median(secs)),
        "ours_batch_s_per_shot": ours_batch / nshots,
        "ours_single_shot_s": ours_single,
        "ours_stats": st,
        "max_rel_err_vs_reference": errs,
    }
    print(json.dumps(rec))
    out = os.environ.get("TOMO_REF_GPU_JSON")
    if out:
        allrec = {}
        if os.path.exists(out):
            with open(out) as f:
                allrec = json.load(f)
        allrec[case] = rec
        with open(out, "w") as f:
            json.dump(allrec, f, indent=1)
    assert max(errs) < REL_TOL
    assert ours_single < float(np.median(secs))
