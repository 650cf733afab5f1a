"""Generates the golden fixtures of tests/golden/ by running the REFERENCE's own code.

The reference (phbastosa/seismic_tomography_3D) has no tests and ships no data, so its
known answers are produced here from its solvers, compiled unmodified from its sources into
oracle/_ref (oracle/Makefile) and driven through their public API:

  eik_ref.npz         Accurate_FSM (eikonal_type 2) and Classic / Podvin-Lecomte (type 0)
                      traveltime volumes on small seeded models (CPU)      [--cpu]
  block_fim_ref.npz   Block_FIM (eikonal_type 1, the reference CUDA kernel built for
                      sm_100a) on the same models -- needs a GPU           [--gpu]
  tomo_ref.npz        one iteration of the reference tomography.exe (FSM forward, ray
                      tracing, Tikhonov CGLS, model update) on a small case [--cpu]

Usage: python tests/golden/make_golden.py --cpu   (here)
       python tests/golden/make_golden.py --gpu   (on a machine with an sm_100 GPU)
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from seismic_tomography_3d_b200 import workloads as wl  # noqa: E402

# (seed, nx, ny, nz, h, shots (metres)) -- odd sizes exercise Block_FIM's padding.
EIK_CASES = [
    (101, 19, 17, 11, 25.0, [(100.0, 75.0, 0.0), (225.0, 300.0, 50.0)]),
    (102, 24, 24, 13, 20.0, [(0.0, 0.0, 0.0), (230.0, 170.0, 120.0)]),
    (103, 15, 22, 9, 30.0, [(211.0, 333.3, 17.5)]),
]


def eik_models():
    out = []
    for seed, nx, ny, nz, h, shots in EIK_CASES:
        sv = wl.small(seed, nx, ny, nz, h=h)
        out.append((seed, sv.velocity, h, np.asarray(shots, np.float32)))
    return out


def make_cpu():
    data = {}
    for seed, v, h, shots in eik_models():
        Tf, _ = oracle.ref_solve(oracle.REF_FSM, v, h, shots)
        Tc, _ = oracle.ref_solve(oracle.REF_CLASSIC, v, h, shots)
        data[f"v_{seed}"] = v
        data[f"h_{seed}"] = np.float32(h)
        data[f"shots_{seed}"] = shots
        data[f"fsm_{seed}"] = Tf
        data[f"pl_{seed}"] = Tc
    np.savez_compressed(os.path.join(HERE, "eik_ref.npz"), **data)
    make_tomo()


def make_gpu(out_dir=HERE):
    data = {}
    for seed, v, h, shots in eik_models():
        T, _ = oracle.ref_solve(oracle.REF_BLOCK_FIM, v, h, shots)
        data[f"fim_{seed}"] = T
    np.savez_compressed(os.path.join(out_dir, "block_fim_ref.npz"), **data)


# --------------------------------------------------------------------------------------
# One reference tomography iteration.  Inversion cells are multiples of the grid spacing
# so every reference ray reaches its source cell (it would loop forever otherwise).
# --------------------------------------------------------------------------------------
TOMO = dict(nx=41, ny=37, nz=21, h=25.0, d_tomo=100.0, shots=(2, 2), nodes=(6, 5), tk_order=2,
            tk_param=0.5, smooth=True, filter_samples=5, stdv=2.0)


def tomo_case():
    t = TOMO
    nx, ny, nz, h = t["nx"], t["ny"], t["nz"], t["h"]
    rng = np.random.default_rng(77)
    true_v = (wl.layered_model(rng, nx, ny, nz, h, speeds=(1500.0, 2200.0, 3000.0))
              * wl._anomalies(rng, nx, ny, nz, h, 2, sigma=3 * h)).astype(np.float32)
    start_v = wl.gradient_model(nx, ny, nz, h, 1500.0, 1.0)
    return true_v, start_v


def _regular(n_x, n_y, lo_x, hi_x, lo_y, hi_y, z):
    xs = np.linspace(lo_x, hi_x, n_x, dtype=np.float32) if n_x > 1 else np.array([lo_x], np.float32)
    ys = np.linspace(lo_y, hi_y, n_y, dtype=np.float32) if n_y > 1 else np.array([lo_y], np.float32)
    # reference order: x[k + j*n_yline] = x_tmp[j], y[...] = y_tmp[k] (regular.cpp:82-104)
    pts = np.zeros((n_x * n_y, 3), np.float32)
    for k in range(n_y):
        for j in range(n_x):
            pts[k + j * n_y] = (xs[j], ys[k], z)
    return pts


def tomo_geometry():
    t = TOMO
    nx, ny, h = t["nx"], t["ny"], t["h"]
    shots = _regular(*t["shots"], 5 * h, (nx - 6) * h, 5 * h, (ny - 6) * h, 0.0)
    nodes = _regular(*t["nodes"], 2 * h, (nx - 3) * h, 2 * h, (ny - 3) * h, 0.0)
    return shots, nodes


def make_tomo():
    t = TOMO
    nx, ny, nz, h = t["nx"], t["ny"], t["nz"], t["h"]
    true_v, start_v = tomo_case()
    shots, nodes = tomo_geometry()
    # observed picks: the reference FSM on the true model, sampled like write_first_arrival
    Tt, _ = oracle.ref_solve(oracle.REF_FSM, true_v, h, shots)
    dobs = np.stack([oracle.first_arrival(Tt[i], h, *nodes.T) for i in range(len(shots))])
    with tempfile.TemporaryDirectory() as d:
        run = os.path.join(d, "run")
        for sub in ("run", "picks", "fa", "conv", "models", "geom", "outputs/illumination"):
            os.makedirs(os.path.join(d, sub), exist_ok=True)
        start_v.tofile(os.path.join(d, "start.bin"))
        for i in range(len(shots)):
            dobs[i].astype(np.float32).tofile(os.path.join(d, "picks", f"obsData_{len(nodes)}_samples_shot_{i + 1}.bin"))
        sh, nd = t["shots"], t["nodes"]
        p = f"""x_samples = {nx}
y_samples = {ny}
z_samples = {nz}
x_spacing = {h}
y_spacing = {h}
z_spacing = {h}
vp_file = {d}/start.bin
reciprocity = False
shots_geometry_type = 0
nodes_geometry_type = 0
shots_elevation = 0
nodes_elevation = 0
shots_topography = False
nodes_topography = False
shots_topography_file = none
nodes_topography_file = none
shots_output_file = {d}/geom/shots.txt
nodes_output_file = {d}/geom/nodes.txt
shots_n_xline = {sh[0]}
shots_n_yline = {sh[1]}
shots_SW = {5 * h}, {5 * h}
shots_NW = {5 * h}, {(ny - 6) * h}
shots_SE = {(nx - 6) * h}, {5 * h}
nodes_n_xline = {nd[0]}
nodes_n_yline = {nd[1]}
nodes_SW = {2 * h}, {2 * h}
nodes_NW = {2 * h}, {(ny - 3) * h}
nodes_SE = {(nx - 3) * h}, {2 * h}
eikonal_type = 2
export_time_volume = False
export_first_arrival = True
time_volume_folder = {d}/fa/
first_arrival_folder = {d}/fa/
tomography_type = 0
max_iteration = 1
dx_tomo = {t['d_tomo']}
dy_tomo = {t['d_tomo']}
dz_tomo = {t['d_tomo']}
tk_order = {t['tk_order']}
tk_param = {t['tk_param']}
smooth = {t['smooth']}
filter_samples = {t['filter_samples']}
standard_deviation = {t['stdv']}
dobs_folder = {d}/picks/
convergency_folder = {d}/conv/
estimated_models_folder = {d}/models/
"""
        with open(os.path.join(d, "params.txt"), "w") as f:
            f.write(p)
        subprocess.run([oracle.ref_tomography_exe(), os.path.join(d, "params.txt")], cwd=run, check=True,
                       stdout=subprocess.DEVNULL, timeout=600)
        model = np.fromfile(os.path.join(d, "models", "fsm_model_iteration_1.bin"), np.float32).reshape(ny, nx, nz)
        conv = np.loadtxt(os.path.join(d, "conv", "fsm_convergency.txt"), dtype=np.float64)
        illum0 = np.fromfile(os.path.join(d, "outputs", "illumination", "fsm_illumination_iteration_0.bin"),
                             np.float32).reshape(ny, nx, nz)
        gshots = np.loadtxt(os.path.join(d, "geom", "shots.txt"), delimiter=",", dtype=np.float32)
        gnodes = np.loadtxt(os.path.join(d, "geom", "nodes.txt"), delimiter=",", dtype=np.float32)
    np.savez_compressed(os.path.join(HERE, "tomo_ref.npz"), true_v=true_v, start_v=start_v, shots=shots,
                        nodes=nodes, dobs=dobs.astype(np.float32), model_iter1=model, convergency=conv,
                        illumination_iter0=illum0, geom_shots=gshots.reshape(-1, 3),
                        geom_nodes=gnodes.reshape(-1, 3))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--cpu", action="store_true")
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--out", default=HERE, help="output folder of the GPU fixtures")
    a = ap.parse_args()
    if a.cpu:
        make_cpu()
    if a.gpu:
        make_gpu(a.out)
