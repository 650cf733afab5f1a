"""The drop-in executables run the reference's parameter files and file layouts end to
end (eikonal_type = 3), and produce the same numbers as the library API."""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden as mg  # noqa: E402

pytestmark = pytest.mark.gpu


def write_params(d, t, extra=""):
    nx, ny, nz, h = t["nx"], t["ny"], t["nz"], t["h"]
    sh, nd = t["shots"], t["nodes"]
    # quoted paths followed by spaces, as in the reference's own parameter files
    text = f"""#--- model
x_samples = {nx}
y_samples = {ny}
z_samples = {nz}
x_spacing = {h}          # in meters [m]
y_spacing = {h}
z_spacing = {h}
vp_file = "{d}/start.bin"   # velocity model
reciprocity = False
shots_geometry_type = 0
nodes_geometry_type = 0
shots_elevation = 0
nodes_elevation = 0
shots_topography = False
nodes_topography = False
shots_topography_file = none
nodes_topography_file = none
shots_output_file = "{d}/xyz_shots.txt"   #
nodes_output_file = "{d}/xyz_nodes.txt"   #
shots_n_xline = {sh[0]}
shots_n_yline = {sh[1]}
shots_SW = [{5 * h}, {5 * h}]
shots_NW = [{5 * h}, {(ny - 6) * h}]
shots_SE = [{(nx - 6) * h}, {5 * h}]
nodes_n_xline = {nd[0]}
nodes_n_yline = {nd[1]}
nodes_SW = [{2 * h}, {2 * h}]
nodes_NW = [{2 * h}, {(ny - 3) * h}]
nodes_SE = [{(nx - 3) * h}, {2 * h}]
eikonal_type = 3    # B200
export_time_volume = True
export_first_arrival = True
time_volume_folder = "{d}/tt/"   #
first_arrival_folder = "{d}/fa/"   #
max_iteration = 1
dx_tomo = {t['d_tomo']}
dy_tomo = {t['d_tomo']}
dz_tomo = {t['d_tomo']}
tk_order = {t['tk_order']}
tk_param = {t['tk_param']}
smooth = True
filter_samples = 5
standard_deviation = 2.0
dobs_folder = "{d}/picks/"   #
convergency_folder = "{d}/conv/"   #
estimated_models_folder = "{d}/models/"   #
{extra}"""
    p = os.path.join(d, "parameters.txt")
    with open(p, "w") as f:
        f.write(text)
    return p


def test_eikonal_and_tomography_executables(tomo, tmp_path):
    g = np.load(os.path.join(HERE, "golden", "tomo_ref.npz"))
    t = mg.TOMO
    d = str(tmp_path)
    for sub in ("tt", "fa", "picks", "conv", "models", "run", "outputs/illumination"):
        os.makedirs(os.path.join(d, sub), exist_ok=True)
    g["start_v"].tofile(os.path.join(d, "start.bin"))
    shots, nodes = g["shots"], g["nodes"]
    with tomo.Context(t["nx"], t["ny"], t["nz"], t["h"]) as ctx:
        ctx.set_velocity(g["true_v"])
        dobs, _ = ctx.eik_solve(shots, receivers=nodes)
    for i in range(len(shots)):
        dobs[i].tofile(os.path.join(d, "picks", f"obsData_{len(nodes)}_samples_shot_{i + 1}.bin"))
    params = write_params(d, t)
    exe_dir = os.path.dirname(tomo.LIB_PATH)

    r = subprocess.run([os.path.join(exe_dir, "eikonal_b200"), params], cwd=os.path.join(d, "run"),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    # API results on the same inputs
    with tomo.Context(t["nx"], t["ny"], t["nz"], t["h"]) as ctx:
        ctx.set_velocity(g["start_v"])
        dcal, _ = ctx.eik_solve(shots, receivers=nodes)
        vols = [ctx.eik_volume(i) for i in range(len(shots))]
        ctx.set_observed(dobs)
        ctx.build_jacobian((t["d_tomo"],) * 3, t["tk_order"], t["tk_param"])
        ctx.cgls(10, want_x=False)
        vel = ctx.model_update()
    nz, nx, ny = t["nz"], t["nx"], t["ny"]
    # The default (asynchronous) schedule relaxes bricks in a run-dependent order; with the
    # 1e-6 s face tolerance two runs agree to ~1e-6 relative, not bit for bit.
    for i in range(len(shots)):
        tt = np.fromfile(os.path.join(d, "tt", f"fim_eikonal_nz{nz}_nx{nx}_ny{ny}_shot_{i + 1}.bin"), np.float32)
        np.testing.assert_allclose(tt.reshape(ny, nx, nz), vols[i], rtol=1e-5, atol=1e-7)
        fa = np.fromfile(os.path.join(d, "fa", f"fim_times_nr{len(nodes)}_shot_{i + 1}.bin"), np.float32)
        np.testing.assert_allclose(fa, dcal[i], rtol=1e-5, atol=1e-7)
    xyz = np.loadtxt(os.path.join(d, "xyz_shots.txt"), delimiter=",", dtype=np.float32).reshape(-1, 3)
    np.testing.assert_array_equal(xyz, shots)

    r = subprocess.run([os.path.join(exe_dir, "tomography_b200"), params], cwd=os.path.join(d, "run"),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    model = np.fromfile(os.path.join(d, "models", "fim_model_iteration_1.bin"), np.float32).reshape(ny, nx, nz)
    np.testing.assert_allclose(model, vel, rtol=1e-4)
    conv = np.loadtxt(os.path.join(d, "conv", "fim_convergency.txt"))
    # the reference's hard-coded interior masks confine the update to a small region of
    # this model, so the residual barely moves (as in the reference's own run)
    assert conv.shape == (2,) and np.all(np.isfinite(conv)) and conv[1] <= conv[0] * 1.05
    il = np.fromfile(os.path.join(d, "outputs", "illumination", "fim_illumination_iteration_0.bin"), np.float32)
    assert il.size == nx * ny * nz and il.sum() > 0


def test_tomography_executable_matches_reference_run(tomo, tmp_path):
    """tomography_b200 with eikonal_operator = fsm (Accurate_FSM's operator, bit for bit on
    the device) on the inputs of the golden reference run (tomo_ref.npz: the reference's own
    tomography.exe, eikonal_type 2, one iteration; the picks are the reference FSM's): the
    recovered model against the reference's fsm_model_iteration_1.bin within the 0.5 % RMS
    bound (the CGLS here reduces in FP64 where the reference accumulates in FP32), and the
    convergence file against the reference's."""
    g = np.load(os.path.join(HERE, "golden", "tomo_ref.npz"))
    t = mg.TOMO
    d = str(tmp_path)
    for sub in ("tt", "fa", "picks", "conv", "models", "run", "outputs/illumination"):
        os.makedirs(os.path.join(d, sub), exist_ok=True)
    g["start_v"].tofile(os.path.join(d, "start.bin"))
    nodes = g["nodes"]
    for i in range(len(g["shots"])):
        g["dobs"][i].astype(np.float32).tofile(os.path.join(d, "picks", f"obsData_{len(nodes)}_samples_shot_{i + 1}.bin"))
    params = write_params(d, t, extra="eikonal_operator = fsm\n")
    exe = os.path.join(os.path.dirname(tomo.LIB_PATH), "tomography_b200")
    r = subprocess.run([exe, params], cwd=os.path.join(d, "run"), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    nz, nx, ny = t["nz"], t["nx"], t["ny"]
    model = np.fromfile(os.path.join(d, "models", "fsm_model_iteration_1.bin"), np.float32).reshape(ny, nx, nz)
    ref = g["model_iter1"].astype(np.float64)
    rms = float(np.sqrt(np.mean(((model - ref) / ref) ** 2)))
    upd = float(np.linalg.norm(model - ref) / np.linalg.norm(ref - g["start_v"]))
    print(f"\ndrop-in vs reference tomography.exe: model RMS rel {rms:.2e}, update rel L2 {upd:.2e}")
    assert rms <= 5e-3
    conv = np.loadtxt(os.path.join(d, "conv", "fsm_convergency.txt"))
    np.testing.assert_allclose(conv, g["convergency"], rtol=1e-4)


def test_wrong_eikonal_type_is_an_error(tomo, tmp_path):
    t = mg.TOMO
    p = write_params(str(tmp_path), t).replace("", "")
    text = open(p).read().replace("eikonal_type = 3", "eikonal_type = 1")
    open(p, "w").write(text)
    exe = os.path.join(os.path.dirname(tomo.LIB_PATH), "tomography_b200")
    r = subprocess.run([exe, p], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "eikonal_type = 3" in r.stderr
