"""Benchmark: shot solves/s of the batched eikonal solve on 201x201x101 nodes.

Workload (one step): the config-2 batch -- 64 shots on a jittered 8x8 surface grid over a
201x201x101 model at 12.5 m (three dipping layers + eight +-10 % anomalies), each on a
brick-aligned window covering 60-100 % of the lateral extent, all solved by one persistent
launch; 2,500 surface receivers (50x50) sampled per shot.  Synthetic seeded data.

  value  shots/s with the model resident in HBM (CUDA events on the library's stream)
  e2e    shots/s through the C ABI with host buffers: pinned velocity upload (16.3 MB) +
         solve + receiver-times download every step
  roofline  dominant kernel (k_fim_solve): algorithmic bytes = brick activations x 64
         nodes x 12 B (slowness + traveltime in + traveltime out) / its event time
  cpu_baseline  the reference's own Accurate_FSM (compiled unmodified into oracle/_ref)
         on a bounded sample of the same shots and windows, all host threads
  accuracy  the timed setting's fields of 8 shots against the FP64 oracle (CPU leg)

On one GPU the line also carries the other configurations, each bounded to seconds:
  config1       the single 101x101x51 shot on the device (JW, NGB) and the reference's own
                FSM and Podvin-Lecomte on 1 core and on all cores
  tomography    config 3: one whole iteration (stage split, CGLS roofline) and the
                reference's own tomography.exe on a 4-shot sample
  learned_warm  config 4: the surrogate trained in-run, its prediction seeding the solve of
                the config-2 batch, against the plain solve
  inversion     config 5: 3 graph-replayed iterations of the 401x401x201 inversion

``--impl reference`` times the reference's CPU eikonal path (Accurate_FSM) the same way.
Multi-GPU (torchrun): shots are independent, each rank solves its own 64-shot batch (weak
scaling, no data-path collective); time = max over ranks.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "shot solves/s on 201x201x101, learned-warm vs plain FIM, at 1e-4 rel err"
UNIT = "shots/s"
BYTES_PER_NODE_ACT = 12  # slowness read + traveltime read + traveltime write (float32)
# DRAM bytes (read + write) per brick activation of the headline solve, from one ncu capture
# of a 16-shot launch of this workload each (dram__bytes_read.sum + dram__bytes_write.sum
# over the launch's activations; profiles/k_fim_solve_config2.md, k_fim_solve8_config2.md,
# k_fim_pair_config2.md):
# roofline.traffic is this figure times the timed launch's own activation count.
DRAM_BYTES_PER_ACTIVATION = {"k_fim_solve": 351.6, "k_fim_solve8": 2787.5, "k_fim_pair": 353.5}
# Solver tolerances of the timed runs (seismic_tomography_3d_b200.workloads): the metric is
# quoted at 1e-4 relative traveltime error, so the face-change and in-brick tolerances are
# loosened until the error against the FP64 oracle (checked in the cpu_baseline leg,
# reported as "accuracy") sits well inside that budget.  Full-grid solves on the smooth
# starting models of configs 3 and 5 add the time-band ordering (0.2 s: 1.18x / 2.3x faster
# solves); on the windowed, layered config-2 batch it costs time and stays off.
from seismic_tomography_3d_b200.workloads import TIMED_TOLERANCES as SOLVER  # noqa: E402
from seismic_tomography_3d_b200.workloads import TIMED_TOLERANCES_BANDED as SOLVER_BANDED  # noqa: E402


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def max_over_ranks(value, dist, device):
    """The largest of every rank's value (the job's time is its slowest rank's); value
    itself without a process group."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event reasons sampled during the timed region (read only).

    Reads NVML directly every 10 ms (the GPU is found by its PCI bus id, so the index
    stays right under CUDA_VISIBLE_DEVICES); falls back to polling nvidia-smi."""

    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []  # (sm_mhz, sm_max_mhz, set of reason names)
        self.stop = threading.Event()
        self.nvml = None
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(device)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            self.handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            self.nvml = pynvml
        except Exception:
            self.nvml = None
        self.th = threading.Thread(target=self._run_nvml if self.nvml else self._run_smi, daemon=True)

    def _run_nvml(self):
        n = self.nvml
        bits = {"hw_slowdown": n.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": n.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": n.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": n.nvmlClocksEventReasonSwPowerCap}
        while not self.stop.is_set():
            try:
                sm = n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM)
                mx = n.nvmlDeviceGetMaxClockInfo(self.handle, n.NVML_CLOCK_SM)
                r = n.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                self.samples.append((float(sm), float(mx), {k for k, v in bits.items() if r & v}))
            except Exception:
                pass
            self.stop.wait(0.01)

    def _run_smi(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                c = [x.strip() for x in out.split(",")]
                if len(c) >= 9 and c[1].replace(".", "").isdigit():
                    self.samples.append((float(c[1]), float(c[2]),
                                         {self.REASONS[i] for i in range(4) if c[5 + i].lower() == "active"}))
            except Exception:
                pass
            self.stop.wait(0.05)

    def __enter__(self):
        self.th.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.th.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(s[0] for s in self.samples),
                "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": sorted(set().union(*(s[2] for s in self.samples))),
                "samples": len(self.samples), "source": "nvml" if self.nvml else "nvidia-smi"}


def workload(rank, shots=None):
    import dataclasses

    from seismic_tomography_3d_b200 import workloads as wl

    sv = wl.config2(seed=2 + 1000 * rank)
    if shots:  # a smaller batch of the same workload (profiling captures)
        sv = dataclasses.replace(sv, shots=sv.shots[:shots], windows=sv.windows[:shots])
    return sv


def cpu_reference_sample(sv, max_shots=None, budget_s=20.0):
    """The reference Accurate_FSM (oracle/_ref) on the host cores over the batch's own
    shots and windows.  Returns (shots/s, threads, sample description)."""
    import oracle

    nthreads = os.cpu_count() or 1
    nshots = len(sv.shots) if max_shots is None else min(max_shots, len(sv.shots))
    # windows differ per shot: group shots by window so each group is one cropped model
    t_start = time.perf_counter()
    done = 0
    solve_s = 0.0
    groups = {}
    for i in range(nshots):
        key = tuple(int(v) for v in sv.windows[i]) if sv.windows is not None else (0, sv.nx, 0, sv.ny)
        groups.setdefault(key, []).append(i)
    # one shot per window here: run windows in parallel by packing them into threads
    import concurrent.futures as cf

    def run_one(key_idx):
        (x0, x1, y0, y1), idx = key_idx
        vel = np.ascontiguousarray(sv.velocity[y0:y1, x0:x1, :])
        shots = sv.shots[idx].copy()
        shots[:, 0] -= np.float32(x0) * np.float32(sv.h)
        shots[:, 1] -= np.float32(y0) * np.float32(sv.h)
        _, secs = oracle.ref_solve(oracle.REF_FSM, vel, sv.h, shots, nthreads=1, want_T=False)
        return len(idx), float(np.sum(secs))

    items = list(groups.items())
    with oracle.quiet_stdout():
        with cf.ThreadPoolExecutor(max_workers=nthreads) as ex:
            futs = []
            for it in items:
                futs.append(ex.submit(run_one, it))
            for f in futs:
                n, s = f.result()
                done += n
                solve_s += s
                if time.perf_counter() - t_start > budget_s:
                    break
            for f in futs:
                f.cancel()
    wall = time.perf_counter() - t_start
    desc = (f"reference Accurate_FSM (NGB 2014 FSM, oracle/_ref, g++ -O3) on {done} of the batch's shots "
            f"(own windows), {nthreads} host threads, {wall:.1f} s wall")
    return done / wall, nthreads, desc


def sample_shots(sv, k=8):
    """k shots of the batch: the smallest and the largest window and k - 2 in between."""
    areas = np.array([(w[1] - w[0]) * (w[3] - w[2]) for w in sv.windows])
    order = np.argsort(areas, kind="stable")
    return sorted(set(int(order[i]) for i in np.linspace(0, len(order) - 1, k).round().astype(int)))


def oracle_accuracy(sv, idx, vols):
    """Max relative error of the timed setting's fields (vols, shots idx) against the FP64
    fixed point of the same operator on each cropped window (the oracle), on nodes with
    T >= 2h/v_max; host threads."""
    import concurrent.futures as cf

    import oracle

    vmax = float(sv.velocity.max())

    def one(k):
        i = idx[k]
        x0, x1, y0, y1 = (int(a) for a in sv.windows[i])
        slow = np.ascontiguousarray((np.float32(1.0) / sv.velocity[y0:y1, x0:x1, :]).astype(np.float32))
        src = (float(np.float32(sv.shots[i][0]) - np.float32(x0) * np.float32(sv.h)),
               float(np.float32(sv.shots[i][1]) - np.float32(y0) * np.float32(sv.h)), float(sv.shots[i][2]))
        Tref, _ = oracle.fim_jw(slow, sv.h, src)
        m = Tref >= 2.0 * sv.h / vmax
        return float(np.max(np.abs(vols[k][m] - Tref[m]) / Tref[m])), int(m.sum())

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(min(len(idx), os.cpu_count() or 1)) as ex:
        res = list(ex.map(one, range(len(idx))))
    return {"max_rel_err_vs_fp64_oracle": max(r[0] for r in res), "per_shot": [r[0] for r in res],
            "shots_checked": [int(i) for i in idx], "nodes_checked": sum(r[1] for r in res), "budget": 1e-4,
            "oracle": "FP64 fixed point of the Block_FIM operator on each shot's cropped window (oracle/tomo_oracle.c)",
            "oracle_s": time.perf_counter() - t0}


def config1_cpu():
    """Config 1 on the host cores: the reference's own Accurate_FSM (NGB operator) and
    Classic (Podvin-Lecomte), compiled unmodified into oracle/_ref, on 1 core (the config-1
    shot) and on every core (one seeded surface shot per thread, solved in parallel)."""
    import oracle

    from seismic_tomography_3d_b200 import workloads as wl

    sv = wl.config1()
    n = os.cpu_count() or 1
    rng = np.random.default_rng(11)
    many = wl.surface_nodes(rng, sv.nx, sv.ny, sv.h, n)
    out = {"workload": "config1: 101x101x51 @25 m, v(z) = 1500 + 0.6 z + two 10 % anomalies, surface shots",
           "kind": "reference", "cores_all": n}
    for name, kind, reps in (("fsm", oracle.REF_FSM, 3), ("podvin_lecomte", oracle.REF_CLASSIC, 1)):
        one = []
        for _ in range(reps):
            _, secs = oracle.ref_solve(kind, sv.velocity, sv.h, sv.shots, nthreads=1, want_T=False)
            one.append(float(secs[0]))
        t0 = time.perf_counter()
        oracle.ref_solve(kind, sv.velocity, sv.h, many, nthreads=n, want_T=False)
        wall = time.perf_counter() - t0
        out[name] = {"s_per_shot_1core": statistics.median(one), "shots_per_s_1core": 1.0 / statistics.median(one),
                     "shots_per_s_all_cores": n / wall, "all_cores_wall_s": wall}
    return out


def config1_gpu(steps=10, warmup=3):
    """Config 1 on the device: the single shot with its 200 receivers, JW (Block_FIM's
    operator) and NGB (Accurate_FSM's, bit for bit); device time per solve and the same
    call end to end with the host velocity upload and receiver download."""
    import torch

    import seismic_tomography_3d_b200 as tomo
    from seismic_tomography_3d_b200 import workloads as wl

    sv = wl.config1()
    ctx = tomo.Context(sv.nx, sv.ny, sv.nz, sv.h)
    stream = torch.cuda.ExternalStream(ctx.stream)
    vel_pinned = torch.from_numpy(sv.velocity.copy()).pin_memory()
    ctx.set_velocity(sv.velocity)
    out = {"workload": "config1: 101x101x51 @25 m, 1 shot x 200 receivers (library default tolerances)"}
    for name, op in (("jw", 0), ("ngb", 1)):
        for _ in range(warmup):
            ctx.eik_solve(sv.shots, receivers=sv.receivers, op=op)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            ctx.eik_solve(sv.shots, receivers=sv.receivers, want_recv=False, op=op)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        e0.record(stream)
        for _ in range(steps):
            assert ctx.lib.tomo_set_velocity(ctx.h, vel_pinned.data_ptr()) == 0
            ctx.eik_solve(sv.shots, receivers=sv.receivers, op=op)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1) / steps
        out[name] = {"ms_per_shot": ms, "shots_per_s": 1000.0 / ms, "e2e_ms_per_shot": e2e_ms}
    ctx.close()
    return out


def _regular_points(n_x, n_y, x0, x1, y0, y1, z):
    """Points of the reference's Regular geometry in its order (regular.cpp:82-104):
    point k + j * n_y is (x_j, y_k)."""
    xs = np.linspace(x0, x1, n_x, dtype=np.float32) if n_x > 1 else np.array([x0], np.float32)
    ys = np.linspace(y0, y1, n_y, dtype=np.float32) if n_y > 1 else np.array([y0], np.float32)
    pts = np.zeros((n_x * n_y, 3), np.float32)
    for k in range(n_y):
        for j in range(n_x):
            pts[k + j * n_y] = (xs[j], ys[k], z)
    return pts


def reference_tomography_exe(timeout_s=240):
    """The reference's own tomography.exe (Least_squares with the FSM forward model, serial),
    compiled unmodified into oracle/_ref, on a bounded sample of config 3: the config-3 true
    and starting models (201x201x101 at 12.5 m), 4 shots (2x2) x 2,500 receivers (the
    config-3 50x50 grid), 50 m cells, lambda 0.1, order 2, smoothing; picks from the
    reference FSM on the true model.  50 m cells (4 h) rather than config 3's 51 m: the
    reference ray tracer loops forever when a cell face splits the source node's box,
    which 51 m cells do.  One iteration = wall time with max_iteration = 1 minus the time
    with max_iteration = 0 (the loop of tomography_main.cpp:19-30 forward-models once more
    before it stops)."""
    import tempfile

    import oracle

    from seismic_tomography_3d_b200 import workloads as wl

    exe = oracle.ref_tomography_exe()
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/tomography.exe not built"}
    sv, start, inv = wl.config3()
    h, nx, ny, nz = sv.h, sv.nx, sv.ny, sv.nz
    lo, hi = 41 * h, 161 * h  # source nodes off the 50 m cell faces
    shots = _regular_points(2, 2, lo, hi, lo, hi, 0.0)
    nodes = _regular_points(50, 50, 25.0, 2475.0, 25.0, 2475.0, 0.0)
    Tt, _ = oracle.ref_solve(oracle.REF_FSM, sv.velocity, h, shots, nthreads=4)
    dobs = np.stack([oracle.first_arrival(Tt[i], h, *nodes.T) for i in range(len(shots))])
    del Tt
    times = {}
    with tempfile.TemporaryDirectory() as d:
        for sub in ("run", "picks", "fa", "conv", "models", "geom", "outputs/illumination"):
            os.makedirs(os.path.join(d, sub), exist_ok=True)
        np.ascontiguousarray(start).tofile(os.path.join(d, "start.bin"))
        for i in range(len(shots)):
            dobs[i].astype(np.float32).tofile(os.path.join(d, "picks", f"obsData_{len(nodes)}_samples_shot_{i + 1}.bin"))
        for max_it in (0, 1):
            par = f"""x_samples = {nx}
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
shots_n_xline = 2
shots_n_yline = 2
shots_SW = {lo}, {lo}
shots_NW = {lo}, {hi}
shots_SE = {hi}, {lo}
nodes_n_xline = 50
nodes_n_yline = 50
nodes_SW = 25.0, 25.0
nodes_NW = 25.0, 2475.0
nodes_SE = 2475.0, 25.0
eikonal_type = 2
export_time_volume = False
export_first_arrival = True
time_volume_folder = {d}/fa/
first_arrival_folder = {d}/fa/
tomography_type = 0
max_iteration = {max_it}
dx_tomo = 50.0
dy_tomo = 50.0
dz_tomo = 50.0
tk_order = {inv['tk_order']}
tk_param = {inv['tk_param']}
smooth = True
filter_samples = {inv['filter_samples']}
standard_deviation = {inv['standard_deviation']}
dobs_folder = {d}/picks/
convergency_folder = {d}/conv/
estimated_models_folder = {d}/models/
"""
            pf = os.path.join(d, f"params{max_it}.txt")
            with open(pf, "w") as f:
                f.write(par)
            t0 = time.perf_counter()
            try:
                subprocess.run([exe, pf], cwd=os.path.join(d, "run"), check=True, stdout=subprocess.DEVNULL,
                               timeout=timeout_s)
            except (subprocess.TimeoutExpired, subprocess.CalledProcessError) as e:
                return {"unavailable": f"reference tomography.exe did not finish: {type(e).__name__}"}
            times[max_it] = time.perf_counter() - t0
    it_s = times[1] - times[0]
    return {"kind": "reference", "cores": 1, "iteration_s": it_s, "run_s_max_iteration_0": times[0],
            "run_s_max_iteration_1": times[1], "shots": len(shots), "receivers": len(nodes),
            "sample": "config-3 models, 4 shots (2x2) x 2,500 receivers, 50 m cells, 10 CGLS iterations "
                      "(the reference's count), FSM forward model, serial"}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return 0
    sv = workload(0)
    per_step = []
    desc = ""
    threads = os.cpu_count() or 1
    sample = min(len(sv.shots), max(8, 2 * threads))
    for i in range(args.warmup + args.steps):
        rate, threads, desc = cpu_reference_sample(sv, max_shots=sample, budget_s=60.0)
        if i >= args.warmup:
            per_step.append(rate)
    value = float(statistics.median(per_step))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sample / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded config-2 model, shots, windows)",
            "config": {"workload": "config2: 64 shots, 201x201x101 @12.5 m, windows 60-100 %",
                       "sample_shots_per_step": sample},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    SOLVER_RUN = dict(SOLVER)  # the headline's options: timed tolerances (+ --brick)

    import seismic_tomography_3d_b200 as tomo

    rank, world, local = rank_info()
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local)
    sv = workload(rank, args.shots)
    ns = len(sv.shots)
    ctx = tomo.Context(sv.nx, sv.ny, sv.nz, sv.h, device=local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    vel_pinned = torch.from_numpy(sv.velocity.copy()).pin_memory()
    ctx.set_velocity(sv.velocity)
    # launch shape and brick shape tuned on this batch (setup, untimed); later solves use them
    tuned = None
    if args.brick:  # a fixed brick shape (profiling), default launch shape
        SOLVER_RUN.update(brick=args.brick)
    elif args.schedule == 3:  # two bricks per warp, its best config-2 shape (profiling)
        SOLVER_RUN.update(schedule=3, block_warps=8, occupancy=3)
    elif not args.no_autotune:
        shape, tst = ctx.eik_autotune(sv.shots, windows=sv.windows, repeats=2)
        tuned = dict(shape, trials=tst["trials"], best_ms=tst["best_ms"], default_ms=tst["default_ms"])

    def step_resident():
        _, st = ctx.eik_solve(sv.shots, windows=sv.windows, receivers=sv.receivers, want_recv=False, **SOLVER_RUN)
        return st

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        step_resident()
    # ---- value: model resident ---------------------------------------------------------
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            stats.append(step_resident())
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    ms_max = ms
    ms_max = max_over_ranks(ms, dist, 'cuda')
    value = world * ns / (ms_max / 1000.0)

    # ---- e2e: host buffers through the C ABI ---------------------------------------------
    nrec = len(sv.receivers)
    t_pinned = torch.empty((ns, nrec), dtype=torch.float32).pin_memory()
    t_out = t_pinned.numpy()  # receiver times land in page-locked host memory
    lib = ctx.lib
    # Every step uploads its velocity model from pinned host memory and reads its receiver
    # times back.  The upload of step k + 1 is staged (tomo_stage_velocity) before step k's
    # solve, so the copy runs during that solve; step 0's upload is not overlapped.
    # The end-to-end loops run more steps than the resident one (host-side jitter of the
    # calling process shows up in them), with Python's garbage collector paused.
    e2e_steps = max(3 * args.steps, 30)
    gc.disable()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.stage_velocity(vel_pinned)
    for k in range(e2e_steps):
        ctx.commit_velocity()
        if k + 1 < e2e_steps:
            ctx.stage_velocity(vel_pinned)
        ctx.eik_solve(sv.shots, windows=sv.windows, receivers=sv.receivers, want_recv=True, out=t_out, **SOLVER_RUN)
    e1.record(stream)
    barrier()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, dist, 'cuda')
    e2e_value = world * ns / (e2e_ms / 1000.0)
    # the same steps with the blocking upload (tomo_set_velocity) before each solve
    barrier()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(e2e_steps):
        tomo_rc = lib.tomo_set_velocity(ctx.h, vel_pinned.data_ptr())
        assert tomo_rc == 0
        ctx.eik_solve(sv.shots, windows=sv.windows, receivers=sv.receivers, want_recv=True, out=t_out, **SOLVER_RUN)
    s1.record(stream)
    barrier()
    gc.enable()
    serial_ms = max_over_ranks(s0.elapsed_time(s1) / e2e_steps, dist, 'cuda')
    # fields of the timed setting (the last e2e solve) for the oracle check of the CPU leg
    cpu_leg = rank == 0 and world == 1 and not args.no_cpu_baseline
    acc_idx = sample_shots(sv) if cpu_leg else []
    acc_vols = [ctx.eik_volume(i) for i in acc_idx]

    # ---- roofline of the dominant kernel -----------------------------------------------
    act = statistics.mean(s["activations"] for s in stats)
    kern_ms = statistics.mean(s["solve_ms"] for s in stats)
    alg_bytes = act * stats[0]["nodes_per_brick"] * BYTES_PER_NODE_ACT
    peak, peak_kind = peaks()
    achieved = alg_bytes / (kern_ms / 1000.0) / 1e9
    # compulsory traffic of the batch whatever the algorithm: slowness read + traveltime
    # written once per window node (8 B/node)
    compulsory = 8.0 * sum(ctx.volume_sizes(ns, sv.windows))
    # DRAM bytes per brick activation from the committed ncu summary of the kernel that ran
    # (one capture of a 16-shot launch of the same workload), scaled to this launch's
    # activations
    kernel = "k_fim_solve8" if stats[0]["nodes_per_brick"] == 512 else \
        "k_fim_pair" if (tuned and tuned.get("schedule") == 3) or args.schedule == 3 else "k_fim_solve"
    per_act = DRAM_BYTES_PER_ACTIVATION.get(kernel)
    traffic = per_act * act if per_act else None

    # ---- the timed setting against the fully converged field of the same solver ---------
    accuracy_conv = solver_accuracy(ctx, sv, SOLVER_RUN)

    # ---- the NGB operator: the reference's own Accurate_FSM sweeps, bit-exact ------------
    ngb_steps = max(1, min(args.steps, 5))
    ctx.eik_solve(sv.shots, windows=sv.windows, receivers=sv.receivers, want_recv=False, op=1)
    barrier()
    n0, n1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0.record(stream)
    for _ in range(ngb_steps):
        ctx.eik_solve(sv.shots, windows=sv.windows, receivers=sv.receivers, want_recv=False, op=1)
    n1.record(stream)
    barrier()
    ngb_ms = n0.elapsed_time(n1) / ngb_steps
    ngb_ms = max_over_ranks(ngb_ms, dist, 'cuda')

    warm = warm_start_bound(ctx, sv, stream, ngb_steps, barrier, dist, world)
    unaligned = unaligned_windows_object(ctx, sv, SOLVER_RUN, stream, ngb_steps, barrier, dist, world, rank)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded config-2 model, shots, windows, receivers)",
            "config": {"workload": "config2: 64 shots/GPU, 201x201x101 @12.5 m, brick-aligned windows "
                                   "60-100 % lateral, 2500 receivers, plain FIM (JW operator)",
                       "tolerances_s": SOLVER, "autotuned_shape": tuned,
                       "shots_per_gpu": ns, "grid": [sv.nx, sv.ny, sv.nz], "h_m": sv.h,
                       "l2": "traveltime pool 1.1 GB > 126 MB L2 (inputs larger than L2)",
                       "parallelism": f"shot-sharded x{world}"},
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": int(sv.velocity.nbytes),
                    "d2h_bytes_per_step": int(t_out.nbytes) if t_out is not None else 0,
                    "steps": e2e_steps,
                    "upload": "pinned host velocity per step, staged during the previous step's solve; "
                              "receiver times into pinned host memory",
                    "serial_upload": {"value": world * ns / (serial_ms / 1000.0), "unit": UNIT,
                                      "ms_per_step": serial_ms}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": kernel, "kernel_ms": kern_ms,
                         "alg_bytes_per_launch": alg_bytes, "activations_per_launch": act,
                         "compulsory_bytes_per_launch": compulsory,
                         "compulsory_frac": compulsory / (kern_ms / 1000.0) / 1e9 / peak},
            "clocks": clk.summary(),
            "gpu_launches": 3 * args.steps,
            "solver": {"rounds": stats[-1]["rounds"], "activations": stats[-1]["activations"],
                       "inner_iterations": stats[-1]["inner_iterations"], **SOLVER},
            "accuracy_vs_converged": accuracy_conv,
            "ngb_fsm": {"value": world * ns / (ngb_ms / 1000.0), "unit": UNIT, "ms_per_step": ngb_ms,
                        "steps": ngb_steps,
                        "what": "TOMO_OP_NGB: the reference Accurate_FSM's 8+8 sweeps on the same batch, "
                                "bit-exact with the reference CPU solver (the cpu_baseline's algorithm)"},
            "warm_start": warm, "unaligned_windows": unaligned}
    ctx.close()
    del stream
    torch.cuda.empty_cache()
    # ---- the other configurations (one GPU only; each bounded to seconds) ----------------
    if world == 1 and not args.headline_only:
        line["config1"] = {"gpu": config1_gpu()}
        line["tomography"] = tomography_object(args, steps=5, warmup=3)
        line["learned_warm"] = learned_warm_object(args.warm_fields, args.warm_epochs)
        if not args.no_inversion:
            line["inversion"] = inversion_object(args, iterations=3)
    # ---- CPU leg: the reference on the host cores, and the oracle as the checker ----------
    if cpu_leg:
        rate, cores, desc = cpu_reference_sample(sv, max_shots=min(ns, max(8, 2 * (os.cpu_count() or 1))),
                                                 budget_s=25.0)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc}
        line["accuracy"] = oracle_accuracy(sv, acc_idx, acc_vols)
        if not args.headline_only:
            line["config1"]["cpu"] = config1_cpu()
            line["tomography"]["reference_tomography_exe"] = reference_tomography_exe()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def unaligned_windows_object(ctx, sv, solver, stream, steps, barrier, dist, world, rank):
    """The same shots on the seeded crops themselves (any origin, not rounded out to bricks):
    those windows read their slowness node by node from the shared model."""
    import torch

    from seismic_tomography_3d_b200 import workloads as wl

    win = wl.config2(seed=2 + 1000 * rank, aligned=False).windows[: len(sv.shots)]
    off_grid = int(np.any(win % 4 != 0, axis=1).sum())
    out = {"windows": f"seeded 60-100 % crops at any origin ({off_grid} of {len(win)} windows off the brick grid)"}
    for name, kw in (("jw", solver), ("ngb", {"op": 1})):
        ctx.eik_solve(sv.shots, windows=win, receivers=sv.receivers, want_recv=False, **kw)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            ctx.eik_solve(sv.shots, windows=win, receivers=sv.receivers, want_recv=False, **kw)
        e1.record(stream)
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps, dist, 'cuda')
        out[name] = {"value": world * len(sv.shots) / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms,
                     "steps": steps}
    return out


def solver_accuracy(ctx, sv, solver):
    """Max relative error of the timed setting (solver options) against the fully converged
    field (any face drop re-queues, exact in-brick convergence) on nodes with T >= 2h/v_max."""
    import torch

    ns = len(sv.shots)
    sizes = ctx.volume_sizes(ns, sv.windows)
    ref = torch.empty(sum(sizes), dtype=torch.float32, device="cuda")
    out = torch.empty_like(ref)
    ctx.eik_solve(sv.shots, windows=sv.windows, want_recv=False, change_tol=-1.0)
    ctx.eik_volumes_to(ref.data_ptr())
    ctx.eik_solve(sv.shots, windows=sv.windows, want_recv=False, **solver)
    ctx.eik_volumes_to(out.data_ptr())
    torch.cuda.synchronize()
    m = ref >= 2.0 * sv.h / float(sv.velocity.max())
    err = float(((out - ref).abs() / ref)[m].max())
    return {"max_rel_err_vs_converged": err, "budget": 1e-4, "nodes_checked": int(m.sum()),
            "reference": "same batch with change_tol < 0 (any drop re-queues) and exact in-brick convergence"}


def warm_start_bound(ctx, sv, stream, steps, barrier, dist, world, inflate=0.02):
    """Plain vs warm-started FIM on the same batch, with the best predictor there can be:
    the plain solution itself, inflated by 2 % into an upper bound (tomo_eik_solve_seeded).
    No learned predictor can seed the solve better, so its speed-up is bounded by this."""
    import torch

    ns = len(sv.shots)
    _, st_plain = ctx.eik_solve(sv.shots, windows=sv.windows, receivers=sv.receivers, want_recv=False)
    sizes = ctx.volume_sizes(ns, sv.windows)
    exact = torch.empty(sum(sizes), dtype=torch.float32, device="cuda")
    ctx.eik_volumes_to(exact.data_ptr())
    ctx.eik_solve_seeded(sv.shots, exact.data_ptr(), inflate, windows=sv.windows, receivers=sv.receivers,
                         want_recv=False)
    barrier()
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0.record(stream)
    for _ in range(steps):
        _, st, ss = ctx.eik_solve_seeded(sv.shots, exact.data_ptr(), inflate, windows=sv.windows,
                                         receivers=sv.receivers, want_recv=False)
    w1.record(stream)
    barrier()
    warm_ms = w0.elapsed_time(w1) / steps
    warm_ms = max_over_ranks(warm_ms, dist, 'cuda')
    out = torch.empty_like(exact)
    ctx.eik_volumes_to(out.data_ptr())
    torch.cuda.synchronize()
    m = exact >= 2.0 * sv.h / float(sv.velocity.max())
    err = float(((out - exact).abs() / exact)[m].max())
    # the same call path with the exact field and no margin: the cost of the check alone
    _, _, sv0 = ctx.eik_solve_seeded(sv.shots, exact.data_ptr(), 0.0, windows=sv.windows, want_recv=False)
    return {"predictor": "exact plain-FIM field x (1 + inflate): the upper bound of any learned predictor",
            "inflate": inflate, "value": world * ns / (warm_ms / 1000.0), "unit": UNIT, "ms_per_step": warm_ms,
            "steps": steps, "activations_plain": st_plain["activations"], "activations_warm": st["activations"],
            "inner_plain": st_plain["inner_iterations"], "inner_warm": st["inner_iterations"],
            "seeded_ms": ss["seeded_ms"], "verify_ms": ss["verify_ms"], "fallback_ms": ss["fallback_ms"],
            "shots_fallback": ss["shots_fallback"], "max_rel_err_vs_plain": err,
            "exact_no_margin": {"activations": sv0["activations_seeded"], "verify_ms": sv0["verify_ms"],
                                "shots_fallback": sv0["shots_fallback"]}}


def run_inversion(args):
    """Config 5 on its own JSON line (not the headline metric); see inversion_object."""
    print(json.dumps(inversion_object(args)), flush=True)
    return 0


def inversion_object(args, iterations=None):
    """Config 5: the large device-resident inversion -- 401x401x201 nodes at 10 m (32.3 M),
    256 shots x 10,000 receivers, 50 m inversion cells, `iterations` (default 5) iterations
    of eikonal -> rays -> CGLS (30) -> model update with every field, matrix and vector kept
    in HBM.  Returns its JSON object."""
    import torch

    import seismic_tomography_3d_b200 as tomo
    from seismic_tomography_3d_b200 import workloads as wl

    t_wall = time.perf_counter()
    sv, start, inv = wl.config5_inversion()
    if iterations:
        inv = dict(inv, iterations=iterations)
    rng = np.random.default_rng(5)
    ctx = tomo.Context(sv.nx, sv.ny, sv.nz, sv.h)
    stream = torch.cuda.ExternalStream(ctx.stream)
    ctx.set_velocity(sv.velocity)
    dobs, st_true = ctx.eik_solve(sv.shots, receivers=sv.receivers)
    dobs = (dobs + rng.normal(0.0, inv["pick_noise"], dobs.shape)).astype(np.float32)
    ctx.set_velocity(start)
    ctx.set_observed(dobs)
    free, total = torch.cuda.mem_get_info()
    iters = []
    for it in range(inv["iterations"] if not args.no_graph else 0):
        # the whole iteration in one call, replayed from CUDA graphs after the first
        st = ctx.iteration(sv.shots, sv.receivers, inv["d_tomo"], tk_order=inv["tk_order"], tk_param=inv["tk_param"],
                           cg_iterations=inv["cg_iterations"], smooth=inv["smooth"],
                           filter_samples=inv["filter_samples"], standard_deviation=inv["standard_deviation"],
                           use_graph=True, **SOLVER_BANDED)
        if it == 0:
            free, total = torch.cuda.mem_get_info()
        iters.append({"residual_l2_s": st["residual"], "total_ms": st["ms"], "nnz": st["nnz"],
                      "activations": st["activations"], "captured": st["captured"], "replayed": st["replayed"],
                      "cgls_rnorm": st["cg_rnorm"]})
    for it in range(inv["iterations"] if args.no_graph else 0):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        ev[0].record(stream)
        _, est = ctx.eik_solve(sv.shots, receivers=sv.receivers, want_recv=False, **SOLVER_BANDED)
        ev[1].record(stream)
        res = ctx.data_residual()
        jst = ctx.build_jacobian(inv["d_tomo"], inv["tk_order"], inv["tk_param"])
        ev[2].record(stream)
        _, hist, cst = ctx.cgls(inv["cg_iterations"], want_x=False)
        ev[3].record(stream)
        ctx.model_update(inv["smooth"], inv["filter_samples"], inv["standard_deviation"], want_velocity=False)
        ev[4].record(stream)
        torch.cuda.synchronize()
        if it == 0:
            free, total = torch.cuda.mem_get_info()
        ms = [a.elapsed_time(b) for a, b in zip(ev[:4], ev[1:])]
        iters.append({"residual_l2_s": res, "eikonal_ms": ms[0], "jacobian_ms": ms[1], "cgls_ms": ms[2],
                      "update_ms": ms[3], "total_ms": ev[0].elapsed_time(ev[4]),
                      "activations": est["activations"], "rounds": est["rounds"], "nnz": jst["nnz"],
                      "rays_ok": jst["rays_ok"], "rays_stalled": jst["rays_stalled"], "rays_capped": jst["rays_capped"],
                      "rays_nonfinite": jst["rays_nonfinite"], "rays_outside": jst["rays_outside"],
                      "rays_overflow": jst["rays_overflow"], "ray_steps": jst["ray_steps"],
                      "cgls_rnorm": cst["rnorm"]})
    ctx.eik_solve(sv.shots, receivers=sv.receivers, want_recv=False, **SOLVER_BANDED)
    final_res = ctx.data_residual()
    v_est = 1.0 / ctx.get_slowness()
    v_true, v0 = sv.velocity.astype(np.float64), start.astype(np.float64)
    rms = float(np.sqrt(np.mean(((v_est - v_true) / v_true) ** 2)))
    rms0 = float(np.sqrt(np.mean(((v0 - v_true) / v_true) ** 2)))
    keys = ("total_ms",) if not args.no_graph else ("eikonal_ms", "jacobian_ms", "cgls_ms", "update_ms", "total_ms")
    med = {k: statistics.median(i[k] for i in iters) for k in keys}
    stages = None
    if not args.no_graph:
        # one more iteration stage by stage (after the model figures above): where the time goes
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        ev[0].record(stream)
        ctx.eik_solve(sv.shots, receivers=sv.receivers, want_recv=False, **SOLVER_BANDED)
        ev[1].record(stream)
        ctx.build_jacobian(inv["d_tomo"], inv["tk_order"], inv["tk_param"])
        ev[2].record(stream)
        ctx.cgls(inv["cg_iterations"], want_x=False)
        ev[3].record(stream)
        ctx.model_update(inv["smooth"], inv["filter_samples"], inv["standard_deviation"], want_velocity=False)
        ev[4].record(stream)
        torch.cuda.synchronize()
        stages = dict(zip(("eikonal_ms", "jacobian_ms", "cgls_ms", "update_ms"),
                          (a.elapsed_time(b) for a, b in zip(ev[:4], ev[1:]))))
        stages["total_ms"] = ev[0].elapsed_time(ev[4])
    br = stages or med
    line = {"metric": "device-resident inversion iteration time (config 5)", "value": med["total_ms"], "unit": "ms",
            "higher_is_better": False, "iterations": len(iters), "iteration_ms_median": med["total_ms"],
            "graph_captured": not args.no_graph, "stage_breakdown_ms": br,
            "shots_per_s_eikonal": len(sv.shots) / (br["eikonal_ms"] / 1000.0),
            "cgls_ms_per_iteration": br["cgls_ms"] / inv["cg_iterations"],
            "recovered_model_rms_rel_err": rms, "starting_model_rms_rel_err": rms0,
            "residual_l2_s": [i["residual_l2_s"] for i in iters] + [final_res],
            "hbm_used_gb": (total - free) / 1e9, "per_iteration": iters,
            "config": {"workload": "config5: 401x401x201 @10 m (32.3 M nodes), 256 shots x 10,000 receivers, "
                                   "full windows, 50 m cells (81x81x41), tk order 2 lambda 0.1, 30 CGLS, 5 iterations",
                       "eikonal_tolerances_s": SOLVER_BANDED,
                       "start": "v(z) = 1500 + 1.0 z", "picks": "plain FIM on the true model + N(0, 2 ms)"},
            "data": "synthetic (seeded config-5 model, shots, receivers)",
            "wall_s": time.perf_counter() - t_wall}
    ctx.close()
    return line


def run_warm_start(args):
    """Config 4 on its own JSON line (not the headline metric); see learned_warm_object."""
    print(json.dumps(learned_warm_object(args.fields, args.epochs)), flush=True)
    return 0


def learned_warm_object(fields, epochs, strides=(1, 4, 8)):
    """Config 4: the learned warm start end to end -- `fields` solver-generated training
    fields on seeded random models, the U-Net trained on the device for `epochs`, then used
    on the config-2 batch: prediction (full resolution, and on every 4th and 8th node with
    tau interpolated back) -> ceiling (x 1.02) -> warm-started FIM (solve at the timed
    tolerances, check, fallback), against the plain FIM at the same tolerances.  Returns
    its JSON object; `value` is the best of the strides."""
    import torch

    import seismic_tomography_3d_b200 as tomo
    from seismic_tomography_3d_b200 import surrogate

    t0 = time.perf_counter()
    ds = surrogate.make_dataset(nfields=fields, tile=64, nz=64, h=12.5)
    net = tomo.Net(seed=0)
    summ = surrogate.train(net, ds, epochs=epochs, batch=8, lr=1e-3)
    gen_s, gen_solve_ms = ds.gen_s, ds.solve_ms
    del ds
    torch.cuda.empty_cache()
    sv = workload(0)
    ns = len(sv.shots)
    ctx = tomo.Context(sv.nx, sv.ny, sv.nz, sv.h)
    ctx.set_velocity(sv.velocity)
    for _ in range(2):
        _, st_plain = ctx.eik_solve(sv.shots, windows=sv.windows, **SOLVER)
    plain_ms = statistics.median(ctx.eik_solve(sv.shots, windows=sv.windows, **SOLVER)[1]["total_ms"]
                                 for _ in range(5))
    sizes = ctx.volume_sizes(ns, sv.windows)
    exact = torch.empty(sum(sizes), dtype=torch.float32, device="cuda")
    ctx.eik_volumes_to(exact.data_ptr())
    vmin_t = 2.0 * sv.h / float(sv.velocity.max())
    out = torch.empty_like(exact)
    variants = []
    for stride in strides:
        # the network on every stride-th node (1: all), tau interpolated back to every node
        pred, infer_ms = surrogate.predict_ceiling(net, ctx, sv.shots, sv.windows, stride=stride)
        pred, infer_ms = surrogate.predict_ceiling(net, ctx, sv.shots, sv.windows, stride=stride)
        m = (exact >= vmin_t) & (pred > 0)
        rel = ((pred - exact) / exact)[m]
        runs = [ctx.eik_solve_seeded(sv.shots, pred.data_ptr(), 0.02, windows=sv.windows, **SOLVER) for _ in range(3)]
        _, st_w, ss_w = runs[-1]
        warm_ms = statistics.median(r[1]["total_ms"] for r in runs)
        ctx.eik_volumes_to(out.data_ptr())
        torch.cuda.synchronize()
        err = float(((out - exact).abs() / exact)[exact >= vmin_t].max())
        variants.append({
            "stride": stride, "value": ns / ((warm_ms + infer_ms) / 1000.0),
            "speedup_vs_plain": plain_ms / (warm_ms + infer_ms),
            "ms_inference": infer_ms, "ms_per_batch_solve": warm_ms,
            "inference_frac_of_plain": infer_ms / plain_ms,
            "activations": st_w["activations"], "inner_iterations": st_w["inner_iterations"],
            "activations_seeded_launch": ss_w["activations_seeded"], "shots_fallback": ss_w["shots_fallback"],
            "violations": ss_w["violations"], "stuck": ss_w["stuck"], "max_rel_err_vs_plain": err,
            "predictor_rel_err": {"median_abs": float(rel.abs().median()),
                                  "p99_abs": float(rel.abs().float().quantile(0.99)) if rel.numel() < 16_000_000 else None,
                                  "frac_below_truth_by_2pct": float((rel < -0.02).float().mean())}})
        del pred
    best = max(variants, key=lambda v: v["speedup_vs_plain"])
    line = {"metric": "learned warm start vs plain FIM (config 4 surrogate on the config-2 batch)",
            "value": best["value"], "unit": UNIT, "higher_is_better": True,
            "speedup_vs_plain": best["speedup_vs_plain"], "best_stride": best["stride"],
            "max_rel_err_vs_plain": max(v["max_rel_err_vs_plain"] for v in variants),
            "shots_fallback": best["shots_fallback"],
            "plain": {"value": ns / (plain_ms / 1000.0), "ms_per_batch": plain_ms,
                      "activations": st_plain["activations"], "inner_iterations": st_plain["inner_iterations"]},
            "warm": variants,
            "tolerances_s": SOLVER, "inflate": 0.02,
            "training": {k: v for k, v in summ.items() if k != "history"}, "history": summ["history"],
            "data": {"fields": fields, "epochs": epochs, "tile": [64, 64, 64], "h_m": 12.5,
                     "models": "seeded random: 3-6 dipping layers 1500-4500 m/s, 0-12 Gaussian anomalies +-15 %",
                     "generation_s": gen_s, "generation_solve_ms": gen_solve_ms},
            "wall_s": time.perf_counter() - t0}
    net.close()
    ctx.close()
    del exact, out
    torch.cuda.empty_cache()
    return line


def run_tomography(args):
    """Config 3 on its own JSON line (not the headline metric); see tomography_object."""
    print(json.dumps(tomography_object(args, args.steps, args.warmup)), flush=True)
    return 0


def tomography_object(args, steps, warmup):
    """Config 3: one full tomography iteration on the device (64 shots x 2,500 receivers,
    201x201x101 at 12.5 m, 50x50x25 cells, Tikhonov order 2, lambda 0.1, 30 CGLS
    iterations), warmup + steps times from the same starting model.  Returns its JSON
    object."""
    import torch

    import seismic_tomography_3d_b200 as tomo
    from seismic_tomography_3d_b200 import workloads as wl

    sv, start, inv = wl.config3()
    rng = np.random.default_rng(3)
    ctx = tomo.Context(sv.nx, sv.ny, sv.nz, sv.h)
    ctx.set_velocity(sv.velocity)
    dobs, _ = ctx.eik_solve(sv.shots, receivers=sv.receivers)
    dobs = (dobs + rng.normal(0.0, inv["pick_noise"], dobs.shape)).astype(np.float32)
    stream = torch.cuda.ExternalStream(ctx.stream)
    timings = {k: [] for k in ("eikonal", "jacobian", "cgls", "update", "total")}
    last = {}
    # the starting model is uploaded every iteration (from pinned host memory, as a caller
    # that keeps its model in a pinned buffer would), so each iteration starts alike
    start_pinned = torch.from_numpy(np.ascontiguousarray(start)).pin_memory()
    for it in range(warmup + steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        ev[0].record(stream)
        assert ctx.lib.tomo_set_velocity(ctx.h, start_pinned.data_ptr()) == 0
        _, est = ctx.eik_solve(sv.shots, receivers=sv.receivers, want_recv=False, **SOLVER_BANDED)
        ev[1].record(stream)
        jst = ctx.build_jacobian(inv["d_tomo"], inv["tk_order"], inv["tk_param"])
        ev[2].record(stream)
        ctx.set_observed(dobs)
        _, hist, cst = ctx.cgls(inv["cg_iterations"], want_x=False)
        ev[3].record(stream)
        ctx.model_update(inv["smooth"], inv["filter_samples"], inv["standard_deviation"], want_velocity=False)
        ev[4].record(stream)
        torch.cuda.synchronize()
        if it >= warmup:
            for k, (a, b) in zip(("eikonal", "jacobian", "cgls", "update"), zip(ev[:4], ev[1:])):
                timings[k].append(a.elapsed_time(b))
            timings["total"].append(ev[0].elapsed_time(ev[4]))
        last = dict(eik=est, jac=jst, cgls=cst, hist=hist)
    med = {k: statistics.median(v) for k, v in timings.items()}
    j, c = last["jac"], last["cgls"]
    N, M, nnz = j["rows"], j["cols"], j["nnz"]
    cg_bytes = 16 * nnz + 4 * (N + M) + 8 * (5 * N + 8 * M)  # per CGLS iteration: A and A^T values + indices (16 B/nnz), row pointers, FP64 vector streams
    cg_ms_it = c["ms"] / max(c["iterations"], 1)
    peak, peak_kind = peaks()
    line = {"metric": "tomography iteration time (config 3)", "value": med["total"], "unit": "ms",
            "higher_is_better": False, "steps": steps, "warmup": warmup,
            "breakdown_ms": med, "shots_per_s_eikonal": len(sv.shots) / (med["eikonal"] / 1000.0),
            "jacobian": {k: j[k] for k in ("rows", "cols", "nnz_rays", "nnz", "rays", "rays_ok", "rays_stalled",
                                           "rays_capped", "rays_nonfinite", "rays_outside", "ray_steps")},
            "ray_steps_per_s": j["ray_steps"] / (med["jacobian"] / 1000.0),
            "cgls": {"iterations": c["iterations"], "ms_per_iteration": cg_ms_it, "rnorm0": c["rnorm0"],
                     "rnorm": c["rnorm"],
                     "roofline": {"bound": "hbm", "achieved": cg_bytes / (cg_ms_it / 1000.0) / 1e9, "peak": peak,
                                  "unit": "GB/s", "frac": cg_bytes / (cg_ms_it / 1000.0) / 1e9 / peak,
                                  "peak_kind": peak_kind, "alg_bytes_per_iteration": cg_bytes}},
            "eikonal_tolerances_s": SOLVER_BANDED,
            "data": "synthetic (seeded config-3 model, 64 shots x 2500 receivers, picks + N(0, 2 ms))"}
    ctx.close()
    return line


def run_jacobian(args):
    """Ray tracing into the Jacobian at config-5 scale: the config-5 starting model and its
    first --shots shots (default all 256) x 10,000 receivers, solved once; then the Jacobian
    (ray march, run sort, emit, Tikhonov rows, transpose) built warmup + steps times.
    Prints its own JSON line (not the headline metric)."""
    import torch

    import seismic_tomography_3d_b200 as tomo
    from seismic_tomography_3d_b200 import workloads as wl

    sv, start, inv = wl.config5_inversion()
    shots = sv.shots[:args.shots] if args.shots else sv.shots
    ctx = tomo.Context(sv.nx, sv.ny, sv.nz, sv.h)
    stream = torch.cuda.ExternalStream(ctx.stream)
    ctx.set_velocity(start)
    ctx.eik_solve(shots, receivers=sv.receivers, want_recv=False, **SOLVER_BANDED)
    ms = []
    for it in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        j = ctx.build_jacobian(inv["d_tomo"], inv["tk_order"], inv["tk_param"])
        e1.record(stream)
        torch.cuda.synchronize()
        if it >= args.warmup:
            ms.append(e0.elapsed_time(e1))
    med = statistics.median(ms)
    line = {"metric": "Jacobian build time (config-5 model)", "value": med, "unit": "ms",
            "higher_is_better": False, "steps": args.steps, "warmup": args.warmup,
            "ray_steps_per_s": j["ray_steps"] / (med / 1000.0),
            "jacobian": {k: j[k] for k in ("rows", "cols", "nnz", "rays", "rays_ok", "rays_stalled", "rays_capped",
                                           "rays_nonfinite", "rays_outside", "ray_steps")},
            "config": {"workload": "config-5 starting model, first %d shots x 10,000 receivers, 50 m cells"
                                   % len(shots)},
            "data": "synthetic (seeded config-5 model, shots, receivers)"}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shots", type=int, default=0, help="first N shots of the batch only (profiling)")
    ap.add_argument("--tomography", action="store_true",
                    help="time one config-3 tomography iteration instead (separate JSON line)")
    ap.add_argument("--inversion", action="store_true",
                    help="run the config-5 device-resident inversion instead (separate JSON line)")
    ap.add_argument("--jacobian", action="store_true",
                    help="time the Jacobian build on the config-5 model (first --shots shots) instead")
    ap.add_argument("--no-graph", action="store_true",
                    help="--inversion: call the stages one by one instead of tomo_iteration's CUDA graphs")
    ap.add_argument("--warm-start", action="store_true",
                    help="run the config-4 learned warm start instead (separate JSON line)")
    ap.add_argument("--fields", type=int, default=20000, help="training fields (--warm-start)")
    ap.add_argument("--epochs", type=int, default=3, help="training epochs (--warm-start)")
    ap.add_argument("--warm-fields", type=int, default=4000,
                    help="training fields of the default line's learned_warm object")
    ap.add_argument("--warm-epochs", type=int, default=2, help="its training epochs")
    ap.add_argument("--headline-only", action="store_true",
                    help="the config-2 headline alone (no config1/tomography/learned_warm/inversion objects)")
    ap.add_argument("--no-inversion", action="store_true", help="skip the config-5 inversion object")
    ap.add_argument("--no-autotune", action="store_true",
                    help="headline solve with the built-in default shape instead of the autotuned one")
    ap.add_argument("--brick", type=int, default=0, choices=[0, 1, 2],
                    help="headline solve with this brick shape (1: 4x4x4, 2: 8x8x8), untuned (profiling)")
    ap.add_argument("--schedule", type=int, default=0, choices=[0, 3],
                    help="3: headline solve with two bricks per warp at 8 warps x 3 CTAs per SM, untuned "
                         "(profiling)")
    args = ap.parse_args()
    if args.warm_start:
        return run_warm_start(args)
    if args.tomography:
        return run_tomography(args)
    if args.inversion:
        return run_inversion(args)
    if args.jacobian:
        return run_jacobian(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
