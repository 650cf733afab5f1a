"""seismic_tomography_3d_b200 -- Python view of the libtomo_b200 C ABI.

The product is the shared library ``_lib/libtomo_b200.so`` (CUDA kernels for sm_100a plus
the C ABI declared in ``include/tomo_b200.h``).  This module only binds it with ctypes for
tests, benchmarks and scripting; every call goes straight through the C ABI.  There is no
CPU fallback: without the library or an sm_100 GPU the calls raise.

Array convention: a volume is a numpy array of shape (ny, nx, nz) in C order, which is
exactly the reference's z-fastest layout ``idx = z + x*nz + y*nx*nz``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "_lib", "libtomo_b200.so")
INCLUDE_DIR = os.path.join(os.path.dirname(_PKG), "include")

TOMO_OK = 0
ERRORS = {
    -1: "TOMO_ERR_INVALID_ARG", -2: "TOMO_ERR_OOM", -3: "TOMO_ERR_CUDA", -4: "TOMO_ERR_NOT_CONVERGED",
    -5: "TOMO_ERR_TIMEOUT", -6: "TOMO_ERR_STATE", -7: "TOMO_ERR_IO", -8: "TOMO_ERR_NO_DEVICE",
    -9: "TOMO_ERR_CAPACITY",
}


class TomoError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{ERRORS.get(status, status)}: {msg}")
        self.status = status


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_float), ("dy", ctypes.c_float), ("dz", ctypes.c_float)]


class Point(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("z", ctypes.c_float)]


class Window(ctypes.Structure):
    _fields_ = [("x0", ctypes.c_int), ("x1", ctypes.c_int), ("y0", ctypes.c_int), ("y1", ctypes.c_int)]


class EikOpts(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int), ("max_inner", ctypes.c_int), ("max_rounds", ctypes.c_int),
                ("brick", ctypes.c_int), ("block_warps", ctypes.c_int), ("occupancy", ctypes.c_int),
                ("change_tol", ctypes.c_float), ("inner_tol", ctypes.c_float),
                ("ieee_sqrt", ctypes.c_int), ("sweep_groups", ctypes.c_int), ("schedule", ctypes.c_int),
                ("time_band", ctypes.c_float), ("spin_limit", ctypes.c_ulonglong)]


class EikStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_longlong), ("activations", ctypes.c_longlong),
                ("inner_iterations", ctypes.c_longlong), ("nodes_per_brick", ctypes.c_longlong),
                ("idle_activations", ctypes.c_longlong),
                ("setup_ms", ctypes.c_float), ("solve_ms", ctypes.c_float), ("total_ms", ctypes.c_float),
                ("deferred", ctypes.c_longlong)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class TuneStats(ctypes.Structure):
    _fields_ = [("trials", ctypes.c_int), ("best_ms", ctypes.c_float), ("default_ms", ctypes.c_float)]


class SeedStats(ctypes.Structure):
    _fields_ = [("violations", ctypes.c_longlong), ("max_deficit", ctypes.c_float), ("shots_fallback", ctypes.c_int),
                ("rounds_seeded", ctypes.c_longlong), ("activations_seeded", ctypes.c_longlong),
                ("inner_iterations_seeded", ctypes.c_longlong), ("seeded_ms", ctypes.c_float),
                ("verify_ms", ctypes.c_float), ("fallback_ms", ctypes.c_float), ("stuck", ctypes.c_longlong)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libtomo_b200.so (raises if it has not been built: no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libtomo_b200.so not built ({path}); run "
                           "`python -m seismic_tomography_3d_b200.build`")
    lib = ctypes.CDLL(path)
    P, I, F, V = ctypes.POINTER, ctypes.c_int, ctypes.c_float, ctypes.c_void_p
    lib.tomo_ctx_create.argtypes = [P(Grid), I, P(V)]
    lib.tomo_ctx_create_on_stream.argtypes = [P(Grid), I, V, P(V)]
    lib.tomo_ctx_destroy.argtypes = [V]
    lib.tomo_last_error.argtypes = [V]
    lib.tomo_last_error.restype = ctypes.c_char_p
    lib.tomo_status_string.argtypes = [I]
    lib.tomo_status_string.restype = ctypes.c_char_p
    lib.tomo_ctx_stream.argtypes = [V]
    lib.tomo_ctx_stream.restype = V
    lib.tomo_set_velocity.argtypes = [V, V]
    lib.tomo_set_slowness.argtypes = [V, V]
    lib.tomo_get_slowness.argtypes = [V, V]
    lib.tomo_stage_velocity.argtypes = [V, V]
    lib.tomo_commit_velocity.argtypes = [V]
    lib.tomo_eik_solve.argtypes = [V, I, P(Point), P(Window), I, P(Point), V, P(EikOpts), P(EikStats)]
    lib.tomo_eik_volume.argtypes = [V, I, V]
    lib.tomo_eik_window.argtypes = [V, I, P(Window)]
    lib.tomo_eik_brick_shapes.argtypes = [P(I), I]
    lib.tomo_eik_volumes.argtypes = [V, V]
    lib.tomo_eik_autotune.argtypes = [V, I, P(Point), P(Window), I, P(EikOpts), P(TuneStats)]
    lib.tomo_eik_solve_seeded.argtypes = [V, I, P(Point), P(Window), I, P(Point), V, V, F, P(EikOpts),
                                          P(EikStats), P(SeedStats)]
    _bind_tomography(lib)
    _lib = lib
    return lib


class JacobianOpts(ctypes.Structure):
    _fields_ = [("dx", ctypes.c_float), ("dy", ctypes.c_float), ("dz", ctypes.c_float),
                ("tk_order", ctypes.c_int), ("tk_param", ctypes.c_float), ("max_ray_steps", ctypes.c_int),
                ("max_cells_per_ray", ctypes.c_int), ("illumination", ctypes.c_int)]


class JacobianStats(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int)] + [
        (n, ctypes.c_longlong) for n in ("rows", "cols", "nnz_rays", "nnz", "rays", "rays_ok", "rays_stalled",
                                         "rays_capped", "rays_nonfinite", "rays_outside", "rays_overflow",
                                         "ray_steps")] + [("ms", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class CglsStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("rnorm0", ctypes.c_double), ("rnorm", ctypes.c_double),
                ("ms", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class UpdateOpts(ctypes.Structure):
    _fields_ = [("smooth", ctypes.c_int), ("filter_samples", ctypes.c_int),
                ("standard_deviation", ctypes.c_float), ("use_reference_masks", ctypes.c_int)]


class NetSample(ctypes.Structure):
    _fields_ = [("slow", ctypes.c_void_p), ("model_nx", ctypes.c_int), ("model_ny", ctypes.c_int),
                ("nz", ctypes.c_int), ("window", Window), ("source", Point), ("T", ctypes.c_void_p)]


def _bind_net(lib):
    """Bindings of the surrogate (learned warm start) part of the ABI."""
    P, I, V, F, D = ctypes.POINTER, ctypes.c_int, ctypes.c_void_p, ctypes.c_float, ctypes.c_double
    lib.tomo_net_create.argtypes = [I, V, ctypes.c_ulonglong, P(V)]
    lib.tomo_net_destroy.argtypes = [V]
    lib.tomo_net_last_error.argtypes = [V]
    lib.tomo_net_last_error.restype = ctypes.c_char_p
    lib.tomo_net_param_count.argtypes = [V]
    lib.tomo_net_param_count.restype = ctypes.c_longlong
    lib.tomo_net_get_params.argtypes = [V, V]
    lib.tomo_net_set_params.argtypes = [V, V]
    lib.tomo_net_gradients.argtypes = [V, I, P(NetSample), F, P(D), V]
    lib.tomo_net_train_step.argtypes = [V, I, P(NetSample), F, F, P(D)]
    lib.tomo_net_evaluate.argtypes = [V, I, P(NetSample), F, P(D)]
    lib.tomo_net_predict.argtypes = [V, I, P(NetSample), F, V, P(F)]
    lib.tomo_net_predict_strided.argtypes = [V, I, P(NetSample), F, I, V, P(F)]
    lib.tomo_random_tiles.argtypes = [V, I, ctypes.c_ulonglong]
    lib.tomo_ctx_slowness_device.argtypes = [V]
    lib.tomo_ctx_slowness_device.restype = V


class IterationOpts(ctypes.Structure):
    _fields_ = [("jacobian", JacobianOpts), ("cg_iterations", ctypes.c_int), ("update", UpdateOpts),
                ("eik", EikOpts), ("use_graph", ctypes.c_int), ("nnz_headroom", ctypes.c_float)]


class IterationStats(ctypes.Structure):
    _fields_ = [("residual", ctypes.c_double), ("cg_rnorm", ctypes.c_double), ("nnz", ctypes.c_longlong),
                ("activations", ctypes.c_longlong), ("replayed", ctypes.c_int), ("captured", ctypes.c_int),
                ("ms", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def _bind_tomography(lib):
    """Bindings of the tomography half of the ABI."""
    _bind_net(lib)
    P, I, V = ctypes.POINTER, ctypes.c_int, ctypes.c_void_p
    lib.tomo_build_jacobian.argtypes = [V, P(JacobianOpts), P(JacobianStats)]
    lib.tomo_jacobian_copy.argtypes = [V, V, V, V]
    lib.tomo_ray_status.argtypes = [V, V]
    lib.tomo_illumination.argtypes = [V, V]
    lib.tomo_set_observed.argtypes = [V, V, I]
    lib.tomo_catch_parameter.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, I]
    lib.tomo_geometry.argtypes = [ctypes.c_char_p, ctypes.c_char_p, I, V, I]
    lib.tomo_data_residual.argtypes = [V, P(ctypes.c_double)]
    lib.tomo_cgls.argtypes = [V, I, V, V, P(CglsStats)]
    lib.tomo_model_update.argtypes = [V, P(UpdateOpts), V]
    lib.tomo_sparse_cgls_gpu.argtypes = [V, V, V, V, V, I, I, I, I, ctypes.c_float]
    lib.tomo_iteration.argtypes = [V, I, P(Point), P(Window), I, P(Point), P(IterationOpts), P(IterationStats)]


def sparse_cgls_gpu(iA, jA, vA, B, N, M, nit, tol=0.0):
    """The reference's sparse_cgls_gpu entry point (src/utils/cgls/cgls.cuh:47)."""
    lib = load_library()
    iA = np.ascontiguousarray(iA, np.int32)
    jA = np.ascontiguousarray(jA, np.int32)
    vA = np.ascontiguousarray(vA, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    x = np.zeros(M, np.float32)
    rc = lib.tomo_sparse_cgls_gpu(iA.ctypes.data, jA.ctypes.data, vA.ctypes.data, B.ctypes.data, x.ctypes.data,
                                  N, M, len(vA), nit, tol)
    if rc != TOMO_OK:
        raise TomoError(rc, lib.tomo_status_string(rc).decode())
    return x


def _points(a):
    """(n, 3) float32 array viewed as tomo_point[n] without copying (tomo_point is three
    packed floats).  Returns (pointer, n, owner) -- keep `owner` alive during the call."""
    a = np.ascontiguousarray(np.asarray(a, np.float32).reshape(-1, 3))
    return a.ctypes.data_as(ctypes.POINTER(Point)), len(a), a


def _windows(w):
    w = np.ascontiguousarray(np.asarray(w, np.int32).reshape(-1, 4))
    return w.ctypes.data_as(ctypes.POINTER(Window)), w


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Context:
    """One device context (tomo_ctx) over a model grid."""

    def __init__(self, nx, ny, nz, dx, dy=None, dz=None, device=0, stream=None):
        self.lib = load_library()
        self.grid = Grid(nx, ny, nz, dx, dy if dy is not None else dx, dz if dz is not None else dx)
        self.shape = (ny, nx, nz)
        h = ctypes.c_void_p()
        if stream is None:
            rc = self.lib.tomo_ctx_create(ctypes.byref(self.grid), device, ctypes.byref(h))
        else:
            rc = self.lib.tomo_ctx_create_on_stream(ctypes.byref(self.grid), device, ctypes.c_void_p(stream),
                                                    ctypes.byref(h))
        if rc != TOMO_OK:
            raise TomoError(rc, self.lib.tomo_status_string(rc).decode())
        self.h = h

    # -- plumbing ---------------------------------------------------------------------
    def _check(self, rc):
        if rc != TOMO_OK:
            raise TomoError(rc, self.lib.tomo_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.tomo_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self):
        return self.lib.tomo_ctx_stream(self.h)

    # -- model --------------------------------------------------------------------------
    def set_velocity(self, v):
        v = _f32(v)
        assert v.shape == self.shape, (v.shape, self.shape)
        self._check(self.lib.tomo_set_velocity(self.h, v.ctypes.data))

    def stage_velocity(self, v):
        """Starts copying the next velocity model to the device (tomo_stage_velocity); the
        array is kept alive here until the next stage call.  Page-locked memory (a pinned
        torch tensor's data) overlaps the copy with queued work."""
        if isinstance(v, np.ndarray):
            v = _f32(v)
            assert v.shape == self.shape, (v.shape, self.shape)
            self._staged_host = v
            ptr = v.ctypes.data
        else:  # a (pinned) float32 torch tensor of the model's shape
            assert tuple(v.shape) == self.shape and str(v.dtype) == "torch.float32" and v.is_contiguous()
            self._staged_host = v
            ptr = v.data_ptr()
        self._check(self.lib.tomo_stage_velocity(self.h, ptr))

    def commit_velocity(self):
        """The staged velocity becomes the model (tomo_commit_velocity)."""
        self._check(self.lib.tomo_commit_velocity(self.h))

    def set_slowness(self, s):
        s = _f32(s)
        assert s.shape == self.shape
        self._check(self.lib.tomo_set_slowness(self.h, s.ctypes.data))

    def get_slowness(self):
        out = np.empty(self.shape, np.float32)
        self._check(self.lib.tomo_get_slowness(self.h, out.ctypes.data))
        return out

    # -- eikonal ------------------------------------------------------------------------
    def eik_solve(self, shots, windows=None, receivers=None, want_recv=True, max_inner=0, max_rounds=0,
                  block_warps=0, op=0, occupancy=0, change_tol=0.0, inner_tol=0.0, ieee_sqrt=0,
                  sweep_groups=0, schedule=0, time_band=0.0, spin_limit=0, brick=0, out=None):
        """Batched solve.  shots (n,3) metres; windows (n,4) [x0,x1,y0,y1] nodes or None;
        receivers (m,3).  Returns (t_recv (n,m) float32 or None, stats dict).  out: a
        C-contiguous float32 (n,m) array to receive t_recv (e.g. a view of page-locked memory,
        which the device copies into directly)."""
        sp, ns, _s = _points(shots)
        wp = _w = None
        if windows is not None:
            wp, _w = _windows(windows)
        nr = 0
        rp = _r = None
        if receivers is not None and len(receivers):
            rp, nr, _r = _points(receivers)
        if want_recv and nr and out is not None:
            assert out.shape == (ns, nr) and out.dtype == np.float32 and out.flags["C_CONTIGUOUS"]
        elif want_recv and nr:
            out = np.empty((ns, nr), np.float32)
        else:
            out = None
        opts = EikOpts(op, max_inner, max_rounds, brick, block_warps, occupancy, change_tol, inner_tol, ieee_sqrt,
                       sweep_groups, schedule, time_band, spin_limit)
        st = EikStats()
        self._check(self.lib.tomo_eik_solve(self.h, ns, sp, wp, nr, rp,
                                            out.ctypes.data if out is not None else None,
                                            ctypes.byref(opts), ctypes.byref(st)))
        return out, st.as_dict()

    def eik_solve_seeded(self, shots, ceiling_ptr, inflate=0.02, windows=None, receivers=None, want_recv=True,
                         max_inner=0, max_rounds=0, block_warps=0, occupancy=0, change_tol=0.0, inner_tol=0.0,
                         ieee_sqrt=0, schedule=0):
        """Warm-started batched solve (tomo_eik_solve_seeded).  ceiling_ptr: device address
        of all shots' predicted window volumes back to back (see volume_sizes).  Returns
        (t_recv or None, stats dict, seed-stats dict)."""
        sp, ns, _s = _points(shots)
        wp = _w = None
        if windows is not None:
            wp, _w = _windows(windows)
        nr = 0
        rp = _r = None
        if receivers is not None and len(receivers):
            rp, nr, _r = _points(receivers)
        out = np.empty((ns, nr), np.float32) if (want_recv and nr) else None
        opts = EikOpts(0, max_inner, max_rounds, 0, block_warps, occupancy, change_tol, inner_tol, ieee_sqrt, 0,
                       schedule)
        st, ss = EikStats(), SeedStats()
        self._check(self.lib.tomo_eik_solve_seeded(self.h, ns, sp, wp, nr, rp,
                                                   out.ctypes.data if out is not None else None,
                                                   ctypes.c_void_p(ceiling_ptr), float(inflate), ctypes.byref(opts),
                                                   ctypes.byref(st), ctypes.byref(ss)))
        return out, st.as_dict(), ss.as_dict()

    def eik_autotune(self, shots, windows=None, repeats=0):
        """Autotunes the launch shape on this batch; returns (chosen shape dict, stats dict)."""
        sp, ns, _s = _points(shots)
        wp = _w = None
        if windows is not None:
            wp, _w = _windows(windows)
        best, st = EikOpts(), TuneStats()
        self._check(self.lib.tomo_eik_autotune(self.h, ns, sp, wp, repeats, ctypes.byref(best), ctypes.byref(st)))
        shape = {"brick": best.brick, "block_warps": best.block_warps, "occupancy": best.occupancy,
                 "max_inner": best.max_inner, "time_band": best.time_band, "schedule": best.schedule}
        return shape, {f: getattr(st, f) for f, _ in st._fields_}

    def volume_sizes(self, nshots, windows=None):
        """Floats of each shot's window volume (nz*wx*wy) in the back-to-back layout."""
        if windows is None:
            return [self.grid.nz * self.grid.nx * self.grid.ny] * nshots
        w = np.asarray(windows).reshape(-1, 4)
        return [int(self.grid.nz * (x1 - x0) * (y1 - y0)) for x0, x1, y0, y1 in w]

    def eik_volumes_to(self, dst_ptr):
        """All window volumes of the last solve into the device array at dst_ptr."""
        self._check(self.lib.tomo_eik_volumes(self.h, ctypes.c_void_p(dst_ptr)))

    def random_tiles(self, tile, seed):
        """Seeded random layered tiles as the model (surrogate training data)."""
        self._check(self.lib.tomo_random_tiles(self.h, tile, seed))

    def slowness_device(self):
        """Device address of the current slowness model (z fastest)."""
        return self.lib.tomo_ctx_slowness_device(self.h)

    def eik_window(self, shot):
        w = Window()
        self._check(self.lib.tomo_eik_window(self.h, shot, ctypes.byref(w)))
        return (w.x0, w.x1, w.y0, w.y1)

    # -- tomography ---------------------------------------------------------------------
    def build_jacobian(self, d_tomo, tk_order=2, tk_param=0.1, max_ray_steps=0, max_cells_per_ray=0,
                       illumination=False):
        o = JacobianOpts(*map(float, d_tomo), tk_order, tk_param, max_ray_steps, max_cells_per_ray,
                         int(illumination))
        st = JacobianStats()
        self._check(self.lib.tomo_build_jacobian(self.h, ctypes.byref(o), ctypes.byref(st)))
        self.jac = st.as_dict()
        return self.jac

    def jacobian(self):
        """A = [G ; lambda L] as CSR (row_ptr, cols, vals)."""
        j = self.jac
        rp = np.empty(j["rows"] + 1, np.int32)
        cols = np.empty(j["nnz"], np.int32)
        vals = np.empty(j["nnz"], np.float32)
        self._check(self.lib.tomo_jacobian_copy(self.h, rp.ctypes.data, cols.ctypes.data, vals.ctypes.data))
        return rp, cols, vals

    def ray_status(self):
        out = np.empty(self.jac["rays"], np.int32)
        self._check(self.lib.tomo_ray_status(self.h, out.ctypes.data))
        return out

    def illumination(self):
        out = np.empty(self.shape, np.float32)
        self._check(self.lib.tomo_illumination(self.h, out.ctypes.data))
        return out

    def set_observed(self, dobs):
        d = _f32(dobs)
        self._check(self.lib.tomo_set_observed(self.h, d.ctypes.data, d.size))

    def data_residual(self):
        v = ctypes.c_double()
        self._check(self.lib.tomo_data_residual(self.h, ctypes.byref(v)))
        return v.value

    def cgls(self, iterations=30, want_x=True):
        x = np.empty(self.jac["cols"], np.float32) if want_x else None
        hist = np.empty(max(iterations, 1), np.float64)
        st = CglsStats()
        self._check(self.lib.tomo_cgls(self.h, iterations, x.ctypes.data if x is not None else None,
                                       hist.ctypes.data, ctypes.byref(st)))
        return x, hist[:iterations], st.as_dict()

    def model_update(self, smooth=True, filter_samples=5, standard_deviation=2.0, reference_masks=True,
                     want_velocity=True):
        o = UpdateOpts(int(smooth), filter_samples, standard_deviation, int(reference_masks))
        v = np.empty(self.shape, np.float32) if want_velocity else None
        self._check(self.lib.tomo_model_update(self.h, ctypes.byref(o), v.ctypes.data if v is not None else None))
        return v

    def iteration(self, shots, receivers, d_tomo, windows=None, tk_order=2, tk_param=0.1, cg_iterations=30,
                  smooth=True, filter_samples=5, standard_deviation=2.0, reference_masks=True, use_graph=True,
                  max_ray_steps=0, max_cells_per_ray=0, nnz_headroom=0.0, change_tol=0.0, inner_tol=0.0,
                  schedule=0, time_band=0.0):
        """One whole tomography iteration on the device (tomo_iteration); returns its stats."""
        sp, ns, _s = _points(shots)
        rp, nr, _r = _points(receivers)
        wp = _w = None
        if windows is not None:
            wp, _w = _windows(windows)
        o = IterationOpts()
        o.jacobian = JacobianOpts(*map(float, d_tomo), tk_order, tk_param, max_ray_steps, max_cells_per_ray, 0)
        o.cg_iterations = cg_iterations
        o.update = UpdateOpts(int(smooth), filter_samples, standard_deviation, int(reference_masks))
        o.eik = EikOpts(0, 0, 0, 0, 0, 0, change_tol, inner_tol, 0, 0, schedule, time_band)
        o.use_graph = int(use_graph)
        o.nnz_headroom = nnz_headroom
        st = IterationStats()
        self._check(self.lib.tomo_iteration(self.h, ns, sp, wp, nr, rp, ctypes.byref(o), ctypes.byref(st)))
        return st.as_dict()

    def eik_volume(self, shot):
        x0, x1, y0, y1 = self.eik_window(shot)
        out = np.empty((y1 - y0, x1 - x0, self.grid.nz), np.float32)
        self._check(self.lib.tomo_eik_volume(self.h, shot, out.ctypes.data))
        return out


def net_samples(items):
    """ctypes array of tomo_net_sample from dicts with keys slow (device address),
    model_nx, model_ny, nz, window (x0, x1, y0, y1), source (x, y, z), T (device address or 0)."""
    arr = (NetSample * len(items))()
    for i, it in enumerate(items):
        arr[i].slow = it["slow"]
        arr[i].model_nx, arr[i].model_ny, arr[i].nz = it["model_nx"], it["model_ny"], it["nz"]
        arr[i].window = Window(*[int(v) for v in it["window"]])
        arr[i].source = Point(*[float(v) for v in it["source"]])
        arr[i].T = it.get("T") or None
    return arr


class Net:
    """The traveltime surrogate (tomo_net): 3D U-Net trained and run on the device."""

    def __init__(self, device=0, seed=0, stream=None):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.tomo_net_create(device, ctypes.c_void_p(stream) if stream else None, seed, ctypes.byref(h))
        if rc != TOMO_OK:
            raise TomoError(rc, self.lib.tomo_status_string(rc).decode())
        self.h = h
        self.n_params = int(self.lib.tomo_net_param_count(self.h))

    def _check(self, rc):
        if rc != TOMO_OK:
            raise TomoError(rc, self.lib.tomo_net_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.tomo_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        out = np.empty(self.n_params, np.float32)
        self._check(self.lib.tomo_net_get_params(self.h, out.ctypes.data))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        self._check(self.lib.tomo_net_set_params(self.h, p.ctypes.data))

    def gradients(self, samples, h):
        arr = net_samples(samples)
        loss = ctypes.c_double()
        g = np.empty(self.n_params, np.float32)
        self._check(self.lib.tomo_net_gradients(self.h, len(arr), arr, h, ctypes.byref(loss), g.ctypes.data))
        return loss.value, g

    def train_step(self, samples, h, lr):
        arr = net_samples(samples)
        loss = ctypes.c_double()
        self._check(self.lib.tomo_net_train_step(self.h, len(arr), arr, h, lr, ctypes.byref(loss)))
        return loss.value

    def evaluate(self, samples, h):
        arr = net_samples(samples)
        loss = ctypes.c_double()
        self._check(self.lib.tomo_net_evaluate(self.h, len(arr), arr, h, ctypes.byref(loss)))
        return loss.value

    def predict(self, samples, h, out_ptr, stride=1):
        """Predicted traveltimes into the device array at out_ptr (back-to-back windows);
        stride > 1 runs the network on every stride-th node and interpolates tau back
        (tomo_net_predict_strided).  Returns the device time in ms."""
        arr = net_samples(samples)
        ms = ctypes.c_float()
        self._check(self.lib.tomo_net_predict_strided(self.h, len(arr), arr, h, int(stride), ctypes.c_void_p(out_ptr),
                                                      ctypes.byref(ms)))
        return ms.value
