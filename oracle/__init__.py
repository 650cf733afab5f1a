"""CPU oracle for the tomography hot path -- TEST INFRASTRUCTURE ONLY.

Two layers, both used only as the checker by ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline / reference legs of ``bench.py``:

* ``liboracle.so`` (``oracle/tomo_oracle.c``): plain-C restatements of the reference
  algorithms (FP64 Jeong-Whitaker fixed point, FP32 receiver trilinear, ray tracing with
  the run-length Jacobian, Tikhonov rows, CGLS, model update, Gaussian smoothing).
* ``oracle/_ref/``: the reference's own solvers compiled unmodified from its sources
  (``oracle/Makefile``) and driven through their public ``Eikonal`` API by
  ``oracle/ref_harness.cpp``.

The product library never imports this package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from contextlib import contextmanager

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(HERE, "_build")
_REF = os.path.join(HERE, "_ref")

RAY_OK, RAY_STALLED, RAY_CAPPED, RAY_NONFINITE, RAY_OUTSIDE, RAY_OVERFLOW = range(6)

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")

_lib = None
_ref_eik = None
_ref_fim = None


def reference_src():
    """Checkout of the reference sources, or None: $TOMO_REFERENCE_SRC, else the checkout
    this container keeps at /root/reference.  The GPU box has neither, and uses the
    prebuilt oracle/_ref files."""
    for cand in (os.environ.get("TOMO_REFERENCE_SRC"), "/root/reference"):
        if cand and os.path.exists(os.path.join(cand, "src", "eikonal", "eikonal.hpp")):
            return cand
    return None


def build() -> None:
    """Compile liboracle.so (and oracle/_ref when the reference sources are present)."""
    ref = reference_src()
    subprocess.run(["make", "-s", "-C", HERE, "-j8"] + ([f"REF={ref}"] if ref else []), check=True)


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(_BUILD, "liboracle.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        c_int, c_float, c_long, c_double = ctypes.c_int, ctypes.c_float, ctypes.c_long, ctypes.c_double
        lib.oracle_fim_jw.argtypes = [c_int, c_int, c_int, c_float, c_float, c_float, _f32p,
                                      c_float, c_float, c_float, _f64p, c_int, c_double]
        lib.oracle_fim_jw.restype = c_int
        lib.oracle_fsm_ngb.argtypes = [c_int, c_int, c_int, c_float, c_float, c_float, _f32p,
                                       c_float, c_float, c_float, _f32p, c_int]
        lib.oracle_fsm_ngb.restype = c_int
        lib.oracle_first_arrival.argtypes = [c_int, c_int, c_int, c_float, c_float, c_float, _f32p,
                                             c_int, _f32p, _f32p, _f32p, _f32p]
        lib.oracle_first_arrival.restype = None
        lib.oracle_raytrace.argtypes = [c_int, c_int, c_int, c_float, c_float, c_float, _f32p,
                                        c_float, c_float, c_float, c_int, _f32p, _f32p, _f32p,
                                        c_float, c_float, c_float, c_int, c_int, c_int, c_int,
                                        c_long, _i64p, _i32p, _f32p, _i32p, _i32p,
                                        ctypes.c_void_p]
        lib.oracle_raytrace.restype = c_long
        lib.oracle_tk_coeffs.argtypes = [c_int, _i32p]
        lib.oracle_tk_coeffs.restype = None
        lib.oracle_cgls_f64.argtypes = [c_int, c_int, c_long, _i32p, _i32p, _f32p, _f32p, c_int,
                                        _f64p, _f64p]
        lib.oracle_cgls_f64.restype = None
        lib.oracle_cgls_f32.argtypes = [c_int, c_int, c_long, _i32p, _i32p, _f32p, _f32p, c_int, _f32p]
        lib.oracle_cgls_f32.restype = None
        lib.oracle_gaussian.argtypes = [_f32p, _f32p, c_int, c_int, c_int, c_int, c_float]
        lib.oracle_gaussian.restype = None
        lib.oracle_model_update.argtypes = [c_int, c_int, c_int, c_float, c_float, c_float,
                                            c_float, c_float, c_float, c_int, c_int, c_int, _f32p,
                                            c_int, c_int, c_float, _f32p, _f32p]
        lib.oracle_model_update.restype = None
        _lib = lib
    return _lib


def _vol(a):
    """(ny, nx, nz) C-order array == z-fastest flat layout of the reference."""
    return np.ascontiguousarray(a, dtype=np.float32)


def fim_jw(slowness, h, src, max_passes=200, tol=1e-10):
    """FP64 fixed point of the Block_FIM operator.  slowness: (ny, nx, nz) float32,
    src = (sx, sy, sz) metres.  Returns (T float64 (ny,nx,nz), passes)."""
    lib = _load()
    s = _vol(slowness)
    ny, nx, nz = s.shape
    dx, dy, dz = (h, h, h) if np.isscalar(h) else h
    out = np.empty_like(s, dtype=np.float64)
    rc = lib.oracle_fim_jw(nx, ny, nz, dx, dy, dz, s.ravel(), src[0], src[1], src[2],
                           out.ravel(), max_passes, tol)
    if rc < 0:
        raise ValueError(f"oracle_fim_jw failed ({rc})")
    return out, rc


def fsm_ngb(slowness, h, src, extra_full_sweeps=0):
    """Noble-Gesret-Belayouni FSM restated (FP32).  extra_full_sweeps=0 reproduces the
    reference's 16 sweeps; -1 sweeps on to the fixed point.  Returns (T, extra passes)."""
    lib = _load()
    s = _vol(slowness)
    ny, nx, nz = s.shape
    dx, dy, dz = (h, h, h) if np.isscalar(h) else h
    out = np.empty_like(s)
    extra = lib.oracle_fsm_ngb(nx, ny, nz, dx, dy, dz, s.ravel(), src[0], src[1], src[2], out.ravel(),
                               extra_full_sweeps)
    return out, extra


def first_arrival(T, h, rx, ry, rz):
    lib = _load()
    t = _vol(T)
    ny, nx, nz = t.shape
    dx, dy, dz = (h, h, h) if np.isscalar(h) else h
    rx, ry, rz = (np.ascontiguousarray(v, np.float32) for v in (rx, ry, rz))
    out = np.empty(len(rx), np.float32)
    lib.oracle_first_arrival(nx, ny, nz, dx, dy, dz, t.ravel(), len(rx), rx, ry, rz, out)
    return out


def raytrace(T, h, src, rx, ry, rz, d_tomo, n_tomo, max_steps=20000, illum=False, cap=None):
    """Ray tracing of one shot.  Returns dict(row_ptr, cols, vals, status, steps, illum)."""
    lib = _load()
    t = _vol(T)
    ny, nx, nz = t.shape
    dx, dy, dz = (h, h, h) if np.isscalar(h) else h
    rx, ry, rz = (np.ascontiguousarray(v, np.float32) for v in (rx, ry, rz))
    nrec = len(rx)
    cap = cap or nrec * 512
    row_ptr = np.zeros(nrec + 1, np.int64)
    cols = np.zeros(cap, np.int32)
    vals = np.zeros(cap, np.float32)
    status = np.zeros(nrec, np.int32)
    steps = np.zeros(nrec, np.int32)
    il = np.zeros_like(t) if illum else None
    nnz = lib.oracle_raytrace(nx, ny, nz, dx, dy, dz, t.ravel(), src[0], src[1], src[2], nrec,
                              rx, ry, rz, d_tomo[0], d_tomo[1], d_tomo[2], n_tomo[0], n_tomo[1],
                              n_tomo[2], max_steps, cap, row_ptr, cols, vals, status, steps,
                              il.ctypes.data if il is not None else None)
    if nnz < 0:
        raise ValueError("oracle_raytrace: capacity exceeded")
    return dict(row_ptr=row_ptr, cols=cols[:nnz].copy(), vals=vals[:nnz].copy(), status=status,
                steps=steps, illum=il)


def tk_coeffs(order):
    df = np.zeros(order + 1, np.int32)
    _load().oracle_tk_coeffs(order, df)
    return df


def cgls_f64(N, M, iA, jA, vA, B, nit):
    x = np.zeros(M, np.float64)
    hist = np.zeros(max(nit, 1), np.float64)
    _load().oracle_cgls_f64(N, M, len(vA), np.ascontiguousarray(iA, np.int32),
                            np.ascontiguousarray(jA, np.int32), np.ascontiguousarray(vA, np.float32),
                            np.ascontiguousarray(B, np.float32), nit, x, hist)
    return x, hist[:nit]


def cgls_f32(N, M, iA, jA, vA, B, nit):
    x = np.zeros(M, np.float32)
    _load().oracle_cgls_f32(N, M, len(vA), np.ascontiguousarray(iA, np.int32),
                            np.ascontiguousarray(jA, np.int32), np.ascontiguousarray(vA, np.float32),
                            np.ascontiguousarray(B, np.float32), nit, x)
    return x


def gaussian(vol, samples, stdv):
    v = _vol(vol)
    ny, nx, nz = v.shape
    out = np.empty_like(v)
    _load().oracle_gaussian(v.ravel(), out.ravel(), nx, ny, nz, samples, stdv)
    return out


def model_update(slowness, h, d_tomo, n_tomo, xdm, smooth=True, samples=5, stdv=2.0):
    """Returns (new_slowness, velocity)."""
    s = _vol(slowness).copy()
    ny, nx, nz = s.shape
    dx, dy, dz = (h, h, h) if np.isscalar(h) else h
    vel = np.empty_like(s)
    _load().oracle_model_update(nx, ny, nz, dx, dy, dz, d_tomo[0], d_tomo[1], d_tomo[2],
                                n_tomo[0], n_tomo[1], n_tomo[2],
                                np.ascontiguousarray(xdm, np.float32), int(smooth), samples, stdv,
                                s.ravel(), vel.ravel())
    return s, vel


# ----------------------------------------------------------------------------------------
# The reference's own solvers (oracle/_ref)
# ----------------------------------------------------------------------------------------
@contextmanager
def quiet_stdout():
    """The reference prints progress to stdout; keep it off the caller's stdout."""
    fd = os.dup(1)
    try:
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        os.close(devnull)
        yield
    finally:
        os.dup2(fd, 1)
        os.close(fd)


def have_ref(gpu=False):
    return os.path.exists(os.path.join(_REF, "libref_fim.so" if gpu else "libref_eik.so"))


def _load_ref(gpu=False):
    global _ref_eik, _ref_fim
    if gpu:
        if _ref_fim is None:
            _ref_fim = ctypes.CDLL(os.path.join(_REF, "libref_fim.so"))
            _setup_ref(_ref_fim)
        return _ref_fim
    if _ref_eik is None:
        _ref_eik = ctypes.CDLL(os.path.join(_REF, "libref_eik.so"))
        _setup_ref(_ref_eik)
    return _ref_eik


def _setup_ref(lib):
    c_int, c_float = ctypes.c_int, ctypes.c_float
    lib.ref_eikonal_solve.argtypes = [c_int, ctypes.c_char_p, c_int, c_int, c_int, c_float,
                                      c_float, c_float, _f32p, c_int, _f32p, _f32p, _f32p,
                                      ctypes.c_void_p, _f64p, c_int]
    lib.ref_eikonal_solve.restype = c_int


REF_CLASSIC, REF_BLOCK_FIM, REF_FSM = 0, 1, 2


def ref_solve(kind, velocity, h, shots, nthreads=1, want_T=True):
    """Run the reference solver `kind` (REF_FSM, REF_CLASSIC, REF_BLOCK_FIM) on the
    velocity model (ny, nx, nz) for shots [(sx, sy, sz), ...].
    Returns (T (nshots, ny, nx, nz) float32 or None, per-shot solve seconds)."""
    lib = _load_ref(gpu=(kind == REF_BLOCK_FIM))
    v = _vol(velocity)
    ny, nx, nz = v.shape
    dx, dy, dz = (h, h, h) if np.isscalar(h) else h
    shots = np.asarray(shots, np.float32).reshape(-1, 3)
    ns = len(shots)
    T = np.empty((ns, ny, nx, nz), np.float32) if want_T else None
    secs = np.zeros(ns, np.float64)
    with tempfile.TemporaryDirectory() as d, quiet_stdout():
        rc = lib.ref_eikonal_solve(kind, d.encode(), nx, ny, nz, dx, dy, dz, v.ravel(), ns,
                                   np.ascontiguousarray(shots[:, 0]),
                                   np.ascontiguousarray(shots[:, 1]),
                                   np.ascontiguousarray(shots[:, 2]),
                                   T.ctypes.data if T is not None else None, secs, nthreads)
    if rc != 0:
        raise RuntimeError(f"ref_eikonal_solve failed ({rc})")
    return T, secs


def ref_tomography_exe():
    return os.path.join(_REF, "tomography.exe")


def ref_catch_parameter(key, param_file):
    """The reference's own catch_parameter (src/utils/file_manager/file_manager.cpp:74-120)."""
    lib = _load_ref()
    lib.ref_catch_parameter.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
    buf = ctypes.create_string_buffer(4096)
    n = lib.ref_catch_parameter(key.encode(), param_file.encode(), buf, len(buf))
    if n < 0:
        raise ValueError("value too long")
    return buf.raw[:n].decode("latin-1")


def ref_geometry(param_file, name, gtype, cap=100000):
    """The reference's own Regular (0) / Circular (1) set_geometry; returns (n, 3) float32."""
    lib = _load_ref()
    lib.ref_geometry.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    out = np.zeros((cap, 3), np.float32)
    with quiet_stdout():
        n = lib.ref_geometry(param_file.encode(), name.encode(), gtype, out.ctypes.data, cap)
    return out[:n].copy()
