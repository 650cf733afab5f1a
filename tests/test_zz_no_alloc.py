"""tomo_eik_solve_static: the allocation-free single-shot solve.

It serves callers that cannot call cudaMalloc -- an application whose framework already
owns the GPU's memory through its own pool, or a loop with a fixed device-memory budget --
by keeping its working memory in a fixed device array inside the library.  Checked through
the C ABI against the regular entry point (tomo_eik_solve + tomo_eik_volume) on two calls
in a row, with the tolerance the batched-vs-single tests use (1e-5 relative), and for its
size limit.  The device buffers of this test are the caller's (allocated here by torch).
"""
import ctypes

import numpy as np
import pytest

from seismic_tomography_3d_b200 import workloads as wl

pytestmark = pytest.mark.gpu

REL = 1e-5


def _bind(lib):
    f = lib.tomo_eik_solve_static
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                  ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _rel(a, b, h, vmax):
    m = b >= 2.0 * h / vmax
    return float(np.max(np.abs(a[m] - b[m]) / b[m]))


def test_static_solve_matches_regular_entry_point(tomo):
    import torch

    lib = tomo.load_library()
    solve_static = _bind(lib)
    stream = torch.cuda.current_stream()
    # two calls in a row; the second is smaller, so stale contents of the shared array
    # from the first call would show up in it
    for seed, dims in ((21, (45, 38, 27)), (22, (19, 23, 13))):
        nx, ny, nz = dims
        sv = wl.small(seed, nx, ny, nz, nshots=1)
        sx, sy, sz = map(float, sv.shots[0])
        slow = (1.0 / sv.velocity).astype(np.float32)
        d_slow = torch.from_numpy(slow).cuda()
        d_out = torch.full_like(d_slow, -1.0)
        torch.cuda.synchronize()
        rc = solve_static(d_slow.data_ptr(), nx, ny, nz, sv.h, sv.h, sv.h, sx, sy, sz, d_out.data_ptr(),
                          stream.cuda_stream)
        assert rc == 0, lib.tomo_last_error(None)
        T_static = d_out.cpu().numpy()
        with tomo.Context(nx, ny, nz, sv.h) as ctx:
            ctx.set_slowness(slow)
            ctx.eik_solve(sv.shots)
            T_ref = ctx.eik_volume(0)
        assert T_static.shape == T_ref.shape
        assert np.all(T_static > 0.0) or np.count_nonzero(T_static == 0.0) == 1
        assert _rel(T_static, T_ref, sv.h, sv.velocity.max()) < REL


def test_static_solve_rejects_oversized_grid(tomo):
    import torch

    lib = tomo.load_library()
    solve_static = _bind(lib)
    dummy = torch.zeros(1, device="cuda")
    # 164 x 164 x 164 pads to 4,410,944 nodes > 4,194,304
    rc = solve_static(dummy.data_ptr(), 164, 164, 164, 10.0, 10.0, 10.0, 5.0, 5.0, 0.0, dummy.data_ptr(), None)
    assert rc == -9  # TOMO_ERR_CAPACITY
    assert b"exceeds" in lib.tomo_last_error(None)
    # sizes whose padded product wraps around 2^64 (4194304^2 x 1048576 = 2^64), and one
    # axis beyond the limit on its own: rejected before any product is formed
    for dims in ((4194304, 4194304, 1048576), (1 << 30, 2, 2), (2, 2, 2147483647)):
        rc = solve_static(dummy.data_ptr(), *dims, 10.0, 10.0, 10.0, 5.0, 5.0, 0.0, dummy.data_ptr(), None)
        assert rc == -9, dims
