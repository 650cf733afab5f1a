"""CPU: the ctypes mirrors of the C-ABI structs (seismic_tomography_3d_b200/__init__.py) have
the size and field offsets the compiler gives the structs of include/tomo_b200.h, so a field
added on one side only is caught without a GPU."""
import ctypes
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C typedef -> ctypes mirror class name
PAIRS = {
    "tomo_grid": "Grid", "tomo_point": "Point", "tomo_window": "Window",
    "tomo_eik_opts": "EikOpts", "tomo_eik_stats": "EikStats", "tomo_seed_stats": "SeedStats",
    "tomo_tune_stats": "TuneStats", "tomo_jacobian_opts": "JacobianOpts",
    "tomo_jacobian_stats": "JacobianStats", "tomo_cgls_stats": "CglsStats",
    "tomo_update_opts": "UpdateOpts", "tomo_iteration_opts": "IterationOpts",
    "tomo_iteration_stats": "IterationStats", "tomo_net_sample": "NetSample",
}


@pytest.fixture(scope="module")
def c_layouts(tmp_path_factory):
    """Sizes and field offsets of the header's structs, printed by a program gcc builds."""
    import seismic_tomography_3d_b200 as tomo

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "tomo_b200.h"', "int main(void) {"]
    for cname, pyname in PAIRS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in getattr(tomo, pyname)._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0; }")
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for ln in out.splitlines():
        name, key, val = ln.split()
        layout[(name, key)] = int(val)
    return layout


@pytest.mark.parametrize("cname", sorted(PAIRS))
def test_ctypes_mirror_matches_header(c_layouts, cname):
    import seismic_tomography_3d_b200 as tomo

    cls = getattr(tomo, PAIRS[cname])
    assert ctypes.sizeof(cls) == c_layouts[(cname, "size")], f"{cname}: size differs"
    for field, _ in cls._fields_:
        assert getattr(cls, field).offset == c_layouts[(cname, field)], f"{cname}.{field}: offset differs"
