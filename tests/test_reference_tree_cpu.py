"""CPU: the plug-in classes (seismic_tomography_3d_b200/host/eikonal_b200.cpp,
least_squares_b200.cpp) compile against the reference's own headers
(src/eikonal/eikonal.hpp:15-58, src/tomography/tomography.hpp:11-56) with
-DTOMO_B200_REFERENCE_TREE, as they do when copied into the reference tree.

The sources are compiled where they lie: their `#include "../eikonal.hpp"` and
`"../tomography.hpp"` resolve through -iquote directories one level below the reference's
src/eikonal and src/tomography.  Needs the reference checkout (this container); skipped
where it is absent.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "seismic_tomography_3d_b200", "host")


def _ref_src():
    import oracle

    ref = oracle.reference_src()
    if ref is None:
        pytest.skip("reference sources not present")
    return os.path.join(ref, "src")


@pytest.mark.parametrize("source", ["eikonal_b200.cpp", "least_squares_b200.cpp"])
def test_plugin_compiles_in_reference_tree(source):
    src = _ref_src()
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    cmd = [cxx, "-std=c++17", "-fsyntax-only", "-Wall", "-DTOMO_B200_REFERENCE_TREE",
           "-iquote", os.path.join(src, "eikonal", "accurate_FSM"),
           "-iquote", os.path.join(src, "tomography", "least_squares"),
           "-I", os.path.join(ROOT, "include"), "-I", HOST, os.path.join(HOST, source)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    # the classes really bound to the reference's declarations, not to the mirror
    pp = subprocess.run(cmd[:2] + ["-E"] + cmd[4:], capture_output=True, text=True, check=True).stdout
    assert os.path.join(src, "eikonal", "eikonal.hpp") in pp or "eikonal/accurate_FSM/../eikonal.hpp" in pp
    assert "tomo_b200_interface.hpp" not in pp
