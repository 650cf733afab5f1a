"""CPU: the C-ABI library builds, loads, and exports every symbol include/*.h declares.
No compute call is made (there is no GPU here)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(tomo_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "tomo_eik_solve" in names and "tomo_ctx_create" in names
    assert len(names) >= 10


def test_library_exports_every_declared_symbol(tomo):
    lib = ctypes.CDLL(tomo.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_no_device_is_a_status_not_a_crash(tomo):
    """Without a GPU, context creation returns TOMO_ERR_NO_DEVICE (no fallback path)."""
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    with pytest.raises(tomo.TomoError) as e:
        tomo.Context(8, 8, 8, 10.0)
    assert e.value.status == -8


def test_status_strings(tomo):
    lib = tomo.load_library()
    for code in range(-9, 1):
        assert lib.tomo_status_string(code)
