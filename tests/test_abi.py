"""CPU checks of the drop-in boundary: the built shared library loads and
exports every entry point include/aerof_gpu.h declares (no GPU call)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "aerof_gpu.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^int\s+(aerof_gpu_\w+)\s*\(", txt, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    from aerof_dev_b200 import build
    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_entry_points():
    names = declared()
    assert "aerof_gpu_residual" in names and "aerof_gpu_gmres" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_lists_every_symbol():
    import aerof_dev_b200 as A
    assert sorted(A.EXPORTS) == declared()


def test_create_without_device_fails_cleanly(lib):
    import aerof_dev_b200 as A
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present: covered by the gpu tests")
    except Exception:
        pass
    with pytest.raises(A.AerofError):
        A.Context()
