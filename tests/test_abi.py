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
    return sorted(set(re.findall(r"^int\s+(aerof_(?:gpu|sower)_\w+)\s*\(", txt, flags=re.M)))


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


CALLER = r"""
/* a C99 caller of the ABI: compiles against the header alone, links the
   library, and exercises calls that need no device (argument checks, the
   launch counter); with a device it creates and destroys a context */
#include <stdio.h>
#include <string.h>
#include "aerof_gpu.h"

int main(void) {
  long long launches = -1;
  if (aerof_gpu_launch_count(&launches) != AEROF_OK || launches < 0) return 1;
  if (aerof_gpu_launch_count(NULL) != AEROF_EINVAL) return 2;
  if (aerof_gpu_residual(NULL, NULL, NULL) != AEROF_EINVAL) return 3;
  aerof_gpu_config cfg;
  memset(&cfg, 0, sizeof cfg);
  cfg.gamma = 1.4;
  cfg.beta = 1.0 / 3.0;
  cfg.reconstruction = AEROF_REC_VANALBADA;
  cfg.reconstruction = 99;                       /* invalid: refused before any CUDA call */
  aerof_gpu_ctx* ctx = NULL;
  if (aerof_gpu_create(&cfg, &ctx) != AEROF_EINVAL || ctx != NULL) return 4;
  cfg.reconstruction = AEROF_REC_VANALBADA;
  int rc = aerof_gpu_create(&cfg, &ctx);
  if (rc == AEROF_OK) {
    aerof_newton_result res;
    memset(&res, 0, sizeof res);
    if (aerof_gpu_newton(ctx, NULL, NULL, &res, NULL) != AEROF_EINVAL) return 5;
    aerof_gpu_destroy(ctx);
  } else if (rc != AEROF_ECUDA) {
    return 6;
  }
  printf("ok %d\n", rc);
  return 0;
}
"""


def test_c_caller_compiles_links_and_runs(lib, tmp_path):
    import subprocess
    src = tmp_path / "caller.c"
    src.write_text(CALLER)
    exe = tmp_path / "caller"
    libdir = os.path.join(ROOT, "aerof_dev_b200")
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                           str(src), "-L", libdir, "-laerof_gpu", f"-Wl,-rpath,{libdir}", "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert out.stdout.startswith("ok")
