"""The residual entry point that allocates nothing.

Some callers cannot allocate device memory once they run: an application
that has given all of the GPU's memory to its own pool, or a thread that must
not take the device allocator's locks.  aerof_gpu_residual_noalloc serves
them with a fixed scratch array inside the library.  This test calls it
through the C ABI twice in a row and checks both results against
aerof_gpu_residual (relative L2 <= 1e-12, the residual parity tolerance);
it also checks that a mesh beyond the array's limit is refused.  Collected
last so that a failure here never hides another test's result."""
import ctypes as C

import numpy as np
import pytest

from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rec", [2, 1])
def test_noalloc_matches_residual_twice(gpu_lib, rec):
    import torch
    A = gpu_lib
    m = W.make_lattice_mesh(15, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    ctx = A.Context.from_mesh(m, Ub, reconstruction=rec)
    U = torch.from_numpy(W.perturbed_state(ctx.N, 0.8)).cuda()
    R_ref = torch.empty_like(U)
    bad_ref = ctx._check(ctx.L.aerof_gpu_residual(ctx.h, C.c_void_p(U.data_ptr()), C.c_void_p(R_ref.data_ptr())))
    for _ in range(2):
        R = torch.full_like(U, float("nan"))
        bad = ctx._check(ctx.L.aerof_gpu_residual_noalloc(ctx.h, C.c_void_p(U.data_ptr()),
                                                          C.c_void_p(R.data_ptr())))
        assert bad == bad_ref == 0
        assert rel_l2(R.cpu().numpy(), R_ref.cpu().numpy()) <= 1e-12


def test_noalloc_rejects_large_mesh_and_host_arrays(gpu_lib):
    import torch
    A = gpu_lib
    m = W.make_lattice_mesh(41, codes="channel")   # 68,921 nodes: beyond the fixed scratch
    ctx = A.Context.from_mesh(m, W.freestream(0.8))
    U = torch.zeros((ctx.N, 5), dtype=torch.float64, device="cuda")
    R = torch.empty_like(U)
    rc = ctx.L.aerof_gpu_residual_noalloc(ctx.h, C.c_void_p(U.data_ptr()), C.c_void_p(R.data_ptr()))
    assert rc == -1
    buf = C.create_string_buffer(512)
    ctx.L.aerof_gpu_last_error(ctx.h, buf, 512)
    assert b"too large" in buf.value
    small = A.Context.from_mesh(W.make_lattice_mesh(5), W.freestream(0.5))
    Uh = np.zeros((small.N, 5))
    Rh = np.zeros((small.N, 5))
    rc = small.L.aerof_gpu_residual_noalloc(small.h, C.c_void_p(Uh.ctypes.data), C.c_void_p(Rh.ctypes.data))
    assert rc == -1
