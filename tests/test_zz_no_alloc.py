"""The residual entry point that allocates nothing.

Some callers cannot allocate device memory once they run: an application
that has given all of the GPU's memory to its own pool, or a thread that must
not take the device allocator's locks.  aerof_gpu_residual_noalloc serves
them with a fixed scratch array inside the library, claimed when the context
is created.  These tests call it through the C ABI twice in a row and check
both results against aerof_gpu_residual (relative L2 <= 1e-12, the residual
parity tolerance), on a mesh with an odd edge count (the scratch parts must
stay 16-byte aligned), on a fresh context whose first residual call is the
allocation-free one, on the failsafe path (tags left in the shared array by
one call must not leak into the next), and with almost no free device
memory.  A mesh beyond the array's limit and host arrays are refused.
Collected last so that a failure here never hides another test's result;
each test also passes when run alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _noalloc(ctx, U, R):
    return ctx._check(ctx.L.aerof_gpu_residual_noalloc(ctx.h, _ptr(U), _ptr(R)))


def _residual(ctx, U, R):
    return ctx._check(ctx.L.aerof_gpu_residual(ctx.h, _ptr(U), _ptr(R)))


@pytest.mark.parametrize("n", [15, 14])   # 14^3: odd edge count (16,939)
@pytest.mark.parametrize("rec", [2, 1])
def test_noalloc_first_call_then_matches_residual(gpu_lib, n, rec):
    import torch
    A = gpu_lib
    m = W.make_lattice_mesh(n, jitter=0.2, codes="channel")
    if n == 14:
        assert W.lattice_sizes(n)["E"] % 2 == 1
    ctx = A.Context.from_mesh(m, W.freestream(0.8), reconstruction=rec)
    U = torch.from_numpy(W.perturbed_state(ctx.N, 0.8)).cuda()
    # the allocation-free call comes first on this context, twice
    outs = []
    for _ in range(2):
        R = torch.full_like(U, float("nan"))
        outs.append((_noalloc(ctx, U, R), R))
    R_ref = torch.empty_like(U)
    bad_ref = _residual(ctx, U, R_ref)
    for bad, R in outs:
        assert bad == bad_ref == 0
        assert rel_l2(R.cpu().numpy(), R_ref.cpu().numpy()) <= TOL


def test_noalloc_failsafe_path_twice(gpu_lib, oracle_mod):
    # unlimited MUSCL next to a pressure spike: some reconstructed pressures
    # go negative, the failsafe re-run zeroes those nodes' gradients
    import torch
    A = gpu_lib
    m = W.make_lattice_mesh(7, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    U0 = W.perturbed_state(7 ** 3, 0.8)
    V = oracle_mod.Oracle(m).prim(U0)
    i = 3 * 49 + 3 * 7 + 3
    V[i, 4] *= 40.0
    V[i + 1, 4] *= 0.02
    Ubad = torch.from_numpy(W.prim_to_cons(V)).cuda()
    Ugood = torch.from_numpy(U0).cuda()
    ctx = A.Context.from_mesh(m, Ub, reconstruction=3, failsafe=1)
    R_ref = torch.empty_like(Ubad)
    bad_ref = _residual(ctx, Ubad, R_ref)
    assert bad_ref > 0
    for _ in range(2):
        R = torch.full_like(Ubad, float("nan"))
        assert _noalloc(ctx, Ubad, R) == bad_ref
        assert rel_l2(R.cpu().numpy(), R_ref.cpu().numpy()) <= TOL
    # a healthy state after the failsafe calls: no tag survives in the array
    R_ref2 = torch.empty_like(Ugood)
    assert _residual(ctx, Ugood, R_ref2) == 0
    R = torch.full_like(Ugood, float("nan"))
    assert _noalloc(ctx, Ugood, R) == 0
    assert rel_l2(R.cpu().numpy(), R_ref2.cpu().numpy()) <= TOL


def test_noalloc_with_device_memory_exhausted(gpu_lib):
    # the caller's own pool takes (almost) all free device memory after the
    # context is set up; the allocation-free call must still run, twice
    import torch
    A = gpu_lib
    m = W.make_lattice_mesh(15, jitter=0.2, codes="channel")
    ctx = A.Context.from_mesh(m, W.freestream(0.8), reconstruction=2)
    U = torch.from_numpy(W.perturbed_state(ctx.N, 0.8)).cuda()
    R_ref = torch.empty_like(U)
    R = [torch.full_like(U, float("nan")) for _ in range(2)]
    _residual(ctx, U, R_ref)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    hog = []
    margin = 8 << 20
    try:
        for _ in range(64):
            free, _total = torch.cuda.mem_get_info()
            if free <= 2 * margin:
                break
            try:
                hog.append(torch.empty(free - margin, dtype=torch.uint8, device="cuda"))
            except torch.OutOfMemoryError:
                margin *= 2
        free, _total = torch.cuda.mem_get_info()
        assert free < 64 << 20, f"could not take the device's memory ({free} bytes still free)"
        bads = [_noalloc(ctx, U, r) for r in R]
    finally:
        del hog
        torch.cuda.empty_cache()
    for bad, r in zip(bads, R):
        assert bad == 0
        assert rel_l2(r.cpu().numpy(), R_ref.cpu().numpy()) <= TOL


def test_noalloc_rejects_large_mesh_and_host_arrays(gpu_lib):
    import torch
    A = gpu_lib
    m = W.make_lattice_mesh(41, codes="channel")   # 68,921 nodes: beyond the fixed scratch
    ctx = A.Context.from_mesh(m, W.freestream(0.8))
    U = torch.zeros((ctx.N, 5), dtype=torch.float64, device="cuda")
    R = torch.empty_like(U)
    rc = ctx.L.aerof_gpu_residual_noalloc(ctx.h, _ptr(U), _ptr(R))
    assert rc == -1
    buf = C.create_string_buffer(512)
    ctx.L.aerof_gpu_last_error(ctx.h, buf, 512)
    assert b"too large" in buf.value
    small = A.Context.from_mesh(W.make_lattice_mesh(5), W.freestream(0.5))
    Uh = np.zeros((small.N, 5))
    Rh = np.zeros((small.N, 5))
    rc = small.L.aerof_gpu_residual_noalloc(small.h, C.c_void_p(Uh.ctypes.data), C.c_void_p(Rh.ctypes.data))
    assert rc == -1
