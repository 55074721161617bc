"""GPU parity of the residual path against the CPU oracle (all through the
C ABI of libaerof_gpu.so).  Tolerances: relative L2 <= 1e-12 for FP64
residual/gradient/geometry, bit-exact for the integer edge list."""
import numpy as np
import pytest

from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module", params=[("channel", 9, 0.2), ("farfield", 6, 0.0)])
def case(request, gpu_lib, oracle_mod):
    codes, n, jit = request.param
    m = W.make_lattice_mesh(n, jitter=jit, codes=codes)
    Ub = W.freestream(0.8 if codes == "channel" else 0.5)
    o = oracle_mod.Oracle(m)
    return m, Ub, o


KERNELS = [0, 1]  # blocked, edge


def ctx_for(A, m, Ub, rec=2, failsafe=0, kernel=0):
    return A.Context.from_mesh(m, Ub, reconstruction=rec, failsafe=failsafe, residual_kernel=kernel)


def test_edges_bit_exact(gpu_lib, case):
    m, Ub, o = case
    ctx = ctx_for(gpu_lib, m, Ub)
    assert ctx.E == o.E
    assert np.array_equal(ctx.edges(), o.edges())


def test_geometry_parity(gpu_lib, case):
    m, Ub, o = case
    g = ctx_for(gpu_lib, m, Ub).geometry()
    r = o.geometry()
    for k in ("edge_normal", "face_normal", "ctrl_vol", "lsq_R"):
        assert rel_l2(g[k], r[k]) < TOL, k


def test_gradients_parity(gpu_lib, case):
    m, Ub, o = case
    ctx = ctx_for(gpu_lib, m, Ub)
    U = W.perturbed_state(o.N, 0.8)
    V = o.prim(U)
    got = gpu_lib.SpaceOperator(ctx).computeGradients(V)
    ref = o.gradients(V)
    for a, b in zip(got, ref):
        assert rel_l2(a, b) < TOL


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("rec", [1, 2, 3])
def test_residual_parity(gpu_lib, case, rec, kernel):
    m, Ub, o = case
    ctx = ctx_for(gpu_lib, m, Ub, rec=rec, kernel=kernel)
    U = W.perturbed_state(o.N, 0.8)
    R, bad = gpu_lib.SpaceOperator(ctx).computeResidual(U)
    Rr, badr = o.residual(U, Ub, rec)
    assert bad == badr == 0
    assert rel_l2(R, Rr) < TOL


@pytest.mark.parametrize("kernel", KERNELS)
def test_residual_device_pointers_and_determinism(gpu_lib, case, kernel):
    import torch
    m, Ub, o = case
    ctx = ctx_for(gpu_lib, m, Ub, kernel=kernel)
    U = W.perturbed_state(o.N, 0.8)
    Ut = torch.from_numpy(U).cuda()
    sp = gpu_lib.SpaceOperator(ctx)
    R1, _ = sp.computeResidual(Ut)
    R2, _ = sp.computeResidual(Ut)
    assert R1.is_cuda
    assert torch.equal(R1, R2)  # bitwise run-to-run
    Rh, _ = sp.computeResidual(U)
    assert np.array_equal(R1.cpu().numpy(), Rh)


@pytest.mark.parametrize("kernel", KERNELS)
def test_freestream_preserved_gpu(gpu_lib, case, kernel):
    m, Ub, o = case
    ctx = ctx_for(gpu_lib, m, Ub, kernel=kernel)
    U = np.tile(Ub, (o.N, 1))
    R, bad = gpu_lib.SpaceOperator(ctx).computeResidual(U)
    assert bad == 0 and np.abs(R).max() < 1e-11


def test_timestep_parity(gpu_lib, case):
    m, Ub, o = case
    ctx = ctx_for(gpu_lib, m, Ub)
    U = W.perturbed_state(o.N, 0.8)
    dt = gpu_lib.SpaceOperator(ctx).computeTimeStep(U, 0.8)
    assert rel_l2(dt, o.timestep(U, 0.8)) < TOL


@pytest.mark.parametrize("kernel", KERNELS)
def test_rk2_parity(gpu_lib, oracle_mod, kernel):
    # CPU-runnable case: first order, far field, Mach 0.5, 10 RK2 steps, CFL 0.8
    m = W.make_lattice_mesh(11, codes="farfield")
    Ub = W.freestream(0.5)
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.5)
    ctx = ctx_for(gpu_lib, m, Ub, rec=1, kernel=kernel)
    Ug, bad = gpu_lib.ExplicitRK2(ctx, 0.8).run(U, 10)
    Ur = o.rk2(U, Ub, 1, 0.8, 10)
    assert bad == 0
    assert rel_l2(Ug, Ur) < TOL
    assert rel_l2(Ug - U, Ur - U) < 1e-10


@pytest.mark.parametrize("kernel", KERNELS)
def test_unphysical_state_counted_and_failsafe(gpu_lib, oracle_mod, kernel):
    m = W.make_lattice_mesh(7, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.8)
    # a pressure spike next to a near-vacuum node makes the unlimited MUSCL
    # extrapolation negative (linear reconstruction)
    V = o.prim(U)
    i = 3 * 49 + 3 * 7 + 3
    V[i, 4] *= 40.0
    V[i + 1, 4] *= 0.02
    U = W.prim_to_cons(V)
    _, bad_ref = o.residual(U, Ub, 3)
    assert bad_ref > 0
    ctx = ctx_for(gpu_lib, m, Ub, rec=3, kernel=kernel)
    _, bad = gpu_lib.SpaceOperator(ctx).computeResidual(U)
    assert bad == bad_ref
    # failsafe: tagged nodes fall back to zero gradients, result matches oracle
    ctx = ctx_for(gpu_lib, m, Ub, rec=3, failsafe=1, kernel=kernel)
    R, bad = gpu_lib.SpaceOperator(ctx).computeResidual(U)
    Rr, bad_r = o.residual(U, Ub, 3, failsafe=1)
    assert bad == bad_r
    assert rel_l2(R, Rr) < TOL


def test_bad_arguments_rejected(gpu_lib):
    A = gpu_lib
    ctx = A.Context()
    with pytest.raises(A.AerofError) as e:
        A.SpaceOperator(ctx).computeResidual(np.zeros((1, 5)))
    assert e.value.code == -6  # ESTATE: no mesh
    m = W.make_lattice_mesh(3)
    bad_tets = m["tets"].copy()
    bad_tets[0, 0] = 10 ** 6
    with pytest.raises(A.AerofError) as e:
        ctx.set_mesh(m["X"], bad_tets, m["faces"], m["codes"], W.freestream(0.5))
    assert e.value.code == -1


def test_blocked_numbering_is_a_permutation(gpu_lib, case):
    # the Morton renumbering must not change the result beyond rounding:
    # both organisations agree with each other as closely as with the oracle
    m, Ub, o = case
    U = W.perturbed_state(o.N, 0.8)
    Rb, _ = gpu_lib.SpaceOperator(ctx_for(gpu_lib, m, Ub, kernel=0)).computeResidual(U)
    Re, _ = gpu_lib.SpaceOperator(ctx_for(gpu_lib, m, Ub, kernel=1)).computeResidual(U)
    assert rel_l2(Rb, Re) < 1e-13


@pytest.mark.parametrize("nb", ["64", "256"])
def test_block_sizes(gpu_lib, oracle_mod, monkeypatch, nb):
    # the staged gradient kernel runs 4, 2 or 1 lanes per node depending on
    # the block size; every block size gives the oracle's residual, also on
    # the failsafe path that recomputes tagged gradients
    monkeypatch.setenv("AEROF_BLOCK_NODES", nb)
    m = W.make_lattice_mesh(13, jitter=0.25, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.8)
    for rec in (2, 3):
        R, bad = gpu_lib.SpaceOperator(ctx_for(gpu_lib, m, Ub, rec=rec)).computeResidual(U)
        Rr, badr = o.residual(U, Ub, rec)
        assert bad == badr == 0
        assert rel_l2(R, Rr) < TOL
    V = o.prim(U)
    i = 5 * 169 + 5 * 13 + 5
    V[i, 4] *= 40.0
    V[i + 1, 4] *= 0.02
    U2 = W.prim_to_cons(V)
    R, bad = gpu_lib.SpaceOperator(ctx_for(gpu_lib, m, Ub, rec=3, failsafe=1)).computeResidual(U2)
    Rr, badr = o.residual(U2, Ub, 3, failsafe=1)
    assert bad == badr > 0
    assert rel_l2(R, Rr) < TOL


def test_launch_count(gpu_lib, case):
    m, Ub, o = case
    ctx = ctx_for(gpu_lib, m, Ub)
    U = W.perturbed_state(o.N, 0.8)
    sp = gpu_lib.SpaceOperator(ctx)
    sp.computeResidual(U)
    gpu_lib.launch_count()
    sp.computeResidual(U)
    n = gpu_lib.launch_count()
    assert 3 <= n <= 6


@pytest.mark.parametrize("rec", [1, 2])
def test_host_array_residual_overlapped_copies(gpu_lib, oracle_mod, rec):
    # page-locked host U and R on a mesh large enough for the overlapped
    # copies (chunks of U in, stages of blocks computed as their rows
    # arrive, chunks of R out): the same residual, bit for bit, as the
    # device-array call, and the oracle's to 1e-12
    import torch
    m = W.make_lattice_mesh(51, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    ctx = ctx_for(gpu_lib, m, Ub, rec=rec)
    assert ctx.N >= 1 << 17
    sp = gpu_lib.SpaceOperator(ctx)
    U = W.perturbed_state(ctx.N, 0.8)
    Ud = torch.from_numpy(U).cuda()
    Rd, bad_d = sp.computeResidual(Ud)
    Uh = torch.from_numpy(U).pin_memory()
    Rh = torch.empty_like(Uh).pin_memory()
    # new output arrays, then the same ones again (the stages' recorded
    # kernels replayed with other copies around them)
    for k in range(4):
        if k < 2:
            Rh = torch.empty_like(Uh).pin_memory()
        Rh.fill_(float("nan"))
        _, bad_h = sp.computeResidual(Uh, Rh)
        assert bad_h == bad_d == 0
        assert torch.equal(Rh, Rd.cpu())
    o = oracle_mod.Oracle(m)
    Rr, _ = o.residual(U, Ub, rec)
    assert rel_l2(Rh.numpy(), Rr) < TOL
