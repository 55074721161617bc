"""GPU block ILU(0) preconditioner (IluPrec in the multicolour ordering)
against the oracle's restatement, and its effect on GMRES and Newton."""
import numpy as np
import pytest

from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(gpu_lib, oracle_mod):
    m = W.make_lattice_mesh(9, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.8)
    dt = o.timestep(U, 100.0)
    return m, Ub, o, U, dt


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("trans", [False, True])
def test_ilu_parity(gpu_lib, setup, prec, trans):
    m, Ub, o, U, dt = setup
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    ctx.set_preconditioner(gpu_lib.PC_ILU0)
    mv = gpu_lib.MatVecProdH1(ctx, prec)
    mv.evaluate(U, dt)
    pc = gpu_lib.JacobiPrec(ctx)
    pc.setup()
    x = np.random.default_rng(3).standard_normal((o.N, 5))
    z = pc.apply(x, transpose=trans)
    zr, bad, nc, _ = o.ilu0(mv.blocks(), x, fp32=(prec == 32), transpose=trans)
    assert bad == 0 and nc > 1
    # FP64: summation order only; FP32: blocks rounded to float after every
    # update on both sides, rounding-boundary cases differ
    assert rel_l2(z, zr) < (1e-12 if prec == 64 else 1e-5)


@pytest.mark.parametrize("prec", [64, 32])
def test_gmres_with_ilu(gpu_lib, setup, prec):
    m, Ub, o, U, dt = setup
    R, _ = o.residual(U, Ub, 2)
    its = {}
    for pcname in ("bj", "ilu"):
        ctx = gpu_lib.Context.from_mesh(m, Ub)
        if pcname == "ilu":
            ctx.set_preconditioner(gpu_lib.PC_ILU0)
        mv = gpu_lib.MatVecProdH1(ctx, prec)
        mv.evaluate(U, dt)
        gpu_lib.JacobiPrec(ctx).setup()
        x, n, res = gpu_lib.GmresSolver(ctx, 30, 300, 1e-8).solve(-R)
        r = -R - o.matvec(mv.blocks(), x)
        assert np.linalg.norm(r) <= (1e-7 if prec == 64 else 1e-5) * np.linalg.norm(R)
        its[pcname] = n
    assert its["ilu"] < its["bj"]


def test_newton_with_ilu(gpu_lib):
    m = W.make_lattice_mesh(8, jitter=0.1, codes="channel")
    Ub = W.freestream(0.8)
    U0 = W.perturbed_state(m["X"].shape[0], 0.8)
    out = {}
    for pcname in ("bj", "ilu"):
        ctx = gpu_lib.Context.from_mesh(m, Ub)
        if pcname == "ilu":
            ctx.set_preconditioner(gpu_lib.PC_ILU0)
        U, info = gpu_lib.ImplicitSteadySolver(ctx, precision=32, tol=1e-8, max_steps=300).solve(U0)
        assert info["rel_residual"] <= 1e-8
        out[pcname] = (U, info["linear_its"])
    assert out["ilu"][1] < out["bj"][1]
    assert rel_l2(out["ilu"][0], out["bj"][0]) < 1e-7


@pytest.mark.parametrize("transpose", [False, True])
def test_linearized_solve_with_ilu(gpu_lib, transpose):
    m = W.make_lattice_mesh(7, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    ctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=2)
    ctx.set_preconditioner(gpu_lib.PC_ILU0)
    S = gpu_lib.Sensitivity(ctx)
    U = W.smooth_state(m["X"], 0.8)
    b = np.random.default_rng(4).standard_normal(U.shape)
    for inner in (0, 10):
        x, its, res = S.solve(U, b, transpose=transpose, krylov=30, maxits=600, eps=1e-10, inner_its=inner)
        Ax = S.vjp(U, x) if transpose else S.jvp(U, x)
        assert np.linalg.norm(Ax - b) <= 1e-9 * np.linalg.norm(b)
