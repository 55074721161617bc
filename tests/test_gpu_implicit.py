"""GPU parity of the Newton-Krylov inner loop against the CPU oracle:
H1 Jacobian (FP64 and FP32 storage), matvec and transpose, block-Jacobi,
GMRES and the pseudo-transient Newton solve."""
import numpy as np
import pytest

from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(gpu_lib, oracle_mod):
    m = W.make_lattice_mesh(8, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.8)
    dt = o.timestep(U, 50.0)
    A = o.jacobian(U, Ub, dt)
    return m, Ub, o, U, dt, A


def test_jacobian_fp64_parity(gpu_lib, setup):
    m, Ub, o, U, dt, A = setup
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    mv = gpu_lib.MatVecProdH1(ctx, gpu_lib.PREC_FP64)
    mv.evaluate(U, dt)
    G = mv.blocks()
    # edge blocks: analytic roejac6, FP64 parity.  Diagonal blocks hold the
    # far-field face blocks, a forward difference with step 1e-6*|V_k|
    # (FluxFcnBase.h:118-136): for a velocity component of 1e-2 the step is
    # 1e-8, so 1e-16 rounding differences in the two flux evaluations
    # (FMA contraction) become ~1e-8 in the quotient.
    assert rel_l2(G[o.N:], A[o.N:]) < 1e-12
    assert rel_l2(G[: o.N], A[: o.N]) < 1e-6


def test_jacobian_fp32_storage(gpu_lib, setup):
    # the FP32 operator of the mixed-precision solver is formed in FP32
    # arithmetic (edge blocks) and summed into the diagonal in FP64: each
    # block agrees with the FP64 oracle to FP32 accuracy
    m, Ub, o, U, dt, A = setup
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    mv = gpu_lib.MatVecProdH1(ctx, gpu_lib.PREC_FP32)
    mv.evaluate(U, dt)
    G = mv.blocks()
    off, ref = G[o.N:].reshape(-1, 25), A[o.N:].reshape(-1, 25)
    scale = np.abs(ref).max(axis=1, keepdims=True)
    assert np.abs(off - ref).max() <= 1e-5 * scale.max()
    assert np.all(np.abs(off - ref) <= 1e-5 * scale + 1e-30)
    assert rel_l2(G, A) < 1e-6


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("trans", [False, True])
def test_matvec_parity(gpu_lib, setup, prec, trans):
    m, Ub, o, U, dt, A = setup
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    mv = gpu_lib.MatVecProdH1(ctx, prec)
    mv.evaluate(U, dt)
    p = np.random.default_rng(1).standard_normal((o.N, 5))
    Aref = mv.blocks()  # the operator the GPU assembled (assembly parity is tested above)
    y = mv.apply(p, transpose=trans)
    assert rel_l2(y, o.matvec(Aref, p, transpose=trans)) < 1e-13


def test_adjointness_of_transpose(gpu_lib, setup):
    m, Ub, o, U, dt, A = setup
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    mv = gpu_lib.MatVecProdH1(ctx, 32)
    mv.evaluate(U, dt)
    rng = np.random.default_rng(2)
    x, y = rng.standard_normal((2, o.N, 5))
    a = np.sum(mv.apply(x) * y)
    b = np.sum(x * mv.applyTranspose(y))
    assert abs(a - b) <= 1e-12 * abs(a)


@pytest.mark.parametrize("prec", [64, 32])
def test_block_jacobi_parity(gpu_lib, setup, prec):
    m, Ub, o, U, dt, A = setup
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    mv = gpu_lib.MatVecProdH1(ctx, prec)
    mv.evaluate(U, dt)
    pc = gpu_lib.JacobiPrec(ctx)
    pc.setup()
    D, bad = o.bj_invert(mv.blocks(), fp32=(prec == 32))
    assert bad == 0
    x = np.random.default_rng(3).standard_normal((o.N, 5))
    z = pc.apply(x)
    zr = np.einsum("nij,nj->ni", D, x)
    assert rel_l2(z, zr) < (1e-13 if prec == 64 else 1e-6)
    zt = pc.applyT(x)
    assert rel_l2(zt, np.einsum("nji,nj->ni", D, x)) < (1e-13 if prec == 64 else 1e-6)


@pytest.mark.parametrize("prec", [64, 32])
def test_gmres_parity(gpu_lib, setup, prec):
    m, Ub, o, U, dt, A = setup
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    mv = gpu_lib.MatVecProdH1(ctx, prec)
    mv.evaluate(U, dt)
    pc = gpu_lib.JacobiPrec(ctx)
    pc.setup()
    R, _ = o.residual(U, Ub, 2)
    b = -R
    ks = gpu_lib.GmresSolver(ctx, 30, 30, 1e-6)
    x, its, res = ks.solve(b)
    Ablk = mv.blocks()
    D, _ = o.bj_invert(Ablk, fp32=(prec == 32))
    xr, itr, resr = o.gmres(Ablk, D, b, 30, 30, 1e-6)
    if prec == 64:
        assert its == itr
        assert rel_l2(x, xr) < 1e-9
    else:
        # FP32 Krylov vectors (FP64 dots, norms and Hessenberg system)
        assert abs(its - itr) <= 2
        assert rel_l2(x, xr) < 1e-4
    # right preconditioning: GMRES's residual estimate is the true residual
    # (to the precision the Krylov vectors are stored in)
    r = b - o.matvec(Ablk, x)
    assert abs(np.linalg.norm(r) - res) <= (1e-6 if prec == 64 else 1e-4) * np.linalg.norm(b)


def test_gmres_saturation_reports_maxits(gpu_lib, setup):
    m, Ub, o, U, dt, A = setup
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    mv = gpu_lib.MatVecProdH1(ctx, 32)
    mv.evaluate(U, dt)
    gpu_lib.JacobiPrec(ctx).setup()
    R, _ = o.residual(U, Ub, 2)
    x, its, res = gpu_lib.GmresSolver(ctx, 30, 1, 1e-12).solve(-R)
    assert its == 1 and res > 1e-12 * np.linalg.norm(R)


@pytest.mark.parametrize("prec", [32, 64])
def test_newton_matches_oracle(gpu_lib, oracle_mod, prec):
    m = W.make_lattice_mesh(6, jitter=0.1, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.8, amp=0.02)
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    sol = gpu_lib.ImplicitSteadySolver(ctx, precision=prec, tol=1e-8, max_steps=300)
    Ug, info = sol.solve(U)
    Ur, hist, lits = o.newton(U, Ub, order=2, tol=1e-8, max_steps=300, fp32_prec=(prec == 32))
    assert info["rel_residual"] <= 1e-8
    assert hist[-1] <= 1e-8
    assert abs(info["steps"] - (len(hist) - 1)) <= (2 if prec == 64 else 6)
    # both states satisfy ||R|| <= 1e-8 ||R0||; they agree to that level
    assert rel_l2(Ug, Ur) < (1e-9 if prec == 64 else 1e-7)
    R, _ = gpu_lib.SpaceOperator(ctx).computeResidual(Ug)
    assert np.linalg.norm(R) <= 1.01e-8 * np.linalg.norm(o.residual(U, Ub, 2)[0])


@pytest.mark.parametrize("fd_order", [1, 2])
def test_matvec_fd_parity(gpu_lib, oracle_mod, fd_order):
    # MatVecProdFD::apply with the reference's computeEpsilon against the
    # oracle's restatement (same step), and against the exact product
    m = W.make_lattice_mesh(9, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.8)
    p = np.random.default_rng(5).standard_normal(U.shape)
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    dt = gpu_lib.SpaceOperator(ctx).computeTimeStep(U, 50.0)
    for with_dt in (False, True):
        mv = gpu_lib.MatVecProdFD(ctx, fd_order)
        mv.evaluate(U, dt=dt if with_dt else None)
        y = mv.apply(p)
        yr, eps_r = o.matvec_fd(U, Ub, p, 2, dt=dt if with_dt else None, fd_order=fd_order)
        assert abs(mv.eps - eps_r) <= 1e-14 * eps_r
        # the difference quotient amplifies the residuals' last-bit
        # differences by |R| / (eps |J p|)
        assert rel_l2(y, yr) < 1e-7
        Jp = gpu_lib.Sensitivity(ctx).jvp(U, p)
        if with_dt:
            Jp = Jp + p / dt[:, None]
        assert rel_l2(y, Jp) < (1e-4 if fd_order == 1 else 1e-7)
    # R(U) given (evaluate keeps F): same product as evaluating it
    if fd_order == 1:
        R, _ = gpu_lib.SpaceOperator(ctx).computeResidual(U)
        mv = gpu_lib.MatVecProdFD(ctx, 1)
        mv.evaluate(U, F=R)
        mv2 = gpu_lib.MatVecProdFD(ctx, 1)
        mv2.evaluate(U)
        assert np.array_equal(mv.apply(p), mv2.apply(p))
    ctx.close()
