"""GPU sensitivities: forward mode (J v, dR/dX . Xdot) against the oracle's
dual-number linearisation, reverse mode (J^T w, (dR/dX)^T lambda) by the
adjoint identity <w, J v> = <J^T w, v>, and both against central finite
differences of the GPU residual."""
import numpy as np
import pytest

from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[2, 3, 1])
def case(request, gpu_lib, oracle_mod):
    rec = request.param
    m = W.make_lattice_mesh(7, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.smooth_state(m["X"], 0.8)
    ctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=rec)
    return rec, m, Ub, o, U, ctx


def test_jvp_matches_oracle(gpu_lib, case):
    rec, m, Ub, o, U, ctx = case
    v = np.random.default_rng(11).standard_normal(U.shape) * 1e-2
    Jv = gpu_lib.Sensitivity(ctx).jvp(U, v)
    assert rel_l2(Jv, o.jvp(U, Ub, v, order=rec)) < 1e-11


def test_dRdX_matches_oracle(gpu_lib, case):
    rec, m, Ub, o, U, ctx = case
    Xdot = W.shape_modes(m["X"], 2)[1]
    dR = gpu_lib.Sensitivity(ctx).dRdX(U, Xdot)
    ref, _ = o.dRdX(U, Ub, Xdot, order=rec)
    assert rel_l2(dR, ref) < 1e-10


def test_vjp_adjoint_identity(gpu_lib, case):
    rec, m, Ub, o, U, ctx = case
    rng = np.random.default_rng(12)
    v = rng.standard_normal(U.shape)
    w = rng.standard_normal(U.shape)
    S = gpu_lib.Sensitivity(ctx)
    a = np.sum(w * S.jvp(U, v))
    b = np.sum(S.vjp(U, w) * v)
    assert abs(a - b) <= 1e-11 * max(abs(a), 1e-300)


def test_dRdX_T_adjoint_identity(gpu_lib, case):
    rec, m, Ub, o, U, ctx = case
    rng = np.random.default_rng(13)
    lam = rng.standard_normal(U.shape)
    Xdot = rng.standard_normal(m["X"].shape)
    S = gpu_lib.Sensitivity(ctx)
    a = np.sum(lam * S.dRdX(U, Xdot))
    b = np.sum(S.dRdX_T(U, lam) * Xdot)
    assert abs(a - b) <= 1e-10 * max(abs(a), 1e-300)


def test_jvp_matches_central_fd(gpu_lib, case):
    rec, m, Ub, o, U, ctx = case
    v = np.random.default_rng(14).standard_normal(U.shape) * 1e-2
    sp = gpu_lib.SpaceOperator(ctx)
    h = 1e-6
    fd = (sp.computeResidual(U + h * v)[0] - sp.computeResidual(U - h * v)[0]) / (2 * h)
    assert rel_l2(gpu_lib.Sensitivity(ctx).jvp(U, v), fd) < 1e-6


@pytest.mark.parametrize("transpose", [False, True])
def test_linearized_solve(gpu_lib, case, transpose):
    rec, m, Ub, o, U, ctx = case
    S = gpu_lib.Sensitivity(ctx)
    b = np.random.default_rng(15).standard_normal(U.shape)
    x, its, res = S.solve(U, b, transpose=transpose, krylov=30, maxits=600, eps=1e-10)
    Ax = S.vjp(U, x) if transpose else S.jvp(U, x)
    assert np.linalg.norm(Ax - b) <= 1e-9 * np.linalg.norm(b)


@pytest.mark.parametrize("transpose", [False, True])
def test_linearized_solve_flexible(gpu_lib, case, transpose):
    # flexible GMRES preconditioned by inner mixed-precision solves of the
    # first-order operator reaches the same FP64 accuracy in fewer outer
    # iterations than block-Jacobi GMRES
    rec, m, Ub, o, U, ctx = case
    S = gpu_lib.Sensitivity(ctx)
    b = np.random.default_rng(16).standard_normal(U.shape)
    x, its, res = S.solve(U, b, transpose=transpose, krylov=30, maxits=300, eps=1e-10, inner_its=10)
    Ax = S.vjp(U, x) if transpose else S.jvp(U, x)
    assert np.linalg.norm(Ax - b) <= 1e-9 * np.linalg.norm(b)
    _, its_bj, _ = S.solve(U, b, transpose=transpose, krylov=30, maxits=600, eps=1e-10)
    assert its < its_bj


def test_transposed_assembly_is_the_transpose(gpu_lib, case):
    # the flexible adjoint solve assembles H1^T directly (coalesced transpose
    # products); read back, it is the FP32 H1 assembled the usual way, and
    # its products with and without transpose match.  Both are formed in
    # FP32 arithmetic by different rows of each edge, so they agree to FP32
    # rounding, not bit for bit.
    rec, m, Ub, o, U, ctx = case
    S = gpu_lib.Sensitivity(ctx)
    b = np.random.default_rng(17).standard_normal(U.shape)
    S.solve(U, b, transpose=True, krylov=5, maxits=2, eps=1e-10, inner_its=3)
    mv = gpu_lib.MatVecProdH1(ctx, gpu_lib.PREC_FP32)
    GT = mv.blocks()
    p = np.random.default_rng(18).standard_normal(U.shape)
    yT, y = mv.apply(p, transpose=True), mv.apply(p)
    mv.evaluate(U)
    G = mv.blocks()
    scale = np.abs(G).reshape(len(G), 25).max(axis=1)
    assert np.all(np.abs(GT - G).reshape(len(G), 25).max(axis=1) <= 1e-5 * scale + 1e-30)
    assert rel_l2(mv.apply(p, transpose=True), yT) < 1e-6
    assert rel_l2(mv.apply(p), y) < 1e-6


def test_dRdX_T_fresh_context_and_fused_products(gpu_lib, case):
    # a fresh context whose first call is the reverse product (no earlier
    # call has left node records or gradients behind), and the fused sweep
    # returning both adjoint products
    rec, m, Ub, o, U, _ = case
    ctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=rec)
    S = gpu_lib.Sensitivity(ctx)
    rng = np.random.default_rng(19)
    lam = rng.standard_normal(U.shape)
    Xdot = rng.standard_normal(m["X"].shape)
    gX = S.dRdX_T(U, lam)
    ref, _ = o.dRdX(U, Ub, Xdot, order=rec)
    a, b = np.sum(lam * ref), np.sum(gX * Xdot)
    assert abs(a - b) <= 1e-10 * max(abs(a), 1e-300)
    ctx2 = gpu_lib.Context.from_mesh(m, Ub, reconstruction=rec)
    JTl, gX2 = gpu_lib.Sensitivity(ctx2).adjoint_products(U, lam)
    assert rel_l2(gX2, gX) < 1e-14
    assert rel_l2(JTl, S.vjp(U, lam)) < 1e-14
