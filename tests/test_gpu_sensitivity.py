"""Shape sensitivities on the GPU: adjoint and direct methods agree, and
both match central finite differences of the re-converged flow (step 1e-6).
The base geometry carries a bump on z=0 so the converged flow is not the
uniform free stream (at a uniform state every edge difference is exactly
zero, where the van Albada limiter is not differentiable)."""
import numpy as np
import pytest

from aerof_dev_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[2, 3])
def flow(gpu_lib, request):
    from aerof_dev_b200 import sensitivity as S
    m = W.make_lattice_mesh(9, jitter=0.1, codes="channel")
    X = m["X"] + W.shape_modes(m["X"], 1, sigma=0.25, amplitude=0.04, seed=7)[0]
    m = dict(m, X=X)
    Ub = W.freestream(0.8)
    ctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=request.param)
    U0 = np.tile(Ub, (X.shape[0], 1))
    U, info = S.converge(ctx, U0, tol=1e-10)
    zf = np.nonzero(m["sides"] == 4)[0]
    F = S.ZForce(m["faces"], zf)
    modes = W.shape_modes(X, 3, seed=11, amplitude=1.0)
    return ctx, m, U, info, F, modes


def test_converged(flow):
    ctx, m, U, info, F, modes = flow
    # exact Newton down to the round-off floor of the residual
    assert info["rel_residual"] <= 1e-10
    assert info["exact_newton_residuals"][-1] <= 1e-3 * info["exact_newton_residuals"][0]


def test_adjoint_equals_direct(flow):
    from aerof_dev_b200 import sensitivity as S
    ctx, m, U, info, F, modes = flow
    ga, _ = S.adjoint_gradient(ctx, U, m["X"], F, modes)
    gd, _ = S.direct_gradient(ctx, U, m["X"], F, modes)
    assert np.abs(ga - gd).max() <= 1e-8 * np.abs(gd).max()


def test_adjoint_matches_fd(flow):
    from aerof_dev_b200 import sensitivity as S
    ctx, m, U, info, F, modes = flow
    ga, _ = S.adjoint_gradient(ctx, U, m["X"], F, modes)
    # central differences at step 1e-6 of the re-converged flow: their
    # round-off floor is ~1e-11 (error in J) / 1e-6 = 1e-5 of the gradient
    gf = S.fd_gradient(ctx, U, m["X"], F, modes, h=1e-6, tol=1e-10)
    assert np.abs(ga - gf).max() <= 5e-5 * np.abs(gf).max()
    if ctx.cfg.reconstruction == 3:
        # smooth scheme (no limiter): Richardson-extrapolated differences
        # (steps 2e-4, 1e-4, truncation O(h^4)) resolve 1e-6
        gr = S.fd_gradient(ctx, U, m["X"], F, modes, h=(2e-4, 1e-4), tol=1e-10)
        assert np.abs(ga - gr).max() <= 1e-6 * np.abs(gr).max()


def test_batched_direct_equals_adjoint(flow):
    # all modes' direct sensitivities from one batched solve (stored exact
    # linearisation) agree with the adjoint gradient; the adjoint solve with
    # the stored operator gives the same gradient as the matrix-free one
    from aerof_dev_b200 import sensitivity as S
    ctx, m, U, info, F, modes = flow
    ga, _ = S.adjoint_gradient(ctx, U, m["X"], F, modes)
    gb, binfo = S.direct_gradient_batch(ctx, U, m["X"], F, modes)
    assert len(binfo["direct_its"]) == len(modes)
    assert np.abs(ga - gb).max() <= 1e-8 * np.abs(ga).max()
    gs, _ = S.adjoint_gradient(ctx, U, m["X"], F, modes, stored_operator=True)
    assert np.abs(ga - gs).max() <= 1e-8 * np.abs(ga).max()


def test_adjoint_matches_oracle_dual_numbers(flow):
    # every mode's adjoint gradient against the oracle's exact directional
    # derivatives: the oracle forms dR/dU column by column from its
    # dual-number J v (FP64, CPU), solves the adjoint system densely, and
    # takes dJ/ds_k = dJ/dX . Xdot_k - lambda . (dR/dX . Xdot_k) with its
    # dual-number dR/dX, so no GPU product enters the reference value
    from aerof_dev_b200 import sensitivity as S
    from oracle.oracle import Oracle, zfaces_of
    ctx, m, U, info, F, modes = flow
    rec = ctx.cfg.reconstruction
    U = S._host(U)
    Ub = W.freestream(0.8)
    o = Oracle(m)
    n = 5 * o.N
    Jd = np.empty((n, n))
    e = np.zeros((o.N, 5))
    for c in range(n):
        e.flat[c] = 1.0
        Jd[:, c] = o.jvp(U, Ub, e, order=rec).reshape(-1)
        e.flat[c] = 0.0
    zf = zfaces_of(m)
    lam = np.linalg.solve(Jd.T, o.zforce_dU(U, zf).reshape(-1))
    g_or = np.array([o.zforce_dX(U, zf, Xd) - lam @ o.dRdX(U, Ub, Xd, order=rec)[0].reshape(-1) for Xd in modes])
    ga, _ = S.adjoint_gradient(ctx, U, m["X"], F, modes)
    assert np.abs(ga - g_or).max() <= 1e-8 * np.abs(g_or).max()
