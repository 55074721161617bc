"""The residual as a torch.autograd.Function (test harness): forward is the
GPU residual R(U, X) through the C ABI, backward is the hand-written adjoint
kernel set, (J^T g, (dR/dX)^T g).  Checked with torch.autograd.gradcheck and
against central finite differences of the GPU residual, as the reference
checks its analytical sensitivities against finite differences
(FluidShapeOptimizationHandler.C:2450-2458)."""
import numpy as np
import pytest

from aerof_dev_b200 import workloads as W

pytestmark = pytest.mark.gpu


class Residual:
    """Factory of an autograd Function bound to one GPU context."""

    def __init__(self, A, gctx, X0):
        import torch

        sp = A.SpaceOperator(gctx)
        S = A.Sensitivity(gctx)
        state = {"X": X0.copy()}

        def set_coordinates(X):
            Xh = X.detach().cpu().numpy()
            if not np.array_equal(Xh, state["X"]):
                gctx.update_coordinates(Xh)
                state["X"] = Xh

        class Fn(torch.autograd.Function):
            @staticmethod
            def forward(fctx, U, X):
                set_coordinates(X)
                R, bad = sp.computeResidual(U.detach().contiguous())
                if bad:
                    raise RuntimeError(f"{bad} unphysical reconstructed states")
                fctx.save_for_backward(U, X)
                return R

            @staticmethod
            def backward(fctx, gR):
                U, X = fctx.saved_tensors
                set_coordinates(X)
                gR = gR.contiguous()
                gU = S.vjp(U.detach(), gR) if fctx.needs_input_grad[0] else None
                gX = S.dRdX_T(U.detach(), gR) if fctx.needs_input_grad[1] else None
                return gU, gX

        self.fn = Fn

    def __call__(self, U, X):
        return self.fn.apply(U, X)


@pytest.fixture(scope="module", params=[3, 2])
def setup(request, gpu_lib):
    import torch
    rec = request.param
    m = W.make_lattice_mesh(4, jitter=0.15, codes="channel")
    Ub = W.freestream(0.8)
    gctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=rec)
    U = W.smooth_state(m["X"], 0.8)
    f = Residual(gpu_lib, gctx, m["X"])
    Ut = torch.tensor(U, device="cuda", dtype=torch.float64, requires_grad=True)
    Xt = torch.tensor(m["X"], device="cuda", dtype=torch.float64, requires_grad=True)
    return rec, f, Ut, Xt, gctx


def test_gradcheck_state_and_coordinates(setup):
    import torch
    rec, f, Ut, Xt, gctx = setup
    if rec != 3:
        pytest.skip("van Albada is not smooth at eps = 1e-6 everywhere; checked directionally below")
    assert torch.autograd.gradcheck(f, (Ut, Xt), eps=1e-6, atol=1e-5, rtol=1e-4, fast_mode=True)


def test_backward_matches_central_differences(setup):
    import torch
    rec, f, Ut, Xt, gctx = setup
    rng = np.random.default_rng(21)
    c = torch.tensor(rng.standard_normal(tuple(Ut.shape)), device="cuda")
    dU = torch.tensor(rng.standard_normal(tuple(Ut.shape)), device="cuda") * 1e-2
    dX = torch.tensor(rng.standard_normal(tuple(Xt.shape)), device="cuda") * 1e-3
    L = (f(Ut, Xt) * c).sum()
    gU, gX = torch.autograd.grad(L, (Ut, Xt))
    ad = float((gU * dU).sum() + (gX * dX).sum())
    h = 1e-6
    with torch.no_grad():
        Lp = float((f(Ut + h * dU, Xt + h * dX) * c).sum())
        Lm = float((f(Ut - h * dU, Xt - h * dX) * c).sum())
        f(Ut, Xt)
    fd = (Lp - Lm) / (2 * h)
    assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1.0)
