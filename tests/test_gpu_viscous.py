"""The laminar viscous Galerkin term on the GPU against the oracle's
restatement (relative L2 <= 1e-12): constant and Sutherland viscosity,
both residual organisations, constant and van Albada reconstruction, the
allocation-free entry point; the Newton solve with it (defect correction
with the inviscid H1) converges; the exact linearisations refuse it."""
import numpy as np
import pytest
import torch

from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12
SUTH = {"alpha": 1.4 * 0.4 * 0.64, "Ts": 0.38}


@pytest.mark.parametrize("kernel", [0, 1])
@pytest.mark.parametrize("rec", [1, 2])
@pytest.mark.parametrize("model", [1, 2])
def test_viscous_residual_parity(gpu_lib, oracle_mod, kernel, rec, model):
    m = W.make_lattice_mesh(9, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.8)
    ctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=rec, residual_kernel=kernel)
    kw = SUTH if model == 2 else {}
    ctx.set_viscosity(model=model, reynolds_mu=200.0, prandtl=0.72,
                      sutherland_alpha=kw.get("alpha", 1.0), sutherland_Ts=kw.get("Ts", 0.0))
    R, bad = gpu_lib.SpaceOperator(ctx).computeResidual(U)
    Rr, bad_r = o.residual_visc(U, Ub, rec, model=model, reynolds=200.0, prandtl=0.72, **kw)
    assert bad == bad_r == 0
    assert rel_l2(R, Rr) <= TOL
    # switching the model off gives the inviscid residual back
    ctx.set_viscosity(model=0)
    R0, _ = gpu_lib.SpaceOperator(ctx).computeResidual(U)
    assert rel_l2(R0, o.residual(U, Ub, rec)[0]) <= TOL
    ctx.close()


def test_viscous_noalloc_and_guards(gpu_lib, oracle_mod):
    import ctypes as C
    m = W.make_lattice_mesh(9, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    ctx.set_viscosity(model=1, reynolds_mu=100.0)
    U = torch.from_numpy(W.perturbed_state(ctx.N, 0.8)).cuda()
    R1 = torch.empty_like(U)
    R2 = torch.empty_like(U)
    ctx._check(ctx.L.aerof_gpu_residual(ctx.h, C.c_void_p(U.data_ptr()), C.c_void_p(R1.data_ptr())))
    ctx._check(ctx.L.aerof_gpu_residual_noalloc(ctx.h, C.c_void_p(U.data_ptr()), C.c_void_p(R2.data_ptr())))
    assert rel_l2(R2.cpu().numpy(), R1.cpu().numpy()) <= TOL
    S = gpu_lib.Sensitivity(ctx)
    with pytest.raises(gpu_lib.AerofError) as e:
        S.jvp(U, U)
    assert e.value.code == -1 and "viscous" in str(e.value)
    with pytest.raises(gpu_lib.AerofError):
        ctx.set_viscosity(model=1, reynolds_mu=-1.0)
    ctx.close()


def test_viscous_newton_converges(gpu_lib, oracle_mod):
    m = W.make_lattice_mesh(9, jitter=0.1, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.8, amp=0.02)
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    ctx.set_viscosity(model=2, reynolds_mu=1000.0, sutherland_alpha=SUTH["alpha"], sutherland_Ts=SUTH["Ts"])
    sol = gpu_lib.ImplicitSteadySolver(ctx, precision=64, tol=1e-8, max_steps=400)
    Ug, info = sol.solve(U)
    assert info["rel_residual"] <= 1e-8
    R0 = np.linalg.norm(o.residual_visc(U, Ub, 2, model=2, reynolds=1000.0, **SUTH)[0])
    Rf = np.linalg.norm(o.residual_visc(Ug, Ub, 2, model=2, reynolds=1000.0, **SUTH)[0])
    assert Rf <= 1.01e-8 * R0
    ctx.close()
