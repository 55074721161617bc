"""GPU parity of the Spalart-Allmaras residual (six components, rho nu~
last) against the oracle's restatement, through the C ABI.  Tolerance:
relative L2 <= 1e-12 for the whole residual and for its sixth component
alone."""
import numpy as np
import pytest

from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12


def sa_state(m, U5, seed=5):
    # a positive, varying nu~ (freestream-like level 1e-3 with a bump) so
    # that production, destruction and the cb2 term are all active
    rng = np.random.default_rng(seed)
    X = m["X"]
    nu = 1e-3 * (1.0 + 4.0 * np.exp(-((X - 0.5) ** 2).sum(1) / 0.05)) * (1.0 + 0.1 * rng.random(len(X)))
    return np.column_stack([U5, U5[:, 0] * nu])


@pytest.fixture(scope="module", params=[("channel", 9, 0.2), ("farfield", 6, 0.0)])
def case(request, gpu_lib, oracle_mod):
    codes, n, jit = request.param
    m = W.make_lattice_mesh(n, jitter=jit, codes=codes)
    mach = 0.8 if codes == "channel" else 0.5
    Ub6 = np.concatenate([W.freestream(mach), [1e-3 * W.freestream(mach)[0]]])
    d2wall = np.abs(m["X"][:, 2]) + 0.02 * m["X"][:, 0]
    return m, Ub6, d2wall, oracle_mod.Oracle(m), mach


@pytest.mark.parametrize("rec,model", [(1, 1), (2, 1), (3, 1), (2, 2), (2, 0)])
def test_sa_residual_parity(gpu_lib, case, rec, model):
    m, Ub6, d2wall, o, mach = case
    A = gpu_lib
    ctx = A.Context.from_mesh(m, Ub6[:5], reconstruction=rec)
    visc = dict(model=model, reynolds_mu=2000.0, prandtl=0.72, bulk_viscosity=0.1, sutherland_alpha=1.3,
                sutherland_Ts=0.35)
    ctx.set_viscosity(**visc)
    ctx.set_turbulence(d2wall, Ub6)
    U6 = sa_state(m, W.perturbed_state(o.N, mach))
    R, bad = A.SpaceOperator(ctx).computeResidualSA(U6)
    Rr, bad_r = o.residual_sa(U6, Ub6, d2wall, order=rec, model=model, reynolds=2000.0, prandtl=0.72, bulk=0.1,
                              alpha=1.3, Ts=0.35)
    assert bad == bad_r == 0
    assert rel_l2(R, Rr) < TOL
    assert rel_l2(R[:, 5], Rr[:, 5]) < TOL
    # the sixth row is not trivially zero: advection, diffusion and source
    assert np.abs(Rr[:, 5]).max() > 0.0


def test_sa_fv3_form_and_device_arrays(gpu_lib, case):
    import torch
    m, Ub6, d2wall, o, mach = case
    A = gpu_lib
    ctx = A.Context.from_mesh(m, Ub6[:5], reconstruction=2)
    ctx.set_viscosity(model=1, reynolds_mu=500.0)
    ctx.set_turbulence(d2wall, Ub6, fv3=1, prandtl_turbulent=0.85)
    U6 = sa_state(m, W.perturbed_state(o.N, mach), seed=9)
    Rd, _ = A.SpaceOperator(ctx).computeResidualSA(torch.from_numpy(U6).cuda())
    sa = (0.1355, 0.622, 0.3, 2.0, 7.1, 5.0, 2.0 / 3.0, 0.41, 0.85)
    Rr, _ = o.residual_sa(U6, Ub6, d2wall, order=2, model=1, reynolds=500.0, sa=sa, fv3=True)
    assert rel_l2(Rd.cpu().numpy(), Rr) < TOL


def test_zero_nu_tilde_matches_the_laminar_residual(gpu_lib, case):
    # the SA residual at nu~ = 0 is the laminar Navier-Stokes residual of
    # the five-component path (a different kernel organisation on the GPU)
    m, Ub6, d2wall, o, mach = case
    A = gpu_lib
    ctx = A.Context.from_mesh(m, Ub6[:5], reconstruction=2)
    ctx.set_viscosity(model=2, reynolds_mu=800.0, sutherland_alpha=1.1, sutherland_Ts=0.4)
    ctx.set_turbulence(d2wall, np.concatenate([Ub6[:5], [0.0]]))
    U5 = W.perturbed_state(o.N, mach)
    R6, _ = A.SpaceOperator(ctx).computeResidualSA(np.column_stack([U5, np.zeros(o.N)]))
    R5, _ = A.SpaceOperator(ctx).computeResidual(U5)
    assert rel_l2(R6[:, :5], R5) < TOL
    assert not R6[:, 5].any()


def test_sa_needs_the_model_and_valid_inputs(gpu_lib, case):
    m, Ub6, d2wall, o, mach = case
    A = gpu_lib
    ctx = A.Context.from_mesh(m, Ub6[:5])
    with pytest.raises(A.AerofError):
        A.SpaceOperator(ctx).computeResidualSA(np.ones((o.N, 6)))
    bad_d = d2wall.copy()
    bad_d[3] = -1.0
    with pytest.raises(A.AerofError):
        ctx.set_turbulence(bad_d, Ub6)
    ctx.set_turbulence(d2wall, Ub6)
    ctx.set_turbulence(None, None)
    with pytest.raises(A.AerofError):
        A.SpaceOperator(ctx).computeResidualSA(np.ones((o.N, 6)))
