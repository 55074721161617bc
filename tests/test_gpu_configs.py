"""GPU parity against the CPU oracle on the benchmark configurations
themselves (all through the C ABI):

* the CPU-runnable plain method: 21^3 lattice (N=9,261, E=59,660), far
  field on every face, Mach 0.5, first-order Roe, 10 RK2 steps at CFL 0.8
  (ExplicitTsDesc::computeRKSecondOrder, ExplicitTsDesc.C:98-117);
* the second-order residual: 101^3 jittered lattice (N=1,030,301,
  E=7,090,300), LSQ gradients + van Albada + Roe, slip walls y/z, far field
  x, Mach 0.8 (SpaceOperator::computeResidual, SpaceOperator.C:524-634;
  DistNodalGrad::compute, DistNodalGrad.C:790-806);
* the pseudo-transient Newton-GMRES converged state (NewtonSolver.h:70-231,
  TsParameters.C:182-217) at 21^3 in FP64 and mixed precision against the
  oracle's FP64 Newton.

Tolerances: relative L2 <= 1e-12 for the FP64 residual, gradients and RK2
state; for Newton both solves stop at ||R||/||R0|| <= 1e-8, so the states
agree to that level (the tolerance of each comparison is written beside it).
"""
import numpy as np
import pytest

from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.parametrize("kernel", [0, 1])
def test_config1_rk2_21cube(gpu_lib, oracle_mod, kernel):
    m = W.make_lattice_mesh(21, codes="farfield")
    assert m["X"].shape[0] == 9261
    Ub = W.freestream(0.5)
    o = oracle_mod.Oracle(m)
    assert o.E == 59660
    U = W.perturbed_state(o.N, 0.5)
    ctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=1, residual_kernel=kernel)
    Ug, bad = gpu_lib.ExplicitRK2(ctx, 0.8).run(U, 10)
    Ur = o.rk2(U, Ub, 1, 0.8, 10)
    assert bad == 0
    assert rel_l2(Ug, Ur) <= TOL
    # the update itself (not only the state, which is dominated by U)
    assert rel_l2(Ug - U, Ur - U) <= 1e-10


@pytest.fixture(scope="module")
def config2(gpu_lib, oracle_mod):
    m = W.make_lattice_mesh(101, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.8)
    ctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=gpu_lib.REC_VANALBADA)
    yield m, Ub, o, U, ctx
    ctx.close()


def test_config2_residual_101cube(gpu_lib, config2):
    m, Ub, o, U, ctx = config2
    assert ctx.E == 7090300 and ctx.N == 1030301
    R, bad = gpu_lib.SpaceOperator(ctx).computeResidual(U)
    Rr, bad_r = o.residual(U, Ub, 2)
    assert bad == bad_r == 0
    assert rel_l2(R, Rr) <= TOL


def test_config2_gradients_101cube(gpu_lib, config2):
    m, Ub, o, U, ctx = config2
    V = o.prim(U)
    got = gpu_lib.SpaceOperator(ctx).computeGradients(V)
    ref = o.gradients(V)
    for a, b in zip(got, ref):
        assert rel_l2(a, b) <= TOL


@pytest.mark.parametrize("prec", [64, 32])
def test_newton_state_vs_oracle_21cube(gpu_lib, oracle_mod, prec):
    m = W.make_lattice_mesh(21, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.8, amp=0.02)
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    sol = gpu_lib.ImplicitSteadySolver(ctx, precision=prec, cfl0=10.0, cfl_max=1e4, ser=0.7, ksp_eps=1e-2,
                                       krylov=30, maxits=30, tol=1e-8, max_steps=300)
    Ug, info = sol.solve(U)
    # the oracle solves in FP64 throughout (the FP64 CPU oracle state)
    Ur, hist, lits = o.newton(U, Ub, order=2, tol=1e-8, max_steps=300, fp32_prec=False)
    assert info["rel_residual"] <= 1e-8
    assert hist[-1] <= 1e-8
    # both states satisfy ||R|| <= 1e-8 ||R0||: their difference is bounded
    # by that level times the conditioning of the steady problem
    assert rel_l2(Ug, Ur) <= 1e-9
    R0 = np.linalg.norm(o.residual(U, Ub, 2)[0])
    Rg, _ = o.residual(Ug, Ub, 2)
    assert np.linalg.norm(Rg) <= 1.01e-8 * R0
    ctx.close()
