"""Failure paths, every one injected on the host (no GPU fault, trap or hang
is provoked): a Newton update that makes the state non-physical (redone at
half the CFL number, NewtonSolver.h:195-205, TsParameters.C:187-195), a CFL
number driven below cfl0/1000 (AEROF_EDIVERGED), a singular diagonal block
(AEROF_ESINGULAR, DiagMatrix.C:65-67), a non-finite input state, and a
degenerate mesh (zero control volumes, rejected at set_mesh)."""
import numpy as np
import pytest

from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _harsh_state(o, trial):
    """Hot high-pressure spots beside near-vacuum spots on a 7^3 channel
    state (seeded): a large first Newton step drives some densities or
    pressures negative."""
    rng = np.random.default_rng(1)
    for t in range(trial + 1):
        V = o.prim(W.perturbed_state(o.N, 0.8, amp=0.02))
        idx = rng.integers(0, o.N, 6)
        V[idx[:3], 4] *= 50.0
        V[idx[3:], 4] *= 0.01
        V[idx[3:], 0] *= 0.01
    return W.prim_to_cons(V)


@pytest.fixture(scope="module")
def harsh(oracle_mod):
    m = W.make_lattice_mesh(7, jitter=0.1, codes="channel")
    o = oracle_mod.Oracle(m)
    return m, W.freestream(0.8), o


def test_newton_redoes_nonphysical_updates_like_the_oracle(gpu_lib, harsh):
    m, Ub, o = harsh
    U = _harsh_state(o, 1)
    Ur, hist, _ = o.newton(U, Ub, order=1, cfl0=100.0, cfl_max=1e6, tol=1e-8, max_steps=300, fp32_prec=False)
    assert o.last_redos > 0
    ctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=gpu_lib.REC_CONSTANT)
    sol = gpu_lib.ImplicitSteadySolver(ctx, precision=64, cfl0=100.0, cfl_max=1e6, tol=1e-8, max_steps=300)
    Ug, info = sol.solve(U)
    assert info["redos"] == o.last_redos
    assert info["steps"] == len(hist) - 1
    assert info["rel_residual"] <= 1e-8
    assert rel_l2(Ug, Ur) <= 1e-9
    ctx.close()


def test_newton_gives_up_below_the_cfl_floor(gpu_lib, harsh):
    m, Ub, o = harsh
    U = _harsh_state(o, 0)
    with pytest.raises(RuntimeError):
        o.newton(U, Ub, order=1, cfl0=100.0, cfl_max=1e6, tol=1e-8, max_steps=300, fp32_prec=False)
    ctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=gpu_lib.REC_CONSTANT)
    sol = gpu_lib.ImplicitSteadySolver(ctx, precision=64, cfl0=100.0, cfl_max=1e6, tol=1e-8, max_steps=300)
    with pytest.raises(gpu_lib.AerofError) as e:
        sol.solve(U)
    assert e.value.code == -7
    assert "cfl0/1000" in str(e.value)
    # the context stays usable
    R, bad = gpu_lib.SpaceOperator(ctx).computeResidual(W.perturbed_state(o.N, 0.8))
    assert bad == 0 and np.isfinite(R).all()
    ctx.close()


@pytest.mark.parametrize("prec", [64, 32])
def test_singular_diagonal_block(gpu_lib, harsh, prec):
    m, Ub, o = harsh
    ctx = gpu_lib.Context.from_mesh(m, Ub)
    mv = gpu_lib.MatVecProdH1(ctx, prec)
    mv.evaluate(W.perturbed_state(o.N, 0.8))
    A = mv.blocks()
    pc = gpu_lib.JacobiPrec(ctx)
    pc.setup()                      # the assembled operator is fine
    A[5] = 1.0                      # rank one, non-zero diagonal: a zero pivot in the elimination
    mv.set_blocks(A)
    assert np.array_equal(mv.blocks()[5], A[5])
    with pytest.raises(gpu_lib.AerofError) as e:
        pc.setup()
    assert e.value.code == -5
    ctx.close()


@pytest.mark.parametrize("rec", [1, 2])
def test_nonfinite_state(gpu_lib, harsh, rec):
    m, Ub, o = harsh
    ctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=rec)
    U = W.perturbed_state(o.N, 0.8)
    U[100, 4] = np.nan
    # the residual counts the node's edges as unphysical (a warning code)
    _, bad = gpu_lib.SpaceOperator(ctx).computeResidual(U)
    assert bad > 0
    # the Newton solve refuses a non-finite residual
    with pytest.raises(gpu_lib.AerofError) as e:
        gpu_lib.ImplicitSteadySolver(ctx, precision=64, max_steps=5).solve(U)
    assert e.value.code == -1 and "non-finite" in str(e.value)
    ctx.close()


def test_degenerate_mesh_rejected(gpu_lib):
    m = W.make_lattice_mesh(4, codes="channel")
    ctx = gpu_lib.Context()
    # an inverted tet alone is accepted (the reference accepts it; the
    # control volumes stay positive)
    X = m["X"].copy()
    X[21] += np.array([0.2, -0.2, 0.0])   # inverts two tets around node 21
    ctx.set_mesh(X, m["tets"], m["faces"], m["codes"], W.freestream(0.8))
    # a flat mesh: every tet and control volume is zero
    X = m["X"].copy()
    X[:, 2] = 0.0
    with pytest.raises(gpu_lib.AerofError) as e:
        ctx.set_mesh(X, m["tets"], m["faces"], m["codes"], W.freestream(0.8))
    assert e.value.code == -1 and "control volume" in str(e.value)
    X = m["X"].copy()
    X[3, 1] = np.inf
    with pytest.raises(gpu_lib.AerofError) as e:
        ctx.set_mesh(X, m["tets"], m["faces"], m["codes"], W.freestream(0.8))
    assert e.value.code == -1 and "non-finite" in str(e.value)
    ctx.set_mesh(m["X"], m["tets"], m["faces"], m["codes"], W.freestream(0.8))
    ctx.close()
