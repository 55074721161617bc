"""CPU tests of the oracle's Spalart-Allmaras restatement: its convective
fluxes are pinned bit for bit to the reference's own Fortran (roeflux7.f and
boundflux5.f with type 1, translated and run by
tests/golden/make_golden_f77.py); its Galerkin term by properties (the
reference's SpalartAllmarasTerm.h / FemEquationTermDesc.C need the MPI
headers and cannot be compiled here)."""
import os

import numpy as np
import pytest

from aerof_dev_b200 import workloads as W

GOLD_F77 = os.path.join(os.path.dirname(__file__), "golden", "reference_fortran.npz")
BC_INLET_MOVING = -4


@pytest.fixture(scope="module")
def gold_f77():
    return np.load(GOLD_F77)


def test_roeflux7_type1_bitwise(oracle_mod, gold_f77):
    ins, outs = gold_f77["roe_sa_in"], gold_f77["roe_sa_out"]
    assert len(ins) >= 300 and (outs[:, 0] < 0).any() and (outs[:, 0] > 0).any()
    for r, o in zip(ins, outs):
        assert np.array_equal(oracle_mod.roeflux7_sa(1.4, r[0:3], r[3:9], r[9:15]), o)


def test_boundflux5_type1_bitwise(oracle_mod, gold_f77):
    ins, outs = gold_f77["bf_sa_in"], gold_f77["bf_sa_out"]
    for r, o in zip(ins, outs):
        assert np.array_equal(oracle_mod.face_flux_sa(1.4, BC_INLET_MOVING, r[0:3], r[3:9], r[9:15]), o)


@pytest.fixture(scope="module")
def mesh_sa(oracle_mod):
    m = W.make_lattice_mesh(7, jitter=0.2, codes="channel")
    return m, oracle_mod.Oracle(m)


@pytest.mark.parametrize("order,model", [(1, 1), (2, 1), (2, 2), (3, 1)])
def test_zero_eddy_viscosity_is_the_laminar_residual(mesh_sa, order, model):
    # nu~ = 0 everywhere: mu_t = 0, no SA diffusion, no source, no nu~
    # flux; the first five components are the laminar Navier-Stokes
    # residual bit for bit and the sixth is zero
    m, o = mesh_sa
    U5 = W.perturbed_state(o.N, 0.8)
    U6 = np.column_stack([U5, np.zeros(o.N)])
    Ub6 = np.concatenate([W.freestream(0.8), [0.0]])
    d = 0.1 + m["X"][:, 2]
    kw = dict(order=order, model=model, reynolds=500.0, alpha=1.2, Ts=0.4)
    R6, e6 = o.residual_sa(U6, Ub6, d, **kw)
    R5, e5 = o.residual_visc(U5, W.freestream(0.8), **kw)
    assert e6 == e5
    assert np.array_equal(R6[:, :5], R5)
    assert not R6[:, 5].any()


def test_uniform_nu_tilde_is_advected_with_the_mass_flux(mesh_sa):
    # inviscid part only (model 0): a uniform nu~ is carried by the mass
    # flux, so R[5] = nu~ R[0] at every node (the continuity residual
    # weighted by the upwind nu~, which is the same on both sides)
    m, o = mesh_sa
    U5 = W.perturbed_state(o.N, 0.8)
    nu = 3e-3
    U6 = np.column_stack([U5, nu * U5[:, 0]])
    Ub6 = np.concatenate([W.freestream(0.8), [nu * W.freestream(0.8)[0]]])
    R6, _ = o.residual_sa(U6, Ub6, np.ones(o.N), order=2, model=0)
    R5, _ = o.residual(U5, W.freestream(0.8), 2)
    assert np.array_equal(R6[:, :5], R5)
    assert np.allclose(R6[:, 5], nu * R6[:, 0], rtol=1e-12, atol=1e-15 * np.abs(R6[:, 0]).max())


def test_source_and_diffusion_change_only_the_sixth_row_through_mu_t(mesh_sa):
    # with nu~ > 0 the sixth component gains diffusion and source terms and
    # the momentum and energy rows gain the eddy viscosity; far from walls
    # (d large) the destruction term vanishes and the sixth row grows with
    # the production, so R[5] decreases (R = -dU/dt) when d grows
    m, o = mesh_sa
    U5 = W.perturbed_state(o.N, 0.8)
    U6 = np.column_stack([U5, 5e-3 * U5[:, 0]])
    Ub6 = np.concatenate([W.freestream(0.8), [5e-3]])
    near, _ = o.residual_sa(U6, Ub6, np.full(o.N, 1e-3), order=2, model=1, reynolds=1e3)
    far, _ = o.residual_sa(U6, Ub6, np.full(o.N, 1e3), order=2, model=1, reynolds=1e3)
    assert np.array_equal(near[:, :5], far[:, :5])
    assert near[:, 5].sum() > far[:, 5].sum()
