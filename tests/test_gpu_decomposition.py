"""Decomposed solvers on the GPU: several subdomain pieces, each on its own
CUDA context through the C ABI, in one process (ghost rows copied between
the pieces' device arrays; no kernel waits on another).  Owned rows against
the single-domain oracle: residual 1e-12, RK2 1e-12, converged Newton state
1e-9 (FP64 operator) and 1e-7 (FP32 operator)."""
import numpy as np
import pytest
import torch

from aerof_dev_b200 import decomposition as D
from aerof_dev_b200 import distributed as DS
from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _team(gpu_lib, m, Ub, parts, rec=2):
    subs = D.decompose(m, D.rcb(m["X"], parts))
    return subs, DS.Team([(s, DS.GpuBackend(s, Ub, reconstruction=rec)) for s in subs])


def _local(subs, U):
    return [torch.from_numpy(D.scatter_local(s, U)).cuda() for s in subs]


@pytest.mark.parametrize("parts", [2, 4])
def test_gpu_pieces_residual_and_rk2(gpu_lib, oracle_mod, parts):
    m = W.make_lattice_mesh(13, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    U = W.perturbed_state(m["X"].shape[0], 0.8)
    N = U.shape[0]
    subs, team = _team(gpu_lib, m, Ub, parts)
    R, bad = team.residual(_local(subs, U))
    Rr, bad_r = oracle_mod.Oracle(m).residual(U, Ub, 2)
    assert bad == bad_r == 0
    assert rel_l2(D.gather_owned(subs, [r.cpu().numpy() for r in R], N), Rr) <= 1e-12
    m1 = W.make_lattice_mesh(11, codes="farfield")
    Ub1 = W.freestream(0.5)
    U1 = W.perturbed_state(m1["X"].shape[0], 0.5)
    subs1, team1 = _team(gpu_lib, m1, Ub1, parts, rec=1)
    Uo = team1.rk2(_local(subs1, U1), 0.8, 10)
    Ur = oracle_mod.Oracle(m1).rk2(U1, Ub1, 1, 0.8, 10)
    assert rel_l2(D.gather_owned(subs1, [u.cpu().numpy() for u in Uo], m1["X"].shape[0]), Ur) <= 1e-12
    for be in team.backends + team1.backends:
        be.close()


@pytest.mark.parametrize("prec", [64, 32])
def test_gpu_pieces_newton(gpu_lib, oracle_mod, prec):
    m = W.make_lattice_mesh(9, jitter=0.1, codes="channel")
    Ub = W.freestream(0.8)
    U = W.perturbed_state(m["X"].shape[0], 0.8, amp=0.02)
    subs, team = _team(gpu_lib, m, Ub, 3)
    Uo, info = team.newton(_local(subs, U), tol=1e-8, max_steps=300, precision=prec)
    assert info["rel_residual"] <= 1e-8
    Uref, hist, _ = oracle_mod.Oracle(m).newton(U, Ub, order=2, tol=1e-8, max_steps=300, fp32_prec=False)
    got = D.gather_owned(subs, [u.cpu().numpy() for u in Uo], U.shape[0])
    assert rel_l2(got, Uref) <= (1e-9 if prec == 64 else 1e-7)
    for be in team.backends:
        be.close()


def test_gpu_pieces_from_sower_files(gpu_lib, oracle_mod, tmp_path):
    # a mesh written in AERO-F's pre-partitioned format and read back: the
    # single-domain residual is unchanged, and GPU pieces built from the
    # files' subdomains (the reference's ownership rule) give it too
    from aerof_dev_b200 import sower
    m = W.make_lattice_mesh(11, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    U = W.perturbed_state(m["X"].shape[0], 0.8)
    names = sower.write(str(tmp_path / "mesh"), m, sower.element_partition(m, 3))
    gs = sower.GeoSource(names["con"], names["geo"], names["dec"])
    g = gs.global_mesh()
    R0, _ = gpu_lib.SpaceOperator(gpu_lib.Context.from_mesh(m, Ub)).computeResidual(U)
    R1, _ = gpu_lib.SpaceOperator(gpu_lib.Context.from_mesh(g, Ub)).computeResidual(U)
    assert np.array_equal(R0, R1)
    subs = D.decompose(g, gs.owners())
    team = DS.Team([(s, DS.GpuBackend(s, Ub)) for s in subs])
    R, _ = team.residual(_local(subs, U))
    assert rel_l2(D.gather_owned(subs, [r.cpu().numpy() for r in R], U.shape[0]), R0) <= 1e-12
    for be in team.backends:
        be.close()
    gs.close()
