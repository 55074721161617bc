"""Decomposed solvers (aerof_dev_b200.decomposition / .distributed) against
the single-domain oracle, on the CPU: subdomains of owned nodes plus two
ghost layers, ghost states exchanged before every operator, owned-row sums
reduced over ranks.  Pieces run in one process, and as two gloo ranks
(torch.distributed, 127.0.0.1); the owned rows must equal the single-domain
results (residual and RK2 to 1e-12, the converged Newton state to 1e-9)."""
import os
import socket

import numpy as np
import pytest
import torch

from aerof_dev_b200 import decomposition as D
from aerof_dev_b200 import distributed as DS
from aerof_dev_b200 import workloads as W
from conftest import rel_l2
from dist_oracle_backend import OracleBackend


def _case(n=9, codes="channel", jit=0.2, mach=0.8):
    m = W.make_lattice_mesh(n, jitter=jit, codes=codes)
    Ub = W.freestream(mach)
    U = W.perturbed_state(m["X"].shape[0], mach)
    return m, Ub, U


def test_rcb_and_subdomain_structure():
    m, Ub, U = _case(9)
    N = m["X"].shape[0]
    owner = D.rcb(m["X"], 4)
    assert sorted(np.bincount(owner).tolist()) == sorted([N // 4 + (i < N % 4) for i in range(4)])
    subs = D.decompose(m, owner)
    got = np.concatenate([s.l2g[: s.n_owned] for s in subs])
    assert np.array_equal(np.sort(got), np.arange(N))          # every node owned once
    for s in subs:
        assert np.all(owner[s.l2g[: s.n_owned]] == s.rank)
        assert np.all(owner[s.l2g[s.n_owned:]] != s.rank)
        for r, rows in s.recv.items():                          # send/recv lists pair up
            assert np.array_equal(s.l2g[rows], subs[r].l2g[subs[r].send[s.rank]])


@pytest.mark.parametrize("parts", [2, 3])
def test_residual_and_rk2_in_one_process(oracle_mod, parts):
    m, Ub, U = _case(9)
    N = U.shape[0]
    subs = D.decompose(m, D.rcb(m["X"], parts))
    team = DS.Team([(s, OracleBackend(oracle_mod, s, Ub)) for s in subs])
    Ul = [torch.from_numpy(D.scatter_local(s, U)) for s in subs]
    for s, u in zip(subs, Ul):
        u[s.n_owned:] = 0.0                       # ghosts come from the exchange only
    R, bad = team.residual(Ul)
    o = oracle_mod.Oracle(m)
    Rr, bad_r = o.residual(U, Ub, 2)
    assert bad == bad_r == 0
    assert rel_l2(D.gather_owned(subs, [r.numpy() for r in R], N), Rr) <= 1e-12
    # explicit RK2, first order, far field (the CPU-runnable configuration)
    m1, Ub1, U1 = _case(9, codes="farfield", jit=0.0, mach=0.5)
    subs1 = D.decompose(m1, D.rcb(m1["X"], parts))
    team1 = DS.Team([(s, OracleBackend(oracle_mod, s, Ub1, order=1)) for s in subs1])
    Uo = team1.rk2([torch.from_numpy(D.scatter_local(s, U1)) for s in subs1], 0.8, 10)
    Ur = oracle_mod.Oracle(m1).rk2(U1, Ub1, 1, 0.8, 10)
    assert rel_l2(D.gather_owned(subs1, [u.numpy() for u in Uo], N), Ur) <= 1e-12


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_worker(rank, world, port, out):
    import torch.distributed as dist
    from oracle import oracle as oracle_mod
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m, Ub, U = _case(7, jit=0.1)
        U = W.perturbed_state(U.shape[0], 0.8, amp=0.02)
        subs = D.decompose(m, D.rcb(m["X"], world))
        sub = subs[rank]
        team = DS.Team([(sub, OracleBackend(oracle_mod, sub, Ub))], comm=dist.group.WORLD)
        u = torch.from_numpy(D.scatter_local(sub, U))
        R, bad = team.residual([u])
        Un, info = team.newton([u], tol=1e-8, max_steps=300)
        out[rank] = (sub.l2g[: sub.n_owned], R[0][: sub.n_owned].numpy(), Un[0][: sub.n_owned].numpy(), info, bad)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_residual_and_newton(oracle_mod):
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_rank_worker, args=(world, port, out), nprocs=world, join=True)
    m, Ub, U = _case(7, jit=0.1)
    U = W.perturbed_state(U.shape[0], 0.8, amp=0.02)
    N = U.shape[0]
    o = oracle_mod.Oracle(m)
    R = np.empty((N, 5))
    Un = np.empty((N, 5))
    for r in range(world):
        ids, Rr, Ur, info, bad = out[r]
        R[ids] = Rr
        Un[ids] = Ur
        assert bad == 0
        assert info["rel_residual"] <= 1e-8
    assert rel_l2(R, o.residual(U, Ub, 2)[0]) <= 1e-12
    Uref, hist, _ = o.newton(U, Ub, order=2, tol=1e-8, max_steps=300, fp32_prec=False)
    assert abs(out[0][3]["steps"] - (len(hist) - 1)) <= 2
    assert rel_l2(Un, Uref) <= 1e-9
