"""The oracle's block ILU(0) restatement (SparseMat::numericILU / lusol in
the multicolour ordering): a valid colouring, identity with block-Jacobi for
a block-diagonal operator, and a stronger preconditioner than block-Jacobi
on an H1 Jacobian (CPU only)."""
import numpy as np
import pytest

from aerof_dev_b200 import workloads as W


@pytest.fixture(scope="module")
def system(oracle_mod):
    m = W.make_lattice_mesh(7, jitter=0.2, codes="channel")
    o = oracle_mod.Oracle(m)
    U = W.perturbed_state(o.N, 0.8)
    Ub = W.freestream(0.8)
    A = o.jacobian(U, Ub, o.timestep(U, 100.0))
    return o, A


def test_colouring_is_proper(system):
    o, A = system
    _, bad, nc, colour = o.ilu0(A, np.zeros((o.N, 5)))
    assert bad == 0 and nc == colour.max() + 1
    e = o.edges()
    assert np.all(colour[e[:, 0]] != colour[e[:, 1]])
    # greedy in ascending node order: every node's colour is the smallest
    # one not taken by a lower-numbered neighbour
    for i in range(o.N):
        lower = {colour[j] for j in np.concatenate([e[e[:, 1] == i, 0], e[e[:, 0] == i, 1]]) if j < i}
        assert colour[i] == min(set(range(nc + 1)) - lower)


def test_block_diagonal_equals_block_jacobi(system):
    o, A = system
    A2 = A.copy()
    A2[o.N:] = 0.0
    x = np.random.default_rng(1).standard_normal((o.N, 5))
    D, _ = o.bj_invert(A2, fp32=False)
    for tr in (False, True):
        y, bad, _, _ = o.ilu0(A2, x, fp32=False, transpose=tr)
        ref = np.einsum("nji,nj->ni" if tr else "nij,nj->ni", D, x)
        assert bad == 0
        assert np.abs(y - ref).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.parametrize("tr", [False, True])
def test_stronger_than_block_jacobi(system, tr):
    # 20 Richardson steps x += M^-1 (b - A x)
    o, A = system
    D, _ = o.bj_invert(A, fp32=False)
    b = np.random.default_rng(2).standard_normal((o.N, 5))
    out = {}
    for name in ("bj", "ilu"):
        x = np.zeros_like(b)
        for _ in range(20):
            r = b - o.matvec(A, x, transpose=tr)
            if name == "bj":
                x = x + np.einsum("nji,nj->ni" if tr else "nij,nj->ni", D, r)
            else:
                x = x + o.ilu0(A, r, fp32=False, transpose=tr)[0]
        out[name] = np.linalg.norm(b - o.matvec(A, x, transpose=tr)) / np.linalg.norm(b)
    assert out["ilu"] < 0.1 * out["bj"]


def test_rcm_order_is_a_breadth_first_permutation(system):
    # reverse Cuthill-McKee (renumRCM): a permutation of the nodes whose
    # reversal visits every node after at least one already visited
    # neighbour (breadth-first from the pseudo-peripheral end node)
    o, A = system
    order = o.rcm_order()
    assert sorted(order.tolist()) == list(range(o.N))
    e = o.edges()
    nb = [set() for _ in range(o.N)]
    for a, b in e:
        nb[a].add(b); nb[b].add(a)
    seen = {int(order[-1])}
    for v in order[::-1][1:]:
        assert nb[int(v)] & seen
        seen.add(int(v))


@pytest.mark.parametrize("cfl", [100.0, 1e4])
def test_rcm_ilu_converges_in_fewer_iterations_than_multicolour(system, cfl):
    # the price of the multicolour ordering the GPU sweeps use: the
    # reference's RCM-ordered ILU(0) (PcData::renumbering = RCM) needs fewer
    # GMRES iterations on the same H1 system; both beat block-Jacobi
    o, _ = system
    U = W.perturbed_state(o.N, 0.8)
    Ub = W.freestream(0.8)
    A = o.jacobian(U, Ub, o.timestep(U, cfl))
    b = -o.residual(U, Ub, 2)[0]
    D, _ = o.bj_invert(A)
    _, its_bj, _ = o.gmres(A, D, b, maxits=2000, eps=1e-6)
    _, its_col, r_col = o.gmres_ilu(A, b, None, maxits=2000, eps=1e-6)
    _, its_rcm, r_rcm = o.gmres_ilu(A, b, o.rcm_order(), maxits=2000, eps=1e-6)
    bn = np.linalg.norm(b)
    assert r_col <= 1e-6 * bn and r_rcm <= 1e-6 * bn
    assert its_rcm < its_col < its_bj
