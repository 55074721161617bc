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
