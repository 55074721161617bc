"""Domain decomposition of the edge-based finite-volume mesh for several
GPUs (one subdomain per rank).

AERO-F partitions the mesh by elements into subdomains that share their
interface nodes; every edge pass computes partial sums on each subdomain
and adds them over the shared nodes (``CommPattern::exchange`` after the
gradients, Domain.C:222-225, and after the fluxes, Domain.C:920-928, and
after the H1 product, MatVecProd.C:1178-1185), with ``globalSum`` for the
Krylov dot products (DistVector.h:1493-1495).

Here a subdomain is the set of nodes a rank owns plus two ghost layers:
all tets that touch an owned node or a first-layer neighbour of one.  With
current states on both ghost layers the unmodified single-GPU kernels give
the owned rows exactly (every edge, face, control volume and least-squares
neighbourhood of an owned node, and every least-squares neighbourhood of a
first-layer node, lies inside the subdomain), so one exchange of the ghost
states per residual replaces the reference's two partial-sum assemblies,
and no kernel needs edge ownership masks.  The owned rows come first in
the local numbering, so reductions over owned rows are prefix sums.

Owners can come from recursive coordinate bisection (``rcb``) or from a
decomposition read from the reference's files (``sower.GeoSource``: the
lowest-numbered subdomain sharing a node owns it, as the reference's
masterFlag rule does).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def rcb(X: np.ndarray, nparts: int) -> np.ndarray:
    """Recursive coordinate bisection of the nodes: owner[N] in [0, nparts),
    splitting the longest extent at the weighted median each time."""
    owner = np.zeros(X.shape[0], dtype=np.int32)

    def split(idx: np.ndarray, p0: int, p: int):
        if p == 1:
            owner[idx] = p0
            return
        pl = p // 2
        ext = X[idx].max(0) - X[idx].min(0)
        ax = int(np.argmax(ext))
        order = idx[np.argsort(X[idx, ax], kind="stable")]
        cut = (len(order) * pl) // p
        split(order[:cut], p0, pl)
        split(order[cut:], p0 + pl, p - pl)

    split(np.arange(X.shape[0]), 0, nparts)
    return owner


def _neighbours(tets: np.ndarray, N: int):
    """Node adjacency (CSR) from the tets' six edges."""
    pairs = tets[:, [0, 0, 0, 1, 1, 2, 1, 2, 3, 2, 3, 3]].reshape(-1, 2, 6).transpose(0, 2, 1).reshape(-1, 2)
    a = np.concatenate([pairs[:, 0], pairs[:, 1]]).astype(np.int64)
    b = np.concatenate([pairs[:, 1], pairs[:, 0]]).astype(np.int64)
    key = np.unique(a * N + b)
    rows, cols = key // N, key % N
    ptr = np.zeros(N + 1, dtype=np.int64)
    np.add.at(ptr, rows + 1, 1)
    return np.cumsum(ptr), cols


@dataclass
class Subdomain:
    """One rank's piece: a mesh in local numbering (owned nodes first, then
    ghosts) and its exchange lists."""
    rank: int
    nparts: int
    l2g: np.ndarray            # [n_local] global node ids
    n_owned: int
    mesh: dict                 # X, tets, faces, codes in local numbering (+ sides when given)
    # per neighbour rank s: local rows this rank receives from s (ghosts owned
    # by s), and local rows it sends to s (owned rows that are ghosts there),
    # both in ascending global id, so the two sides pair up
    recv: dict = field(default_factory=dict)
    send: dict = field(default_factory=dict)

    @property
    def n_local(self) -> int:
        return int(self.l2g.size)


def decompose(mesh: dict, owner: np.ndarray) -> list[Subdomain]:
    """Ghost-layer subdomains of a global mesh {X, tets, faces, codes} for
    the node owners owner[N] (ranks 0..P-1)."""
    X, tets, faces, codes = mesh["X"], mesh["tets"], mesh["faces"], mesh["codes"]
    N = X.shape[0]
    P = int(owner.max()) + 1
    ptr, nbr = _neighbours(tets, N)
    subs = []
    for r in range(P):
        own = owner == r
        # first ghost layer: neighbours of owned nodes that are not owned
        oidx = np.nonzero(own)[0]
        deg = ptr[oidx + 1] - ptr[oidx]
        nb = nbr[np.repeat(ptr[oidx], deg) + (np.arange(deg.sum()) - np.repeat(np.cumsum(deg) - deg, deg))]
        l1 = np.zeros(N, dtype=bool)
        l1[nb] = True
        l1 &= ~own
        core = own | l1
        tsel = core[tets].any(axis=1)
        ltets = tets[tsel]
        used = np.zeros(N, dtype=bool)
        used[ltets.ravel()] = True
        owned_ids = np.nonzero(own)[0]
        ghost_ids = np.nonzero(used & ~own)[0]
        l2g = np.concatenate([owned_ids, ghost_ids]).astype(np.int64)
        g2l = np.full(N, -1, dtype=np.int64)
        g2l[l2g] = np.arange(l2g.size)
        fsel = core[faces].any(axis=1) & (g2l[faces] >= 0).all(axis=1)
        lm = {"X": X[l2g].copy(), "tets": g2l[ltets].astype(np.int32), "faces": g2l[faces[fsel]].astype(np.int32),
              "codes": codes[fsel].copy()}
        if "sides" in mesh:
            lm["sides"] = mesh["sides"][fsel].copy()
        sub = Subdomain(rank=r, nparts=P, l2g=l2g, n_owned=int(owned_ids.size), mesh=lm)
        gown = owner[ghost_ids]
        for s in np.unique(gown):
            sub.recv[int(s)] = (owned_ids.size + np.nonzero(gown == s)[0]).astype(np.int64)
        subs.append(sub)
    # send lists: what each neighbour receives from this rank, in the same
    # global order, as local rows here
    for r, sub in enumerate(subs):
        for s, rows in sub.recv.items():
            gids = sub.l2g[rows]
            peer = subs[s]
            g2l_peer = {int(g): i for i, g in enumerate(peer.l2g[: peer.n_owned])}
            peer.send[r] = np.array([g2l_peer[int(g)] for g in gids], dtype=np.int64)
    return subs


def gather_owned(subs: list[Subdomain], parts: list[np.ndarray], N: int) -> np.ndarray:
    """Global array from each subdomain's owned rows."""
    out = np.empty((N,) + parts[0].shape[1:], dtype=parts[0].dtype)
    for sub, a in zip(subs, parts):
        out[sub.l2g[: sub.n_owned]] = a[: sub.n_owned]
    return out


def scatter_local(sub: Subdomain, a: np.ndarray) -> np.ndarray:
    """A subdomain's local copy (owned and ghost rows) of a global array."""
    return np.ascontiguousarray(a[sub.l2g])
