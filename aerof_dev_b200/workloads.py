"""Seeded synthetic workloads for the edge-based finite-volume hot path.

AERO-F reads pre-partitioned meshes in its sower binary format
(``GeoSource.C:94-444``); no public mesh or dataset is involved in the
hot-path benchmarks, so this module builds the stand-in inputs:

* a unit-cube tetrahedral mesh from an ``n^3`` node lattice, each hex split
  into 6 positively oriented tets by the Kuhn (Freudenthal) split along the
  (0,0,0)->(1,1,1) diagonal, so face diagonals agree between neighbours;
* interior-node jitter, uniform in +-``jitter*h`` per coordinate;
* boundary triangles ordered so that ``0.5*((x2-x0)^(x1-x0))`` points out
  of the domain, the orientation ``FaceTria::computeNormal``
  (``FaceTriaCore.C:31-48``) assumes;
* boundary codes from ``BcDef.h``: ``BC_INLET_MOVING=-4``,
  ``BC_OUTLET_MOVING=-5``, ``BC_SLIP_WALL_MOVING=-2``;
* the nondimensional free stream of ``IoDataCore.C:7019-7027`` (rho=1,
  |u|=1 along +x, p=1/(gamma M^2)) plus a seeded perturbation.

Sizes (exact for the Kuhn split): N=n^3, T=6(n-1)^3,
E=3n^2(n-1)+3n(n-1)^2+(n-1)^3, F_b=12(n-1)^2.
"""
from __future__ import annotations

import numpy as np

BC_SLIP_WALL_MOVING = -2
BC_INLET_MOVING = -4
BC_OUTLET_MOVING = -5
BC_INTERNAL = 0

DEFAULT_SEED = 20261203


def lattice_sizes(n: int) -> dict:
    m = n - 1
    return {"N": n ** 3, "T": 6 * m ** 3,
            "E": 3 * n * n * m + 3 * n * m * m + m ** 3, "F": 12 * m * m}


def _kuhn_tets(n: int) -> np.ndarray:
    """Six positively oriented tets per hex cell of an n^3 lattice."""
    m = n - 1
    i, j, k = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    # lexicographic node id: x fastest
    base = (i + n * j + n * n * k).astype(np.int64).reshape(-1)
    step = np.array([1, n, n * n], dtype=np.int64)
    # the 6 axis orders; vertices walk 000 -> e_a -> e_a+e_b -> 111
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    out = np.empty((base.size, 6, 4), dtype=np.int64)
    for p, (a, b, c) in enumerate(perms):
        v0 = base
        v1 = base + step[a]
        v2 = v1 + step[b]
        v3 = v2 + step[c]
        # even permutations of (x,y,z) keep det > 0; odd ones swap v1 and v2
        even = (a, b, c) in [(0, 1, 2), (1, 2, 0), (2, 0, 1)]
        if even:
            out[:, p] = np.stack([v0, v1, v2, v3], axis=1)
        else:
            out[:, p] = np.stack([v0, v2, v1, v3], axis=1)
    return out.reshape(-1, 4).astype(np.int32)


def _boundary_faces(n: int, X: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Boundary triangles (outward by 0.5*((x2-x0)^(x1-x0))) and side ids.

    Each boundary square is split along the diagonal from its low corner to
    its high corner, which is the tet face the Kuhn split puts there.
    side: 0:x=0 1:x=1 2:y=0 3:y=1 4:z=0 5:z=1.
    """
    m = n - 1
    a, b = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    a = a.reshape(-1).astype(np.int64)
    b = b.reshape(-1).astype(np.int64)
    tris, sides = [], []

    def nid(x, y, z):
        return x + n * y + n * n * z

    for side, (axis, val) in enumerate([(0, 0), (0, m), (1, 0), (1, m), (2, 0), (2, m)]):
        fixed = np.full_like(a, val)
        if axis == 0:
            c00 = nid(fixed, a, b); c10 = nid(fixed, a + 1, b)
            c01 = nid(fixed, a, b + 1); c11 = nid(fixed, a + 1, b + 1)
        elif axis == 1:
            c00 = nid(a, fixed, b); c10 = nid(a + 1, fixed, b)
            c01 = nid(a, fixed, b + 1); c11 = nid(a + 1, fixed, b + 1)
        else:
            c00 = nid(a, b, fixed); c10 = nid(a + 1, b, fixed)
            c01 = nid(a, b + 1, fixed); c11 = nid(a + 1, b + 1, fixed)
        t1 = np.stack([c00, c10, c11], axis=1)
        t2 = np.stack([c00, c11, c01], axis=1)
        t = np.stack([t1, t2], axis=1).reshape(-1, 3)
        tris.append(t)
        sides.append(np.full(t.shape[0], side, dtype=np.int32))
    tris = np.concatenate(tris)
    sides = np.concatenate(sides)
    # orient outward
    x0, x1, x2 = X[tris[:, 0]], X[tris[:, 1]], X[tris[:, 2]]
    nrm = 0.5 * np.cross(x2 - x0, x1 - x0)
    outward = np.zeros((6, 3))
    outward[0, 0] = -1; outward[1, 0] = 1; outward[2, 1] = -1
    outward[3, 1] = 1; outward[4, 2] = -1; outward[5, 2] = 1
    flip = np.einsum("ij,ij->i", nrm, outward[sides]) < 0
    tris[flip] = tris[flip][:, [0, 2, 1]]
    return tris.astype(np.int32), sides


def make_lattice_mesh(n: int, jitter: float = 0.0, seed: int = DEFAULT_SEED,
                      codes: str = "farfield") -> dict:
    """Unit-cube Kuhn tet mesh.

    codes="farfield": x=0 faces inlet (-4), every other face outlet (-5).
    codes="channel":  x=0 inlet (-4), x=1 outlet (-5), y/z faces slip wall (-2).
    """
    h = 1.0 / (n - 1)
    g = np.arange(n, dtype=np.float64) * h
    zz, yy, xx = np.meshgrid(g, g, g, indexing="ij")
    X = np.stack([xx.reshape(-1), yy.reshape(-1), zz.reshape(-1)], axis=1)
    if jitter > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        d = rng.uniform(-jitter * h, jitter * h, size=X.shape)
        idx = np.arange(n)
        iz, iy, ix = np.meshgrid(idx, idx, idx, indexing="ij")
        interior = ((ix > 0) & (ix < n - 1) & (iy > 0) & (iy < n - 1)
                    & (iz > 0) & (iz < n - 1)).reshape(-1)
        X[interior] += d[interior]
    tets = _kuhn_tets(n)
    faces, sides = _boundary_faces(n, X)
    if codes == "farfield":
        code = np.where(sides == 0, BC_INLET_MOVING, BC_OUTLET_MOVING)
    elif codes == "channel":
        code = np.where(sides == 0, BC_INLET_MOVING,
                        np.where(sides == 1, BC_OUTLET_MOVING, BC_SLIP_WALL_MOVING))
    else:
        raise ValueError(f"unknown boundary layout {codes!r}")
    return {"n": n, "X": np.ascontiguousarray(X), "tets": np.ascontiguousarray(tets),
            "faces": np.ascontiguousarray(faces), "codes": code.astype(np.int32),
            "sides": sides}


def freestream(mach: float, gamma: float = 1.4) -> np.ndarray:
    """Conservative free stream (rho, rho u, rho v, rho w, E): rho=1, u=(1,0,0),
    p = 1/(gamma M^2)  (IoDataCore.C:7019-7027, DistBcData.C:679-700)."""
    p = 1.0 / (gamma * mach * mach)
    return np.array([1.0, 1.0, 0.0, 0.0, p / (gamma - 1.0) + 0.5])


def prim_to_cons(V: np.ndarray, gamma: float = 1.4) -> np.ndarray:
    U = np.empty_like(V)
    U[:, 0] = V[:, 0]
    U[:, 1:4] = V[:, 0:1] * V[:, 1:4]
    U[:, 4] = V[:, 4] / (gamma - 1.0) + 0.5 * V[:, 0] * np.sum(V[:, 1:4] ** 2, axis=1)
    return U


def perturbed_state(N: int, mach: float, amp: float = 0.01, seed: int = DEFAULT_SEED,
                    gamma: float = 1.4) -> np.ndarray:
    """Free stream with a seeded multiplicative perturbation of rho and p and
    an additive one on each velocity component, returned as U[N][5]."""
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    p = 1.0 / (gamma * mach * mach)
    V = np.empty((N, 5))
    V[:, 0] = 1.0 * (1.0 + amp * rng.standard_normal(N))
    V[:, 1] = 1.0 + amp * rng.standard_normal(N)
    V[:, 2] = amp * rng.standard_normal(N)
    V[:, 3] = amp * rng.standard_normal(N)
    V[:, 4] = p * (1.0 + amp * rng.standard_normal(N))
    return prim_to_cons(V, gamma)


def smooth_state(X: np.ndarray, mach: float, amp: float = 0.02, gamma: float = 1.4) -> np.ndarray:
    """Free stream plus a smooth sinusoidal disturbance (for adjoint/FD checks,
    where a smooth field keeps van Albada away from its a*b==0 kink)."""
    p = 1.0 / (gamma * mach * mach)
    s = np.sin(np.pi * X[:, 0]) * np.sin(np.pi * X[:, 1]) * np.sin(np.pi * X[:, 2])
    c = np.cos(2.0 * np.pi * X[:, 0]) * np.sin(np.pi * X[:, 2])
    # a generic linear ramp per component keeps every edge difference away
    # from exactly zero (van Albada switches branch at a*b == 0)
    d = np.array([[1.0, 0.37, 0.61], [0.43, 1.0, 0.29], [0.71, 0.23, 1.0], [0.19, 0.83, 0.47],
                  [0.57, 0.31, 0.89]])
    lin = X @ d.T
    V = np.empty((X.shape[0], 5))
    V[:, 0] = 1.0 + amp * (s + 0.3 * lin[:, 0])
    V[:, 1] = 1.0 + amp * (c + 0.3 * lin[:, 1])
    V[:, 2] = amp * (0.5 * s + 0.3 * lin[:, 2])
    V[:, 3] = amp * (-0.5 * c + 0.3 * lin[:, 3])
    V[:, 4] = p * (1.0 + amp * (s + 0.5 * c + 0.3 * lin[:, 4]))
    return prim_to_cons(V, gamma)


def shape_modes(X: np.ndarray, n_modes: int, seed: int = DEFAULT_SEED, sigma: float = 0.1,
                amplitude: float = 1.0) -> np.ndarray:
    """Gaussian-bump shape modes on z=0, decaying linearly to 0 at z=1.

    Mode k displaces z by a*exp(-((x-xk)^2+(y-yk)^2)/(2 sigma^2))*(1-z), with
    seeded centres (xk, yk) in [0.2, 0.8]^2. Returned as [n_modes][N][3].
    """
    rng = np.random.Generator(np.random.PCG64(seed + 2))
    cen = rng.uniform(0.2, 0.8, size=(n_modes, 2))
    out = np.zeros((n_modes, X.shape[0], 3))
    for k in range(n_modes):
        r2 = (X[:, 0] - cen[k, 0]) ** 2 + (X[:, 1] - cen[k, 1]) ** 2
        out[k, :, 2] = amplitude * np.exp(-r2 / (2 * sigma * sigma)) * (1.0 - X[:, 2])
    return out
