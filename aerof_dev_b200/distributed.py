"""Solvers over a decomposed mesh (decomposition.Subdomain pieces).

A ``Team`` holds the pieces this process computes and the means to talk to
the others:

* several pieces in one process (``comm=None``): ghost rows are copied
  between the pieces' arrays directly;
* one piece per rank (``comm`` = a torch.distributed process group): ghost
  rows travel with one batched send/receive per neighbour pair
  (``batch_isend_irecv``: NCCL point-to-point over NVLink for CUDA tensors,
  gloo for CPU tensors), and the owned-row sums of the Krylov dot products
  are added with ``all_reduce`` (the reference's CommPattern::exchange and
  Communicator::globalSum, Communicator.C:323-347, 392).

Each piece has a backend that evaluates the single-domain operators on its
local mesh: ``GpuBackend`` runs them through the C ABI on the piece's own
CUDA context.  Vectors are torch tensors [n_local, 5] (CPU or CUDA); only
owned rows are meaningful after a local operator, and ghost rows are
refreshed by ``exchange`` before every operator that reads them.

The algorithms restate the single-GPU ones at the host level: the
residual (SpaceOperator::computeResidual), Heun RK2
(ExplicitTsDesc::computeRKSecondOrder, ExplicitTsDesc.C:98-117), and the
pseudo-transient Newton with right-preconditioned GMRES(m), MGS and Givens
rotations (NewtonSolver.h:70-231, KspSolver.C:351-492, 917-982) with the
RESIDUAL CFL law and the physical-solution check.
"""
from __future__ import annotations

import math

import numpy as np

from .decomposition import Subdomain


class Team:
    def __init__(self, pieces: list, comm=None):
        """pieces: [(Subdomain, backend)]; comm: None or a torch.distributed
        group (then exactly one piece, whose rank is the process's rank)."""
        self.subs = [p[0] for p in pieces]
        self.backends = [p[1] for p in pieces]
        self.comm = comm
        if comm is not None and len(pieces) != 1:
            raise ValueError("with a process group every rank holds one piece")

    # ---------------------------------------------------------------- comms
    def exchange(self, fields: list):
        """Ghost rows of every piece's field from their owners (in place)."""
        import torch
        if self.comm is None:
            by_rank = {sub.rank: f for sub, f in zip(self.subs, fields)}
            for sub, f in zip(self.subs, fields):
                for s, rows in sub.recv.items():
                    src = by_rank[s]
                    peer = self.subs[[x.rank for x in self.subs].index(s)]
                    f[torch.as_tensor(rows, device=f.device)] = src[torch.as_tensor(peer.send[sub.rank],
                                                                                    device=src.device)]
            return
        import torch.distributed as dist
        sub, f = self.subs[0], fields[0]
        ops, recv_bufs = [], []
        for s in sorted(set(sub.send) | set(sub.recv)):
            if s in sub.send:
                buf = f[torch.as_tensor(sub.send[s], device=f.device)].contiguous()
                ops.append(dist.P2POp(dist.isend, buf, s, group=self.comm))
            if s in sub.recv:
                rb = torch.empty((len(sub.recv[s]),) + tuple(f.shape[1:]), dtype=f.dtype, device=f.device)
                recv_bufs.append((s, rb))
                ops.append(dist.P2POp(dist.irecv, rb, s, group=self.comm))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for s, rb in recv_bufs:
            f[torch.as_tensor(sub.recv[s], device=f.device)] = rb

    def allsum(self, values: list) -> float:
        """Sum of the pieces' (owned-row) partial values over all ranks."""
        local = 0.0
        for v in values:
            local += float(v)
        if self.comm is None:
            return local
        import torch
        import torch.distributed as dist
        dev = self.backends[0].device
        t = torch.tensor([local], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.comm)
        return float(t.item())

    def allmax_int(self, values: list) -> int:
        local = sum(int(v) for v in values)
        if self.comm is None:
            return local
        import torch
        import torch.distributed as dist
        t = torch.tensor([local], dtype=torch.float64, device=self.backends[0].device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.comm)
        return int(t.item())

    # ------------------------------------------------------------- vectors
    def dot(self, a: list, b: list) -> float:
        return self.allsum([float((x[: s.n_owned] * y[: s.n_owned]).sum()) for s, x, y in zip(self.subs, a, b)])

    def norm(self, a: list) -> float:
        return math.sqrt(self.dot(a, a))

    def like(self, a: list) -> list:
        import torch
        return [torch.zeros_like(x) for x in a]

    # ----------------------------------------------------------- operators
    def residual(self, U: list) -> tuple[list, int]:
        """R = residual(U) on every piece (owned rows exact); returns the
        unphysical count summed over all ranks."""
        self.exchange(U)
        R, bad = [], 0
        for be, u in zip(self.backends, U):
            r, b = be.residual(u)
            R.append(r)
            bad += b
        return R, self.allmax_int([bad])

    def rk2(self, U: list, cfl: float, nsteps: int) -> list:
        """Heun RK2 with local time steps: k1 = dt R(U), U0 = U - k1,
        k2 = dt R(U0), U <- U - (k1 + k2)/2 (ExplicitTsDesc.C:98-117)."""
        U = [u.clone() for u in U]
        for _ in range(nsteps):
            self.exchange(U)
            dts = [be.timestep(u, cfl) for be, u in zip(self.backends, U)]
            R1, _ = self.residual(U)
            k1 = [r * d[:, None] for r, d in zip(R1, dts)]
            U0 = [u - k for u, k in zip(U, k1)]
            R2, _ = self.residual(U0)
            for u, k, r, d in zip(U, k1, R2, dts):
                u -= 0.5 * (k + r * d[:, None])
        self.exchange(U)
        return U

    def matvec(self, p: list) -> list:
        self.exchange(p)
        return [be.matvec(x) for be, x in zip(self.backends, p)]

    def prec(self, x: list) -> list:
        return [be.prec_apply(v) for be, v in zip(self.backends, x)]

    def gmres(self, b: list, numVec: int = 30, maxits: int = 30, eps: float = 1e-2) -> tuple[list, int]:
        """Right-preconditioned GMRES(numVec) from x = 0 (KspSolver.C:351-492):
        MGS with global dot products, Givens rotations and back substitution
        on the host (KspSolver.C:917-982).  Returns (x, iterations)."""
        x = self.like(b)
        bnorm = self.norm(b)
        target = eps * bnorm
        it = 0
        while True:
            if it == 0:
                r = [v.clone() for v in b]
            else:
                Ax = self.matvec(x)
                r = [bv - av for bv, av in zip(b, Ax)]
            beta = self.norm(r)
            if beta == 0.0:
                return x, it
            V = [[v / beta for v in r]]
            H = np.zeros((numVec + 1, numVec))
            cs = np.zeros(2 * numVec)
            g = np.zeros(numVec + 1)
            g[0] = beta
            done = False
            j = 0
            for j in range(numVec):
                z = self.prec(V[j])
                w = self.matvec(z)
                for i in range(j + 1):
                    h = self.dot(w, V[i])
                    H[i, j] = h
                    w = [wv - h * vv for wv, vv in zip(w, V[i])]
                H[j + 1, j] = self.norm(w)
                breakdown = H[j + 1, j] == 0.0
                if not breakdown:
                    V.append([wv / H[j + 1, j] for wv in w])
                for i in range(j):
                    hj = cs[2 * i + 1] * H[i, j] + cs[2 * i] * H[i + 1, j]
                    hjp1 = -cs[2 * i] * H[i, j] + cs[2 * i + 1] * H[i + 1, j]
                    H[i, j], H[i + 1, j] = hj, hjp1
                if H[j, j] * H[j, j] == 0.0:
                    cs[2 * j + 1], cs[2 * j] = 0.0, 1.0
                else:
                    coef = 1.0 / math.sqrt(H[j, j] * H[j, j] + H[j + 1, j] * H[j + 1, j])
                    cs[2 * j + 1] = math.sqrt(H[j, j] * H[j, j]) * coef
                    cs[2 * j] = cs[2 * j + 1] * H[j + 1, j] / H[j, j]
                H[j, j] = cs[2 * j + 1] * H[j, j] + cs[2 * j] * H[j + 1, j]
                H[j + 1, j] = 0.0
                g[j + 1] = -cs[2 * j] * g[j]
                g[j] = cs[2 * j + 1] * g[j]
                it += 1
                if breakdown or abs(g[j + 1]) <= target or it >= maxits:
                    done = True
                    break
            y = np.zeros(j + 1)
            for i in range(j, -1, -1):
                y[i] = g[i]
                for k in range(j, i, -1):
                    y[i] -= H[i, k] * y[k]
                y[i] /= H[i, i]
            comb = [sum(float(y[m]) * V[m][q] for m in range(j + 1)) for q in range(len(b))]
            dx = self.prec(comb)
            x = [xv + d for xv, d in zip(x, dx)]
            if done:
                return x, it

    def newton(self, U: list, cfl0: float = 10.0, cfl_max: float = 1e4, ser: float = 0.7, tol: float = 1e-8,
               max_steps: int = 300, precision: int = 64, krylov: int = 30, maxits: int = 30,
               ksp_eps: float = 1e-2) -> tuple[list, dict]:
        """Pseudo-transient Newton (one Newton step per pseudo-time step)
        with the RESIDUAL CFL law, block-Jacobi GMRES, and the physical-
        solution check (redo at half the CFL number, TsParameters.C:187-195)."""
        U = [u.clone() for u in U]
        res0, rel, rel_prev, cfl = 0.0, 1.0, 1.0, cfl0
        k, lits, redos, redo = 0, 0, 0, False
        R = None
        while k <= max_steps:
            if not redo:
                R, _ = self.residual(U)
                res = self.norm(R)
                if not math.isfinite(res):
                    raise FloatingPointError(f"non-finite residual at Newton step {k}")
                if k == 0:
                    res0 = res
                rel = res / res0 if res0 > 0 else 0.0
                if rel <= tol or k == max_steps:
                    break
                if k > 0:
                    cfl = min(max(cfl * (rel_prev / rel) ** ser, 0.0), cfl_max)
                rel_prev = rel
            redo = False
            self.exchange(U)
            dts = [be.timestep(u, cfl) for be, u in zip(self.backends, U)]
            for be, u, d in zip(self.backends, U, dts):
                be.jacobian(u, d, precision)
                be.prec_setup()
            dQ, its = self.gmres([-r for r in R], krylov, maxits, ksp_eps)
            lits += its
            Unew = [u + d for u, d in zip(U, dQ)]
            bad = self.allmax_int([be.count_unphysical(u, s.n_owned) for be, u, s in
                                   zip(self.backends, Unew, self.subs)])
            if bad:
                redos += 1
                cfl *= 0.5
                if cfl < cfl0 / 1000.0:
                    raise FloatingPointError("Newton updates stayed non-physical down to CFL cfl0/1000")
                redo = True
                continue
            U = Unew
            k += 1
        self.exchange(U)
        return U, {"steps": k, "linear_its": lits, "rel_residual": rel, "redos": redos}


class GpuBackend:
    """The single-domain operators of one piece through the C ABI, on its
    own CUDA context (torch CUDA tensors in and out)."""

    def __init__(self, sub: Subdomain, Ub, device: int = 0, reconstruction: int = 2):
        import torch
        from . import Context, JacobiPrec, MatVecProdH1, SpaceOperator
        self.device = torch.device("cuda", device)
        self.ctx = Context.from_mesh(sub.mesh, Ub, reconstruction=reconstruction, device=device)
        self.ctx.set_owned_rows(sub.n_owned)
        self.sp = SpaceOperator(self.ctx)
        self._mv = None
        self._pc = JacobiPrec(self.ctx)
        self._MatVecProdH1 = MatVecProdH1
        self.gamma = 1.4

    def residual(self, U):
        return self.sp.computeResidual(U)

    def timestep(self, U, cfl):
        return self.sp.computeTimeStep(U, cfl)

    def jacobian(self, U, dt, precision=64):
        self._mv = self._MatVecProdH1(self.ctx, precision)
        self._mv.evaluate(U, dt)

    def prec_setup(self):
        self._pc.setup()

    def prec_apply(self, x):
        return self._pc.apply(x)

    def matvec(self, p):
        return self._mv.apply(p)

    def count_unphysical(self, U, n_owned: int) -> int:
        rho = U[:n_owned, 0]
        ke = 0.5 * (U[:n_owned, 1:4] ** 2).sum(1) / rho
        p = (self.gamma - 1.0) * (U[:n_owned, 4] - ke)
        return int((~(rho > 0)).sum().item() + (~(p > 0)).sum().item())

    def close(self):
        self.ctx.close()
