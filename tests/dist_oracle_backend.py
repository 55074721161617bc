"""Test infrastructure: the single-domain operators of one subdomain piece
evaluated by the CPU oracle (torch CPU tensors in and out), so that the
decomposed solvers of aerof_dev_b200.distributed can run on gloo ranks
without a GPU and be compared with the single-domain oracle."""
import numpy as np
import torch


class OracleBackend:
    def __init__(self, oracle_mod, sub, Ub, order=2):
        self.o = oracle_mod.Oracle(sub.mesh)
        self.Ub = np.asarray(Ub, dtype=np.float64)
        self.order = order
        self.n_owned = sub.n_owned
        self.device = torch.device("cpu")
        self.A = None
        self.D = None

    def residual(self, U):
        R, bad = self.o.residual(U.numpy(), self.Ub, self.order)
        return torch.from_numpy(R), bad

    def timestep(self, U, cfl):
        return torch.from_numpy(self.o.timestep(U.numpy(), cfl))

    def jacobian(self, U, dt, precision=64):
        self.A = self.o.jacobian(U.numpy(), self.Ub, dt.numpy())

    def prec_setup(self):
        D, _ = self.o.bj_invert(self.A, fp32=False)
        D[self.n_owned:] = np.eye(5)          # ghost rows: identity
        self.D = D

    def prec_apply(self, x):
        return torch.from_numpy(np.einsum("nij,nj->ni", self.D, x.numpy()))

    def matvec(self, p):
        return torch.from_numpy(self.o.matvec(self.A, p.numpy()))

    def count_unphysical(self, U, n_owned):
        u = U[:n_owned].numpy()
        rho = u[:, 0]
        p = 0.4 * (u[:, 4] - 0.5 * (u[:, 1:4] ** 2).sum(1) / rho)
        return int((~(rho > 0)).sum() + (~(p > 0)).sum())
