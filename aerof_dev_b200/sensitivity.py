"""Shape sensitivities of a boundary-force functional (AERO-F's sensitivity
analysis path, FluidShapeOptimizationHandler.C).

The flow sensitivities come from the GPU (exact J v, J^T w, dR/dX . Xdot,
(dR/dX)^T lambda and the linearised GMRES solves of the C ABI); the
functional and its partial derivatives live on a few thousand boundary
faces and are evaluated here on the host.

Functional: the pressure force along +z on a set of boundary faces,
J(U, X) = sum_f p_f * (-n_z(f)), p_f the mean of the face's three node
pressures, n_f = 0.5 (x2 - x0) ^ (x1 - x0) the outward area normal
(cf. PostOperator::computeForceAndMoment, PostOperator.C:379-).

Adjoint method (fso_on_AdjointSensitivityMesh, :2209-2357):
    (dR/dU)^T lambda = (dJ/dU)^T ;  dJ/dX_total = dJ/dX - (dR/dX)^T lambda
    dJ/ds_k = dJ/dX_total . Xdot_k
Direct method (fso_on_sensitivityMesh, :2362-2433):
    (dR/dU) x_k = -(dR/dX) Xdot_k ;  dJ/ds_k = dJ/dX . Xdot_k + dJ/dU . x_k
"""
from __future__ import annotations

import numpy as np


def _face_normals(X, faces):
    x0, x1, x2 = X[faces[:, 0]], X[faces[:, 1]], X[faces[:, 2]]
    return 0.5 * np.cross(x2 - x0, x1 - x0)


def pressure(U, gamma=1.4):
    return (gamma - 1.0) * (U[:, 4] - 0.5 * np.sum(U[:, 1:4] ** 2, axis=1) / U[:, 0])


class ZForce:
    """J = sum over the given faces of mean nodal pressure times (-n_z)."""

    def __init__(self, faces: np.ndarray, zfaces: np.ndarray, gamma: float = 1.4):
        self.f = np.ascontiguousarray(faces[zfaces], dtype=np.int64)
        self.gamma = gamma

    def value(self, U, X):
        n = _face_normals(X, self.f)
        p = pressure(U, self.gamma)
        pf = (p[self.f[:, 0]] + p[self.f[:, 1]] + p[self.f[:, 2]]) / 3.0
        return float(np.sum(pf * (-n[:, 2])))

    def dU(self, U, X):
        """dJ/dU as [N][5]."""
        g = np.zeros_like(U)
        n = _face_normals(X, self.f)
        w = -n[:, 2] / 3.0
        gm1 = self.gamma - 1.0
        u = U[:, 1:4] / U[:, 0:1]
        dp = np.empty_like(U)
        dp[:, 0] = gm1 * 0.5 * np.sum(u * u, axis=1)
        dp[:, 1:4] = -gm1 * u
        dp[:, 4] = gm1
        for l in range(3):
            np.add.at(g, self.f[:, l], w[:, None] * dp[self.f[:, l]])
        return g

    def dX(self, U, X):
        """dJ/dX as [N][3] (through the face normals)."""
        p = pressure(U, self.gamma)
        pf = (p[self.f[:, 0]] + p[self.f[:, 1]] + p[self.f[:, 2]]) / 3.0
        x0, x1, x2 = X[self.f[:, 0]], X[self.f[:, 1]], X[self.f[:, 2]]
        a, b = x2 - x0, x1 - x0
        # n_z = 0.5 (a_x b_y - a_y b_x)
        ga = np.zeros_like(a); gb = np.zeros_like(b)
        c = -0.5 * pf
        ga[:, 0] = c * b[:, 1]; ga[:, 1] = -c * b[:, 0]
        gb[:, 1] = c * a[:, 0]; gb[:, 0] = -c * a[:, 1]
        g = np.zeros_like(X)
        np.add.at(g, self.f[:, 2], ga)
        np.add.at(g, self.f[:, 1], gb)
        np.add.at(g, self.f[:, 0], -ga - gb)
        return g


def _norm(x) -> float:
    if type(x).__module__.startswith("torch"):
        return float(x.norm().item())
    return float(np.linalg.norm(x))


def _host(x):
    if type(x).__module__.startswith("torch"):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def converge(ctx, U, precision=32, tol=1e-10, max_steps=2000, exact_steps=3, krylov=30, inner_its=20):
    """Steady solve: pseudo-transient Newton (H1 operator) to ``tol``, then a
    few exact Newton steps with the matrix-free exact Jacobian (flexible
    GMRES preconditioned by inner_its mixed-precision H1 iterations)."""
    import aerof_dev_b200 as A
    sol = A.ImplicitSteadySolver(ctx, precision=precision, tol=tol, max_steps=max_steps)
    U, info = sol.solve(U)
    sp = A.SpaceOperator(ctx)
    S = A.Sensitivity(ctx)
    hist = [_norm(sp.computeResidual(U)[0])]
    for _ in range(exact_steps):
        R, _ = sp.computeResidual(U)
        dU, its, res = S.solve(U, -R, transpose=False, krylov=krylov, maxits=600, eps=1e-8, inner_its=inner_its)
        U = U + dU
        hist.append(_norm(sp.computeResidual(U)[0]))
    info["exact_newton_residuals"] = hist
    return U, info


def adjoint_gradient(ctx, U, X, functional: ZForce, modes, eps=1e-10, krylov=30, maxits=2000, inner_its=20,
                     stored_operator=False):
    """dJ/ds_k for every mode by the adjoint method.  stored_operator: the
    adjoint solve applies the stored exact linearisation (evaluated once)
    instead of re-evaluating it per product.  The info dict also holds the
    adjoint state lambda ([N][5], host)."""
    import aerof_dev_b200 as A
    S = A.Sensitivity(ctx)
    U = _host(U)
    gU = functional.dU(U, X)
    S.set_exact_operator(stored_operator)
    try:
        lam, its, res = S.solve(U, gU, transpose=True, krylov=krylov, maxits=maxits, eps=eps, inner_its=inner_its)
    finally:
        S.set_exact_operator(False)
        if stored_operator:
            S.h2_release()
    gX = functional.dX(U, X) - S.dRdX_T(U, lam)
    return np.einsum("kni,ni->k", modes, gX), {"adjoint_its": its, "adjoint_res": res, "lambda": _host(lam)}


def direct_gradient(ctx, U, X, functional: ZForce, modes, eps=1e-10, krylov=30, maxits=2000, inner_its=20):
    """dJ/ds_k for every mode by the direct method (one solve per mode)."""
    import aerof_dev_b200 as A
    S = A.Sensitivity(ctx)
    U = _host(U)
    gU = functional.dU(U, X)
    gX = functional.dX(U, X)
    out, its_all = [], []
    for Xd in modes:
        rhs = -S.dRdX(U, Xd)
        x, its, res = S.solve(U, rhs, transpose=False, krylov=krylov, maxits=maxits, eps=eps, inner_its=inner_its)
        out.append(float(np.sum(gX * Xd) + np.sum(gU * x)))
        its_all.append(its)
    return np.array(out), {"direct_its": its_all}


def direct_gradient_batch(ctx, U, X, functional: ZForce, modes, eps=1e-10, krylov=30, maxits=2000, inner_its=20):
    """dJ/ds_k for every mode by the direct method, all right-hand sides in
    one batched solve (the exact linearisation stored once)."""
    import aerof_dev_b200 as A
    S = A.Sensitivity(ctx)
    U = _host(U)
    gU = functional.dU(U, X)
    gX = functional.dX(U, X)
    rhs = np.stack([-S.dRdX(U, Xd) for Xd in modes])
    x, its, res = S.solve_batch(U, rhs, transpose=False, krylov=krylov, maxits=maxits, eps=eps,
                                inner_its=inner_its)
    S.h2_release()
    out = np.einsum("kni,ni->k", modes, gX) + np.einsum("kni,ni->k", x, gU)
    return out, {"direct_its": its.tolist(), "direct_res": res.tolist()}


def fd_gradient(ctx, U, X, functional: ZForce, modes, h=1e-6, **conv):
    """Central finite differences with the flow re-converged at X +- h Xdot.

    h may be a pair (h1, h2 = h1/2): Richardson extrapolation
    (4 D(h2) - D(h1)) / 3 of the two central differences, O(h^4)."""
    def central(Xd, step):
        vals = []
        for sgn in (1.0, -1.0):
            Xp = X + sgn * step * Xd
            ctx.update_coordinates(Xp)
            Up, _ = converge(ctx, U, **conv)
            vals.append(functional.value(_host(Up), Xp))
        return (vals[0] - vals[1]) / (2 * step)

    out = []
    for Xd in modes:
        if isinstance(h, (tuple, list)):
            d1, d2 = central(Xd, h[0]), central(Xd, h[1])
            ratio = (h[0] / h[1]) ** 2
            out.append((ratio * d2 - d1) / (ratio - 1.0))
        else:
            out.append(central(Xd, h))
    ctx.update_coordinates(X)
    return np.array(out)


def sensoutput_lines(J: float, grads) -> str:
    """The reference's sensitivity report lines (sa.sensoutput,
    FluidShapeOptimizationHandler.C:2553-2573): 'Fz= ...' and 'dFz/ds= ...'."""
    lines = [f"Fz= {J:.16e}"]
    for k, g in enumerate(grads):
        lines.append(f"dFz/ds{k}= {g:.16e}")
    return "\n".join(lines) + "\n"
