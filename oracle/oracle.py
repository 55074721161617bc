"""ctypes front end of the CPU oracle (oracle/aerof_oracle.cpp).

Test infrastructure only: imported by tests/, bench.py's CPU-baseline leg and
__graft_entry__.smoke(), never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "aerof_oracle.cpp")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_fp = C.POINTER(C.c_float)


def build(force: bool = False) -> str:
    """Compile the oracle (g++ -O3 -fopenmp -ffp-contract=off)."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        cmd = ["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-ffp-contract=off", "-std=c++17",
               "-shared", "-fPIC", SRC, "-o", LIB]
        subprocess.check_call(cmd)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _ip, _ip, _ip, C.c_double]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_num_edges.argtypes = [C.c_void_p]
        L.orc_get_edges.argtypes = [C.c_void_p, _ip]
        L.orc_get_geometry.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.orc_prim.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_gradients.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.orc_residual.argtypes = [C.c_void_p, _dp, _dp, C.c_int, C.c_double, C.c_int, _dp]
        L.orc_baseline_create.restype = C.c_void_p
        L.orc_baseline_destroy.argtypes = [C.c_void_p]
        L.orc_residual_threaded.argtypes = [C.c_void_p, C.c_void_p, _dp, _dp, C.c_int, C.c_int, _dp]
        L.orc_timestep.argtypes = [C.c_void_p, _dp, C.c_double, _dp]
        L.orc_rk2.argtypes = [C.c_void_p, _dp, _dp, C.c_int, C.c_double, C.c_int]
        L.orc_roeflux7.argtypes = [C.c_double, _dp, C.c_double, _dp, _dp, _dp]
        L.orc_boundflux5.argtypes = [C.c_double, _dp, C.c_double, _dp, _dp, _dp]
        L.orc_roejac6.argtypes = [C.c_double, _dp, _dp, _dp, _dp, _dp]
        L.orc_vanalbada.argtypes = [C.c_double, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_linear_rec.argtypes = [C.c_double, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_cons2prim.argtypes = [C.c_double, _dp, _dp]
        L.orc_post_dVdU.argtypes = [C.c_double, _dp, _dp, _dp]
        L.orc_invert5.argtypes = [_dp]
        L.orc_invert5f.argtypes = [_fp]
        L.orc_jacobian.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.orc_matvec.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int]
        L.orc_bj_invert.argtypes = [C.c_void_p, _dp, _dp, C.c_int]
        L.orc_gmres.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_int, _dp]
        L.orc_ilu0.restype = C.c_int
        L.orc_ilu0.argtypes = [C.c_void_p, _dp, C.c_int, C.c_int, _dp, _dp, C.POINTER(C.c_int), _ip]
        L.orc_ilu_factor.restype = C.c_void_p
        L.orc_ilu_factor.argtypes = [C.c_void_p, _dp, C.c_int, C.c_int, _ip, C.POINTER(C.c_int)]
        L.orc_ilu_apply.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_ilu_free.argtypes = [C.c_void_p]
        L.orc_rcm_order.argtypes = [C.c_void_p, _ip]
        L.orc_gmres_ilu.restype = C.c_int
        L.orc_gmres_ilu.argtypes = [C.c_void_p, _dp, C.c_void_p, _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_int,
                                    _dp]
        L.orc_newton.argtypes = [C.c_void_p, _dp, _dp, C.c_int, C.c_double, C.c_double, C.c_double,
                                 C.c_double, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                 _dp, _ip, _ip]
        L.orc_jvp.argtypes = [C.c_void_p, _dp, _dp, C.c_int, _dp, _dp]
        L.orc_residual_sa.restype = C.c_int
        L.orc_residual_sa.argtypes = [C.c_void_p, _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_double, _dp, C.c_int, _dp, _dp]
        L.orc_roeflux7_sa.argtypes = [C.c_double, _dp, _dp, _dp, _dp]
        L.orc_face_flux_sa.argtypes = [C.c_double, C.c_int, _dp, _dp, _dp, _dp]
        L.orc_residual_visc.restype = C.c_int
        L.orc_residual_visc.argtypes = [C.c_void_p, _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double,
                                        C.c_double, C.c_double, C.c_double, _dp]
        L.orc_matvec_fd.restype = C.c_double
        L.orc_matvec_fd.argtypes = [C.c_void_p, _dp, _dp, C.c_int, _dp, _dp, _dp, C.c_int, _dp]
        L.orc_dRdX.argtypes = [C.c_void_p, _dp, _dp, C.c_int, _dp, _dp, _dp]
        L.orc_residual_at.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int, _dp]
        L.orc_zforce.restype = C.c_double
        L.orc_zforce.argtypes = [C.c_void_p, _dp, _dp, _ip, C.c_int]
        L.orc_zforce_dU.argtypes = [C.c_void_p, _dp, _ip, C.c_int, _dp]
        L.orc_zforce_dX.restype = C.c_double
        L.orc_zforce_dX.argtypes = [C.c_void_p, _dp, _ip, C.c_int, _dp]
        _lib = L
    return _lib


# Spalart-Allmaras constants (cb1, cb2, cw2, cw3, cv1, cv2, sigma, vkcst,
# prandtl_turbulent): SAModelData's and TurbulenceClosureData's defaults
# (IoDataCore.C:1411-1418, 1839)
SA_DEFAULTS = (0.1355, 0.622, 0.3, 2.0, 7.1, 5.0, 2.0 / 3.0, 0.41, 0.9)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Oracle:
    """CPU restatement of the reference path on one mesh."""

    def __init__(self, mesh: dict, gamma: float = 1.4):
        self.L = lib()
        self.X = f64(mesh["X"])
        self.tets = i32(mesh["tets"])
        self.faces = i32(mesh["faces"])
        self.codes = i32(mesh["codes"])
        self.N, self.T, self.F = self.X.shape[0], self.tets.shape[0], self.faces.shape[0]
        self.gamma = gamma
        self.h = self.L.orc_create(self.N, self.T, self.F, _d(self.X), _i(self.tets), _i(self.faces),
                                   _i(self.codes), gamma)
        self.E = self.L.orc_num_edges(self.h)
        self._bl = None

    def __del__(self):
        try:
            if self._bl:
                self.L.orc_baseline_destroy(self._bl)
            self.L.orc_destroy(self.h)
        except Exception:
            pass

    def edges(self):
        e = np.empty((self.E, 2), dtype=np.int32)
        self.L.orc_get_edges(self.h, _i(e))
        return e

    def geometry(self):
        en = np.empty((self.E, 3)); fn = np.empty((self.F, 3)); cv = np.empty(self.N); R = np.empty((self.N, 6))
        self.L.orc_get_geometry(self.h, _d(en), _d(fn), _d(cv), _d(R))
        return {"edge_normal": en, "face_normal": fn, "ctrl_vol": cv, "lsq_R": R}

    def prim(self, U):
        U = f64(U); V = np.empty_like(U)
        self.L.orc_prim(self.h, _d(U), _d(V))
        return V

    def gradients(self, V):
        V = f64(V)
        gx = np.empty_like(V); gy = np.empty_like(V); gz = np.empty_like(V)
        self.L.orc_gradients(self.h, _d(V), _d(gx), _d(gy), _d(gz))
        return gx, gy, gz

    def residual(self, U, Ub, order=2, beta=1.0 / 3.0, failsafe=0):
        U = f64(U); Ub = f64(Ub); R = np.empty_like(U)
        ierr = self.L.orc_residual(self.h, _d(U), _d(Ub), order, beta, failsafe, _d(R))
        return R, ierr

    def residual_sa(self, U, Ub, d2wall, order=2, model=1, reynolds=100.0, prandtl=0.72, bulk=0.0, alpha=1.0,
                    Ts=0.0, sa=None, fv3=False):
        """Spalart-Allmaras residual of U [N][6] (rho nu~ last) with the
        viscous Galerkin term; sa = (cb1, cb2, cw2, cw3, cv1, cv2, sigma,
        vkcst, prandtl_turbulent), the reference's defaults when None."""
        U = f64(U); R = np.empty_like(U)
        sa = f64(SA_DEFAULTS if sa is None else sa)
        ierr = self.L.orc_residual_sa(self.h, _d(U), _d(f64(Ub)), order, model, 1.0 / reynolds, 1.0 / prandtl,
                                      bulk, alpha, Ts, _d(sa), int(fv3), _d(f64(d2wall)), _d(R))
        return R, ierr

    def residual_visc(self, U, Ub, order=2, model=1, reynolds=100.0, prandtl=0.72, bulk=0.0, alpha=1.0,
                      Ts=0.0):
        """Residual plus the laminar viscous Galerkin term (model 1:
        constant viscosity, 2: Sutherland)."""
        U = f64(U); R = np.empty_like(U)
        ierr = self.L.orc_residual_visc(self.h, _d(U), _d(f64(Ub)), order, model, 1.0 / reynolds, 1.0 / prandtl,
                                        bulk, alpha, Ts, _d(R))
        return R, ierr

    def residual_threaded(self, U, Ub, order=2, nthreads=None, out=None):
        if self._bl is None:
            self._bl = self.L.orc_baseline_create()
        nthreads = nthreads or os.cpu_count()
        U = f64(U); Ub = f64(Ub)
        R = out if out is not None else np.empty_like(U)
        self.L.orc_residual_threaded(self.h, self._bl, _d(U), _d(Ub), order, nthreads, _d(R))
        return R

    def timestep(self, U, cfl):
        U = f64(U); dt = np.empty(self.N)
        self.L.orc_timestep(self.h, _d(U), cfl, _d(dt))
        return dt

    def rk2(self, U, Ub, order, cfl, nsteps):
        U = f64(U).copy()
        self.L.orc_rk2(self.h, _d(U), _d(f64(Ub)), order, cfl, nsteps)
        return U

    def jacobian(self, U, Ub, dt=None):
        U = f64(U)
        A = np.empty((self.N + 2 * self.E, 5, 5))
        dtp = _d(f64(dt)) if dt is not None else None
        self.L.orc_jacobian(self.h, _d(U), _d(f64(Ub)), dtp, _d(A))
        return A

    def matvec(self, A, p, transpose=False):
        p = f64(p); y = np.empty_like(p)
        self.L.orc_matvec(self.h, _d(f64(A)), _d(p), _d(y), int(transpose))
        return y

    def bj_invert(self, A, fp32=True):
        D = np.empty((self.N, 5, 5))
        bad = self.L.orc_bj_invert(self.h, _d(f64(A)), _d(D), int(fp32))
        return D, bad

    def ilu0(self, A, x, fp32=True, transpose=False):
        """(LU)^-1 x with the block ILU(0) of A (or A^T) in the multicolour
        ordering; also returns the colour of every node."""
        x = f64(x); y = np.empty_like(x)
        nc = C.c_int(0); colour = np.empty(self.N, dtype=np.int32)
        bad = self.L.orc_ilu0(self.h, _d(f64(A)), int(fp32), int(transpose), _d(x), _d(y), C.byref(nc),
                              _i(colour))
        return y, bad, nc.value, colour

    def rcm_order(self):
        """Reverse Cuthill-McKee order of the ILU rows (order[r] = node of
        row r), the reference's default ILU renumbering."""
        order = np.empty(self.N, dtype=np.int32)
        self.L.orc_rcm_order(self.h, _i(order))
        return order

    def gmres_ilu(self, A, b, order=None, fp32=True, numVec=30, maxits=30, eps=1e-2, transpose=False):
        """GMRES right-preconditioned by the block ILU(0) of A factored on
        the multicolour order (order None) or on the given node order."""
        b = f64(b); x = np.empty_like(b); res = C.c_double(0); bad = C.c_int(0)
        o = None if order is None else np.ascontiguousarray(order, dtype=np.int32)
        f = self.L.orc_ilu_factor(self.h, _d(f64(A)), int(fp32), int(transpose),
                                  _i(o) if o is not None else None, C.byref(bad))
        try:
            its = self.L.orc_gmres_ilu(self.h, _d(f64(A)), f, _d(b), _d(x), numVec, maxits, eps, int(transpose),
                                       C.byref(res))
        finally:
            self.L.orc_ilu_free(f)
        return x, its, res.value

    def gmres(self, A, Dinv, b, numVec=30, maxits=30, eps=1e-2, transpose=False):
        b = f64(b); x = np.empty_like(b); res = C.c_double(0)
        its = self.L.orc_gmres(self.h, _d(f64(A)), _d(f64(Dinv)), _d(b), _d(x), numVec, maxits, eps,
                               int(transpose), C.byref(res))
        return x, its, res.value

    def newton(self, U, Ub, order=2, cfl0=10.0, cfl_min=0.0, cfl_max=1e4, ser=0.7, numVec=30,
               maxits=30, eps=1e-2, tol=1e-8, max_steps=200, fp32_prec=True):
        """Pseudo-transient Newton; returns (U, history, GMRES its per step).
        self.last_redos holds the steps redone at half the CFL number after a
        non-physical update; a CFL number driven below cfl0/1000 raises."""
        U = f64(U).copy()
        hist = np.zeros(max_steps + 1); lits = np.zeros(max_steps + 1, dtype=np.int32)
        redos = np.zeros(1, dtype=np.int32)
        k = self.L.orc_newton(self.h, _d(U), _d(f64(Ub)), order, cfl0, cfl_min, cfl_max, ser, numVec,
                              maxits, eps, tol, max_steps, int(fp32_prec), _d(hist), _i(lits), _i(redos))
        self.last_redos = int(redos[0])
        if k < 0:
            raise RuntimeError(f"oracle Newton diverged (code {k}) after {self.last_redos} redone steps")
        return U, hist[:k + 1], lits[:k]

    def matvec_fd(self, U, Ub, p, order=2, dt=None, fd_order=1, F=None):
        """MatVecProdFD::apply: finite-difference Jacobian product; returns
        (prod, eps)."""
        U = f64(U); p = f64(p); prod = np.empty_like(U)
        eps = self.L.orc_matvec_fd(self.h, _d(U), _d(f64(Ub)), order, _d(f64(F)) if F is not None else None,
                                   _d(p), _d(f64(dt)) if dt is not None else None, int(fd_order), _d(prod))
        return prod, eps

    def jvp(self, U, Ub, v, order=2):
        U = f64(U); v = f64(v); Jv = np.empty_like(U)
        self.L.orc_jvp(self.h, _d(U), _d(f64(Ub)), order, _d(v), _d(Jv))
        return Jv

    def dRdX(self, U, Ub, Xdot, order=2):
        U = f64(U); dR = np.empty_like(U); R = np.empty_like(U)
        self.L.orc_dRdX(self.h, _d(U), _d(f64(Ub)), order, _d(f64(Xdot)), _d(dR), _d(R))
        return dR, R

    def residual_at(self, X, U, Ub, order=2):
        U = f64(U); R = np.empty_like(U)
        self.L.orc_residual_at(self.h, _d(f64(X)), _d(U), _d(f64(Ub)), order, _d(R))
        return R

    def zforce(self, U, zfaces, X=None):
        zf = i32(zfaces)
        Xp = _d(f64(X)) if X is not None else None
        return self.L.orc_zforce(self.h, Xp, _d(f64(U)), _i(zf), zf.size)

    def zforce_dU(self, U, zfaces):
        zf = i32(zfaces); g = np.empty((self.N, 5))
        self.L.orc_zforce_dU(self.h, _d(f64(U)), _i(zf), zf.size, _d(g))
        return g

    def zforce_dX(self, U, zfaces, Xdot):
        zf = i32(zfaces)
        return self.L.orc_zforce_dX(self.h, _d(f64(U)), _i(zf), zf.size, _d(f64(Xdot)))


# pointwise kernels ---------------------------------------------------------

def roeflux7(gam, n, Vi, Vj, ndot=0.0):
    out = np.empty(5)
    lib().orc_roeflux7(gam, _d(f64(n)), ndot, _d(f64(Vi)), _d(f64(Vj)), _d(out))
    return out


def roeflux7_sa(gam, n, Vi, Vj):
    out = np.empty(6)
    lib().orc_roeflux7_sa(gam, _d(f64(n)), _d(f64(Vi)), _d(f64(Vj)), _d(out))
    return out


def face_flux_sa(gam, code, n3, V, Ub):
    out = np.empty(6)
    lib().orc_face_flux_sa(gam, int(code), _d(f64(n3)), _d(f64(V)), _d(f64(Ub)), _d(out))
    return out


def boundflux5(gam, n, V, Ub, sig=0.0):
    out = np.empty(5)
    lib().orc_boundflux5(gam, _d(f64(n)), sig, _d(f64(V)), _d(f64(Ub)), _d(out))
    return out


def roejac6(gam, n, Vi, Vj):
    jl = np.empty(25); jr = np.empty(25)
    lib().orc_roejac6(gam, _d(f64(n)), _d(f64(Vi)), _d(f64(Vj)), _d(jl), _d(jr))
    return jl.reshape(5, 5), jr.reshape(5, 5)


def vanalbada(beta, Vi, ddVij, Vj, ddVji):
    a = np.empty(5); b = np.empty(5)
    lib().orc_vanalbada(beta, _d(f64(Vi)), _d(f64(ddVij)), _d(f64(Vj)), _d(f64(ddVji)), _d(a), _d(b))
    return a, b


def linear_rec(beta, Vi, ddVij, Vj, ddVji):
    a = np.empty(5); b = np.empty(5)
    lib().orc_linear_rec(beta, _d(f64(Vi)), _d(f64(ddVij)), _d(f64(Vj)), _d(f64(ddVji)), _d(a), _d(b))
    return a, b


def cons2prim(gam, U):
    V = np.empty(5)
    lib().orc_cons2prim(gam, _d(f64(U)), _d(V))
    return V


def post_dVdU(gam, V, mat):
    out = np.empty(25)
    lib().orc_post_dVdU(gam, _d(f64(V)), _d(f64(mat).reshape(-1)), _d(out))
    return out.reshape(5, 5)


def invert5(a, fp32=False):
    if fp32:
        b = np.ascontiguousarray(a, dtype=np.float32).copy()
        info = lib().orc_invert5f(b.ctypes.data_as(_fp))
    else:
        b = f64(a).copy()
        info = lib().orc_invert5(_d(b))
    return b, info


def zfaces_of(mesh: dict) -> np.ndarray:
    """Indices of the boundary faces on z=0 (side 4 of the lattice mesh)."""
    return np.nonzero(mesh["sides"] == 4)[0].astype(np.int32)
