"""Golden vectors of the reference's Fortran flux kernels.

AERO-F's Roe flux (f77src/roeflux7.f), Steger-Warming boundary flux
(f77src/boundflux5.f) and approximate Roe Jacobian (f77src/roejac6.f) are
Fortran 77; no Fortran compiler is available, so ``make -C oracle ref
REF=<aerof tree>`` translates those three files mechanically to C
(oracle/f77_to_c.py) into oracle/_ref/libref_f77.so.  This script runs that
library on seeded inputs that cover both upwind branches, moving-mesh terms,
subsonic and supersonic boundary states, and stores inputs and outputs in
tests/golden/reference_fortran.npz; the tests read the committed .npz.

    python tests/golden/make_golden_f77.py --ref /path/to/aerof
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_f77.so")
SEED = 20261203
GAM = 1.4

dp = C.POINTER(C.c_double)


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(dp)


def _d(x):
    return C.byref(C.c_double(x))


def _i(x):
    return C.byref(C.c_int(x))


def states(rng, n, mach_spread=1.0):
    """Primitive states (rho, u, v, w, p) around a Mach 0.8 free stream
    (rho = 1, |u| = 1, p = 1/(gamma M^2)), with some supersonic ones."""
    V = np.empty((n, 5))
    V[:, 0] = 0.5 + rng.random(n)
    V[:, 1:4] = mach_spread * rng.standard_normal((n, 3))
    V[:, 1] += 1.0
    V[:, 4] = (1.0 / (GAM * 0.64)) * (0.3 + 1.4 * rng.random(n))
    return V


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("AEROF_REFERENCE_TREE"),
                    help="AERO-F source tree (or set AEROF_REFERENCE_TREE)")
    a = ap.parse_args()
    if not a.ref:
        ap.error("name the AERO-F source tree with --ref or AEROF_REFERENCE_TREE")
    subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={a.ref}"])
    L = C.CDLL(LIB)
    rng = np.random.Generator(np.random.PCG64(SEED))
    out = {}

    # roeflux7(type, gam, pstiff, enormal, evitno, Ug, Ud, phi)
    n = 600
    Vi = states(rng, n)
    Vj = Vi * (1 + 0.1 * rng.standard_normal((n, 5)))
    Vj[:, 0] = np.abs(Vj[:, 0]) + 0.05
    Vj[:, 4] = np.abs(Vj[:, 4]) + 0.05
    Vj[: n // 4, 1:4] = -Vj[: n // 4, 1:4]                       # both upwind sides
    nrm = rng.standard_normal((n, 3)) * 10.0 ** rng.uniform(-4, 0, (n, 1))
    ndot = np.where(rng.random(n) < 0.25, 0.3 * rng.standard_normal(n), 0.0)
    phi = np.empty((n, 5))
    for k in range(n):
        o = np.zeros(7)
        L.roeflux7_f77_(_i(0), _d(GAM), _d(0.0), _p(nrm[k]), _d(ndot[k]), _p(Vi[k]), _p(Vj[k]),
                        o.ctypes.data_as(dp))
        phi[k] = o[:5]
    out["roe_in"] = np.column_stack([nrm, ndot, Vi, Vj])
    out["roe_out"] = phi

    # boundflux5(type, gam, normal, sig, ua (primitive), ub (conservative), flux)
    n = 600
    V = states(rng, n, mach_spread=1.5)                           # sub- and supersonic
    Vb = states(rng, n)
    Ub = np.column_stack([Vb[:, 0], Vb[:, 0:1] * Vb[:, 1:4],
                          Vb[:, 4] / (GAM - 1) + 0.5 * Vb[:, 0] * (Vb[:, 1:4] ** 2).sum(1)])
    nrm = rng.standard_normal((n, 3)) * 10.0 ** rng.uniform(-4, 0, (n, 1))
    sig = np.where(rng.random(n) < 0.25, 0.2 * rng.standard_normal(n), 0.0)
    fl = np.empty((n, 5))
    for k in range(n):
        o = np.zeros(7)
        L.boundflux5_f77_(_i(0), _d(GAM), _p(nrm[k]), _d(sig[k]), _p(V[k]), _p(Ub[k]), o.ctypes.data_as(dp))
        fl[k] = o[:5]
    out["bf_in"] = np.column_stack([nrm, sig, V, Ub])
    out["bf_out"] = fl

    # roejac6(type, gamma, gam, pstiff, enormal, evitno, Ug, Ud, jac, sw, mach, k1,
    #         cmach, shockreducer, irey, length, prec): the Roe dissipation
    # coefficient gamma = 1, no low-Mach preconditioning, as computeJacobians
    # calls it for the first endpoint (sw = 1) and the second (sw = 2, states
    # swapped)
    n = 250
    Vi = states(rng, n)
    Vj = Vi * (1 + 0.1 * rng.standard_normal((n, 5)))
    Vj[:, 0] = np.abs(Vj[:, 0]) + 0.05
    Vj[:, 4] = np.abs(Vj[:, 4]) + 0.05
    nrm = rng.standard_normal((n, 3)) * 10.0 ** rng.uniform(-4, 0, (n, 1))
    jac = np.empty((n, 50))
    for k in range(n):
        for sw, (a_, b_) in ((1, (Vi[k], Vj[k])), (2, (Vj[k], Vi[k]))):
            o = np.zeros(25)
            L.roejac6_f77_(_i(0), _d(1.0), _d(GAM), _d(0.0), _p(nrm[k]), _d(0.0), _p(a_), _p(b_),
                           o.ctypes.data_as(dp), _i(sw), _d(0.0), _d(0.0), _d(0.0), _d(0.0), _d(0.0), _d(1.0),
                           _i(0))
            jac[k, 25 * (sw - 1): 25 * sw] = o
    out["jac_in"] = np.column_stack([nrm, Vi, Vj])
    out["jac_out"] = jac

    # the Spalart-Allmaras variants (type 1: a sixth, advected component,
    # nu~ primitive, rho nu~ in the conservative boundary state), both
    # upwind directions of the mass flux
    n = 300
    Vi = np.column_stack([states(rng, n), 1e-3 * (0.5 + rng.random(n))])
    Vj = np.column_stack([Vi[:, :5] * (1 + 0.1 * rng.standard_normal((n, 5))), 1e-3 * (0.5 + rng.random(n))])
    Vj[:, 0] = np.abs(Vj[:, 0]) + 0.05
    Vj[:, 4] = np.abs(Vj[:, 4]) + 0.05
    Vj[: n // 3, 1:4] = -Vj[: n // 3, 1:4]
    nrm = rng.standard_normal((n, 3)) * 10.0 ** rng.uniform(-4, 0, (n, 1))
    phi = np.empty((n, 6))
    for k in range(n):
        o = np.zeros(7)
        L.roeflux7_f77_(_i(1), _d(GAM), _d(0.0), _p(nrm[k]), _d(0.0), _p(Vi[k]), _p(Vj[k]), o.ctypes.data_as(dp))
        phi[k] = o[:6]
    out["roe_sa_in"] = np.column_stack([nrm, Vi, Vj])
    out["roe_sa_out"] = phi
    n = 300
    V = np.column_stack([states(rng, n, mach_spread=1.5), 1e-3 * (0.5 + rng.random(n))])
    Vb = states(rng, n)
    Ub = np.column_stack([Vb[:, 0], Vb[:, 0:1] * Vb[:, 1:4],
                          Vb[:, 4] / (GAM - 1) + 0.5 * Vb[:, 0] * (Vb[:, 1:4] ** 2).sum(1),
                          Vb[:, 0] * 1e-3 * (0.5 + rng.random(n))])
    nrm = rng.standard_normal((n, 3)) * 10.0 ** rng.uniform(-4, 0, (n, 1))
    fl = np.empty((n, 6))
    for k in range(n):
        o = np.zeros(7)
        L.boundflux5_f77_(_i(1), _d(GAM), _p(nrm[k]), _d(0.0), _p(V[k]), _p(Ub[k]), o.ctypes.data_as(dp))
        fl[k] = o[:6]
    out["bf_sa_in"] = np.column_stack([nrm, V, Ub])
    out["bf_sa_out"] = fl

    dst = os.path.join(HERE, "reference_fortran.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    sys.exit(main())
