"""B200 (sm_100a) implementation of AERO-F's implicit edge-based FV hot path.

The compute lives in ``libaerof_gpu.so`` (hand-written CUDA behind the C ABI
of ``include/aerof_gpu.h``).  This module is the Python host side of that
ABI and mirrors the reference's C++ call surface for the path:

* :class:`SpaceOperator`  -- ``SpaceOperator<5>::computeResidual``,
  ``DistTimeState::computeTimeStep``, ``DistNodalGrad::compute``
* :class:`MatVecProdH1`   -- ``MatVecProdH1<5,MatScalar,5>::evaluate/apply/applyTranspose``
* :class:`JacobiPrec`     -- ``JacobiPrec<PrecScalar,5>::setup/apply/applyT``
* :class:`GmresSolver`    -- ``GmresSolver<...>::solve/solveT``
* :class:`ImplicitSteadySolver` -- the pseudo-transient Newton loop
* :class:`ExplicitRK2`    -- ``ExplicitTsDesc::computeRKSecondOrder``
* :class:`Sensitivity`    -- exact J v, J^T w, dR/dX . Xdot, (dR/dX)^T lambda

Arrays may be numpy arrays (host memory) or torch CUDA tensors (device
memory); results come back in the same kind of container as the input.
There is no CPU fallback: importing works anywhere, but creating a
:class:`Context` needs the built library and a CUDA device, and fails loudly
otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

from . import workloads  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaerof_gpu.so")

AEROF_OK = 0
ERRORS = {-1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "ETIMEDOUT", -5: "ESINGULAR", -6: "ESTATE",
          -7: "EDIVERGED"}
REC_CONSTANT, REC_VANALBADA, REC_LINEAR = 1, 2, 3
KERNEL_BLOCKED, KERNEL_EDGE = 0, 1
PREC_FP32, PREC_FP64 = 32, 64
PC_JACOBI, PC_ILU0 = 0, 1

# every entry point of include/aerof_gpu.h
EXPORTS = [
    "aerof_gpu_create", "aerof_gpu_destroy", "aerof_gpu_set_stream", "aerof_gpu_launch_count",
    "aerof_gpu_last_error",
    "aerof_gpu_set_mesh", "aerof_gpu_mesh_sizes", "aerof_gpu_get_edges", "aerof_gpu_get_geometry",
    "aerof_gpu_residual", "aerof_gpu_gradients", "aerof_gpu_timestep", "aerof_gpu_rk2",
    "aerof_gpu_jacobian", "aerof_gpu_get_jacobian", "aerof_gpu_matvec", "aerof_gpu_prec_setup",
    "aerof_gpu_prec_apply", "aerof_gpu_gmres", "aerof_gpu_newton",
    "aerof_gpu_jvp", "aerof_gpu_vjp", "aerof_gpu_dRdX", "aerof_gpu_dRdX_T", "aerof_gpu_adjoint_products",
    "aerof_gpu_residual_async", "aerof_gpu_status", "aerof_gpu_profile", "aerof_gpu_timers",
    "aerof_gpu_update_coordinates", "aerof_gpu_linearized_solve", "aerof_gpu_residual_noalloc",
    "aerof_gpu_h2_evaluate", "aerof_gpu_h2_apply", "aerof_gpu_h2_release", "aerof_gpu_set_exact_operator",
    "aerof_gpu_linearized_solve_batch", "aerof_gpu_set_preconditioner", "aerof_gpu_set_jacobian",
    "aerof_gpu_matvec_fd", "aerof_gpu_set_owned_rows", "aerof_gpu_set_viscosity",
    "aerof_gpu_set_turbulence", "aerof_gpu_residual_sa",
    "aerof_sower_open", "aerof_sower_close", "aerof_sower_num_subdomains", "aerof_sower_subdomain_sizes",
    "aerof_sower_read_subdomain", "aerof_sower_last_error",
]
TIMER_NAMES = ["nodal_grad", "fv_term", "time_step", "fv_jac", "prec_setup", "ksp_matvec", "ksp_other", "fv_edges"]


class AerofError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"aerof_gpu error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [("gamma", C.c_double), ("beta", C.c_double), ("reconstruction", C.c_int),
                ("failsafe", C.c_int), ("device", C.c_int), ("residual_kernel", C.c_int),
                ("reserved", C.c_int * 4)]


class NewtonParams(C.Structure):
    _fields_ = [("cfl0", C.c_double), ("cfl_min", C.c_double), ("cfl_max", C.c_double),
                ("ser", C.c_double), ("ksp_eps", C.c_double), ("tol", C.c_double),
                ("ksp_krylov", C.c_int), ("ksp_maxits", C.c_int), ("max_steps", C.c_int),
                ("precision", C.c_int), ("reserved", C.c_int * 4)]


class ViscousParams(C.Structure):
    _fields_ = [("model", C.c_int), ("reynolds_mu", C.c_double), ("prandtl", C.c_double),
                ("bulk_viscosity", C.c_double), ("sutherland_alpha", C.c_double), ("sutherland_Ts", C.c_double),
                ("reserved", C.c_int * 4)]


class SAParams(C.Structure):
    _fields_ = [("cb1", C.c_double), ("cb2", C.c_double), ("cw2", C.c_double), ("cw3", C.c_double),
                ("cv1", C.c_double), ("cv2", C.c_double), ("sigma", C.c_double), ("vkcst", C.c_double),
                ("prandtl_turbulent", C.c_double), ("fv3", C.c_int), ("reserved", C.c_int * 3)]


# Spalart-Allmaras constants: SAModelData's and TurbulenceClosureData's
# defaults (IoDataCore.C:1411-1418, 1839)
SA_DEFAULTS = dict(cb1=0.1355, cb2=0.622, cw2=0.3, cw3=2.0, cv1=7.1, cv2=5.0, sigma=2.0 / 3.0, vkcst=0.41,
                   prandtl_turbulent=0.9, fv3=0)


class NewtonResult(C.Structure):
    _fields_ = [("steps", C.c_int), ("linear_its", C.c_int), ("rel_residual", C.c_double),
                ("seconds", C.c_double), ("redos", C.c_int), ("reserved", C.c_int * 3)]


_lib = None


def library(path: str | None = None):
    """Load libaerof_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise AerofError(-3, f"{p} is missing: build it with `python -m aerof_dev_b200.build`")
        L = C.CDLL(p)
        vp, dp, ip = C.c_void_p, C.c_void_p, C.c_void_p
        sig = {
            "aerof_gpu_create": [C.POINTER(Config), C.POINTER(C.c_void_p)],
            "aerof_gpu_destroy": [vp],
            "aerof_gpu_set_stream": [vp, vp],
            "aerof_gpu_launch_count": [vp],
            "aerof_gpu_last_error": [vp, C.c_char_p, C.c_int],
            "aerof_gpu_set_mesh": [vp, C.c_int, C.c_int, C.c_int, dp, ip, ip, ip, dp],
            "aerof_gpu_mesh_sizes": [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)],
            "aerof_gpu_get_edges": [vp, ip],
            "aerof_gpu_get_geometry": [vp, dp, dp, dp, dp],
            "aerof_gpu_residual": [vp, dp, dp],
            "aerof_gpu_gradients": [vp, dp, dp, dp, dp],
            "aerof_gpu_timestep": [vp, dp, C.c_double, dp],
            "aerof_gpu_rk2": [vp, dp, C.c_double, C.c_int],
            "aerof_gpu_jacobian": [vp, dp, dp, C.c_int],
            "aerof_gpu_get_jacobian": [vp, dp],
            "aerof_gpu_matvec": [vp, dp, dp, C.c_int],
            "aerof_gpu_prec_setup": [vp],
            "aerof_gpu_prec_apply": [vp, dp, dp, C.c_int],
            "aerof_gpu_gmres": [vp, dp, dp, C.c_int, C.c_int, C.c_double, C.c_int,
                                C.POINTER(C.c_int), C.POINTER(C.c_double)],
            "aerof_gpu_newton": [vp, dp, C.POINTER(NewtonParams), C.POINTER(NewtonResult), dp],
            "aerof_gpu_jvp": [vp, dp, dp, dp],
            "aerof_gpu_vjp": [vp, dp, dp, dp],
            "aerof_gpu_dRdX": [vp, dp, dp, dp],
            "aerof_gpu_dRdX_T": [vp, dp, dp, dp],
            "aerof_gpu_adjoint_products": [vp, dp, dp, dp, dp],
            "aerof_gpu_residual_async": [vp, dp, dp],
            "aerof_gpu_status": [vp],
            "aerof_gpu_profile": [vp, C.c_int],
            "aerof_gpu_timers": [vp, dp, dp, C.c_int],
            "aerof_gpu_update_coordinates": [vp, dp],
            "aerof_gpu_residual_noalloc": [vp, dp, dp],
            "aerof_gpu_linearized_solve": [vp, dp, dp, dp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                           C.POINTER(C.c_int), C.POINTER(C.c_double)],
            "aerof_gpu_h2_evaluate": [vp, dp],
            "aerof_gpu_h2_apply": [vp, dp, dp, C.c_int],
            "aerof_gpu_h2_release": [vp],
            "aerof_gpu_set_exact_operator": [vp, C.c_int],
            "aerof_gpu_linearized_solve_batch": [vp, dp, C.c_int, dp, dp, C.c_int, C.c_int, C.c_double, C.c_int,
                                                 C.c_int, dp, dp],
            "aerof_gpu_set_preconditioner": [vp, C.c_int],
            "aerof_gpu_set_jacobian": [vp, dp, C.c_int],
            "aerof_gpu_matvec_fd": [vp, dp, dp, dp, dp, C.c_int, dp, C.POINTER(C.c_double)],
            "aerof_gpu_set_owned_rows": [vp, C.c_int],
            "aerof_gpu_set_viscosity": [vp, C.POINTER(ViscousParams)],
            "aerof_gpu_set_turbulence": [vp, C.POINTER(SAParams), dp, dp],
            "aerof_gpu_residual_sa": [vp, dp, dp],
        }
        for name, args in sig.items():
            if hasattr(L, name):
                f = getattr(L, name)
                f.argtypes = args
                f.restype = C.c_int
        _lib = L
    return _lib


# ----------------------------------------------------------------- buffers
def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


class _Arg:
    """Pointer to a float64/int32 array: numpy (host) or torch CUDA tensor."""

    def __init__(self, a, dtype, shape=None, writable=False):
        if _is_torch(a):
            import torch
            want = torch.float64 if dtype == np.float64 else torch.int32
            if a.dtype != want or not a.is_contiguous():
                if writable:
                    raise ValueError("output tensors must be contiguous with the right dtype")
                a = a.to(want).contiguous()
            self.obj = a
            self.ptr = C.c_void_p(a.data_ptr())
        else:
            if writable:
                if not (isinstance(a, np.ndarray) and a.dtype == dtype and a.flags.c_contiguous):
                    raise ValueError("output arrays must be C-contiguous " + str(np.dtype(dtype)))
                self.obj = a
            else:
                self.obj = np.ascontiguousarray(a, dtype=dtype)
            self.ptr = C.c_void_p(self.obj.ctypes.data)
        if shape is not None and 0 not in shape and tuple(self.obj.shape) != tuple(shape):
            if int(np.prod(self.obj.shape)) != int(np.prod(shape)):
                raise ValueError(f"array of shape {tuple(self.obj.shape)}, expected {tuple(shape)}")


def _like(a, shape, dtype=np.float64):
    if _is_torch(a):
        import torch
        return torch.empty(shape, dtype=torch.float64 if dtype == np.float64 else torch.int32, device=a.device)
    return np.empty(shape, dtype=dtype)


_CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy


def launch_count() -> int:
    """Kernels the library launched since the previous call (process-wide)."""
    n = C.c_longlong(0)
    rc = library().aerof_gpu_launch_count(C.byref(n))
    if rc != 0:
        raise AerofError(rc, "aerof_gpu_launch_count")
    return int(n.value)


class _StreamOrdered:
    """The library's entry points, each called after the context has been
    put on torch's current stream (see ``Context._follow_torch``)."""

    def __init__(self, ctx, lib):
        self._ctx, self._lib = ctx, lib

    def __getattr__(self, name):
        fn = getattr(self._lib, name)
        ctx = self._ctx

        def call(*args):
            ctx._follow_torch()
            return fn(*args)
        return call


class Context:
    """One GPU context: ``aerof_gpu_create`` + ``aerof_gpu_set_mesh``.

    Unless ``set_stream`` chose a stream, the context's work is ordered on
    torch's current stream whenever torch has initialised CUDA, so device
    tensors produced by torch are complete before the library reads them."""

    def __init__(self, reconstruction: int = REC_VANALBADA, gamma: float = 1.4, beta: float = 1.0 / 3.0,
                 failsafe: int = 0, device: int = 0, residual_kernel: int = KERNEL_BLOCKED):
        self._raw = library()
        self._explicit_stream = False
        self._torch_stream = None
        self.h = None
        self.L = _StreamOrdered(self, self._raw)
        cfg = Config(gamma, beta, reconstruction, failsafe, device, residual_kernel)
        h = C.c_void_p()
        self._check(self._raw.aerof_gpu_create(C.byref(cfg), C.byref(h)), None)
        self.h = h
        self.cfg = cfg
        self.N = self.E = self.F = 0

    def _follow_torch(self):
        if self._explicit_stream or not self.h:
            return
        torch = sys.modules.get("torch")
        if torch is None or not torch.cuda.is_initialized():
            return
        hs = torch.cuda.current_stream(self.cfg.device).cuda_stream or _CUDA_STREAM_LEGACY
        if hs != self._torch_stream:
            self._raw.aerof_gpu_set_stream(self.h, C.c_void_p(hs))
            self._torch_stream = hs

    def _check(self, rc: int, h=0):
        if rc < 0:
            msg = ""
            hh = self.h if h == 0 else h
            if hh:
                buf = C.create_string_buffer(512)
                self._raw.aerof_gpu_last_error(hh, buf, 512)
                msg = buf.value.decode()
            raise AerofError(rc, msg)
        return rc

    def close(self):
        if getattr(self, "h", None):
            self._raw.aerof_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        """Run the context's work on a CUDA stream: a ``torch.cuda.Stream``, a
        raw ``cudaStream_t`` handle, or None for the context's own stream.  A
        handle of 0 is the legacy default stream (torch reports its default
        stream as 0), passed to the library as ``cudaStreamLegacy``."""
        if stream is None:
            h = 0
        else:
            h = getattr(stream, "cuda_stream", stream) or _CUDA_STREAM_LEGACY
        self._explicit_stream = stream is not None
        self._torch_stream = None
        self._check(self._raw.aerof_gpu_set_stream(self.h, C.c_void_p(h)))

    def set_mesh(self, X, tets, faces, codes, Ub):
        X = _Arg(X, np.float64)
        t = _Arg(tets, np.int32)
        f = _Arg(faces, np.int32)
        c = _Arg(codes, np.int32)
        ub = _Arg(Ub, np.float64)
        N, T, F = X.obj.shape[0], t.obj.shape[0], f.obj.shape[0]
        self._check(self.L.aerof_gpu_set_mesh(self.h, N, T, F, X.ptr, t.ptr, f.ptr, c.ptr, ub.ptr))
        n, e, ff = C.c_int(), C.c_int(), C.c_int()
        self._check(self.L.aerof_gpu_mesh_sizes(self.h, C.byref(n), C.byref(e), C.byref(ff)))
        self.N, self.E, self.F = n.value, e.value, ff.value
        return self

    def set_owned_rows(self, n_owned: int):
        """Rows [n_owned, N) are ghost rows of a subdomain mesh."""
        self._check(self.L.aerof_gpu_set_owned_rows(self.h, int(n_owned)))

    def set_viscosity(self, model: int = 1, reynolds_mu: float = 100.0, prandtl: float = 0.72,
                      bulk_viscosity: float = 0.0, sutherland_alpha: float = 1.0, sutherland_Ts: float = 0.0):
        """Laminar viscous Galerkin term in every residual (model 0 off,
        1 constant viscosity, 2 Sutherland)."""
        p = ViscousParams(model, reynolds_mu, prandtl, bulk_viscosity, sutherland_alpha, sutherland_Ts)
        self._check(self.L.aerof_gpu_set_viscosity(self.h, C.byref(p)))

    def set_turbulence(self, d2wall, Ub, **constants):
        """Spalart-Allmaras model on (wall distances d2wall [N], conservative
        free stream Ub [6] with rho nu~ last, constants overriding
        SA_DEFAULTS); d2wall None turns it off."""
        if d2wall is None:
            self._check(self.L.aerof_gpu_set_turbulence(self.h, None, None, None))
            return
        c = dict(SA_DEFAULTS, **constants)
        p = SAParams(c["cb1"], c["cb2"], c["cw2"], c["cw3"], c["cv1"], c["cv2"], c["sigma"], c["vkcst"],
                     c["prandtl_turbulent"], int(c["fv3"]))
        d = _Arg(d2wall, np.float64, (self.N,))
        ub = _Arg(np.asarray(Ub, dtype=np.float64), np.float64, (6,))
        self._check(self.L.aerof_gpu_set_turbulence(self.h, C.byref(p), d.ptr, ub.ptr))

    def status(self) -> int:
        """Wait for the stream; unphysical count of async calls since last status."""
        return self._check(self.L.aerof_gpu_status(self.h))

    def set_preconditioner(self, pc: int):
        """Preconditioner of the Krylov solvers: PC_JACOBI or PC_ILU0."""
        self._check(self.L.aerof_gpu_set_preconditioner(self.h, int(pc)))

    def profile(self, enable: bool = True):
        self._check(self.L.aerof_gpu_profile(self.h, int(enable)))

    def timers(self) -> dict:
        """Per-category device milliseconds and interval counts (resets them)."""
        ms = np.zeros(8); cnt = np.zeros(8, dtype=np.int64)
        self._check(self.L.aerof_gpu_timers(self.h, C.c_void_p(ms.ctypes.data), C.c_void_p(cnt.ctypes.data), 8))
        return {n: (float(m), int(c)) for n, m, c in zip(TIMER_NAMES, ms, cnt)}

    @classmethod
    def from_mesh(cls, mesh: dict, Ub, **kw) -> "Context":
        ctx = cls(**kw)
        return ctx.set_mesh(mesh["X"], mesh["tets"], mesh["faces"], mesh["codes"], Ub)

    def update_coordinates(self, X):
        x = _Arg(X, np.float64, (self.N, 3))
        self._check(self.L.aerof_gpu_update_coordinates(self.h, x.ptr))

    def edges(self) -> np.ndarray:
        e = np.empty((self.E, 2), dtype=np.int32)
        self._check(self.L.aerof_gpu_get_edges(self.h, C.c_void_p(e.ctypes.data)))
        return e

    def geometry(self) -> dict:
        en = np.empty((self.E, 3)); fn = np.empty((max(self.F, 1), 3)); cv = np.empty(self.N)
        R = np.empty((self.N, 6))
        p = lambda a: C.c_void_p(a.ctypes.data)
        self._check(self.L.aerof_gpu_get_geometry(self.h, p(en), p(fn), p(cv), p(R)))
        return {"edge_normal": en, "face_normal": fn[: self.F], "ctrl_vol": cv, "lsq_R": R}


class SpaceOperator:
    """``SpaceOperator<5>`` on the GPU (SpaceOperator.C:524-634)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def computeResidual(self, U, R=None):
        """R = residual(U) / ctrlVol.  Returns (R, n_unphysical)."""
        ctx = self.ctx
        u = _Arg(U, np.float64, (ctx.N, 5))
        R = _like(U, (ctx.N, 5)) if R is None else R
        r = _Arg(R, np.float64, (ctx.N, 5), writable=True)
        bad = ctx._check(ctx.L.aerof_gpu_residual(ctx.h, u.ptr, r.ptr))
        return r.obj, bad

    def computeResidualSA(self, U, R=None):
        """Spalart-Allmaras residual of U [N][6] (after Context.set_turbulence).
        Returns (R, n_unphysical)."""
        ctx = self.ctx
        u = _Arg(U, np.float64, (ctx.N, 6))
        R = _like(U, (ctx.N, 6)) if R is None else R
        r = _Arg(R, np.float64, (ctx.N, 6), writable=True)
        bad = ctx._check(ctx.L.aerof_gpu_residual_sa(ctx.h, u.ptr, r.ptr))
        return r.obj, bad

    def computeResidualAsync(self, U, R):
        """Enqueue R = residual(U) for device tensors without waiting."""
        ctx = self.ctx
        u = _Arg(U, np.float64, (ctx.N, 5))
        r = _Arg(R, np.float64, (ctx.N, 5), writable=True)
        ctx._check(ctx.L.aerof_gpu_residual_async(ctx.h, u.ptr, r.ptr))
        return r.obj

    def computeResidualNoAlloc(self, U, R):
        """R = residual(U) for device tensors through the entry point that
        allocates nothing (fixed 16 MiB scratch, meshes up to ~40k nodes)."""
        ctx = self.ctx
        u = _Arg(U, np.float64, (ctx.N, 5))
        r = _Arg(R, np.float64, (ctx.N, 5), writable=True)
        bad = ctx._check(ctx.L.aerof_gpu_residual_noalloc(ctx.h, u.ptr, r.ptr))
        return r.obj, bad

    def computeGradients(self, V):
        ctx = self.ctx
        v = _Arg(V, np.float64, (ctx.N, 5))
        out = [_like(V, (ctx.N, 5)) for _ in range(3)]
        a = [_Arg(o, np.float64, writable=True) for o in out]
        ctx._check(ctx.L.aerof_gpu_gradients(ctx.h, v.ptr, a[0].ptr, a[1].ptr, a[2].ptr))
        return tuple(x.obj for x in a)

    def computeTimeStep(self, U, cfl):
        ctx = self.ctx
        u = _Arg(U, np.float64, (ctx.N, 5))
        dt = _like(U, (ctx.N,))
        d = _Arg(dt, np.float64, writable=True)
        ctx._check(ctx.L.aerof_gpu_timestep(ctx.h, u.ptr, float(cfl), d.ptr))
        return d.obj


class ExplicitRK2:
    """``ExplicitTsDesc::computeRKSecondOrder`` with local time stepping."""

    def __init__(self, ctx: Context, cfl: float):
        self.ctx, self.cfl = ctx, cfl

    def run(self, U, nsteps: int):
        ctx = self.ctx
        if _is_torch(U):
            out = U.clone()
        else:
            out = np.array(U, dtype=np.float64, copy=True, order="C")
        a = _Arg(out, np.float64, (ctx.N, 5), writable=True)
        bad = ctx._check(ctx.L.aerof_gpu_rk2(ctx.h, a.ptr, float(self.cfl), int(nsteps)))
        return a.obj, bad


class MatVecProdH1:
    """Assembled first-order Jacobian (``MatVecProdH1``, MatVecProd.C:945-1208)."""

    def __init__(self, ctx: Context, precision: int = PREC_FP32):
        self.ctx, self.precision = ctx, precision

    def evaluate(self, U, dt=None):
        ctx = self.ctx
        u = _Arg(U, np.float64, (ctx.N, 5))
        d = _Arg(dt, np.float64, (ctx.N,)) if dt is not None else None
        ctx._check(ctx.L.aerof_gpu_jacobian(ctx.h, u.ptr, d.ptr if d else None, int(self.precision)))

    def apply(self, p, transpose=False):
        ctx = self.ctx
        a = _Arg(p, np.float64, (ctx.N, 5))
        y = _like(p, (ctx.N, 5))
        b = _Arg(y, np.float64, writable=True)
        ctx._check(ctx.L.aerof_gpu_matvec(ctx.h, a.ptr, b.ptr, int(transpose)))
        return b.obj

    def applyTranspose(self, p):
        return self.apply(p, transpose=True)

    def set_blocks(self, A):
        """Make an operator given in MvpMat layout a[N+2E][5][5] (reference
        numbering) the context's H1 in this object's precision."""
        ctx = self.ctx
        a = _Arg(A, np.float64, (ctx.N + 2 * ctx.E, 5, 5))
        ctx._check(ctx.L.aerof_gpu_set_jacobian(ctx.h, a.ptr, int(self.precision)))

    def blocks(self) -> np.ndarray:
        """The operator in MvpMat layout a[N+2E][5][5] (reference numbering)."""
        ctx = self.ctx
        A = np.empty((ctx.N + 2 * ctx.E, 5, 5))
        ctx._check(ctx.L.aerof_gpu_get_jacobian(ctx.h, C.c_void_p(A.ctypes.data)))
        return A


class MatVecProdFD:
    """``MatVecProdFD`` (MatVecProd.C:262-372): finite-difference products
    of the residual at the state given to ``evaluate``."""

    def __init__(self, ctx: Context, fd_order: int = 1):
        self.ctx, self.fd_order = ctx, fd_order
        self.U = self.F = self.dt = None

    def evaluate(self, U, F=None, dt=None):
        """Keep the linearisation point (and R(U) when known, and the time
        steps of the backward-Euler term)."""
        self.U, self.F, self.dt = U, F, dt

    def apply(self, p):
        ctx = self.ctx
        u = _Arg(self.U, np.float64, (ctx.N, 5))
        f = _Arg(self.F, np.float64, (ctx.N, 5)) if self.F is not None else None
        d = _Arg(self.dt, np.float64, (ctx.N,)) if self.dt is not None else None
        a = _Arg(p, np.float64, (ctx.N, 5))
        y = _like(p, (ctx.N, 5))
        b = _Arg(y, np.float64, writable=True)
        eps = C.c_double()
        ctx._check(ctx.L.aerof_gpu_matvec_fd(ctx.h, u.ptr, f.ptr if f else None, a.ptr, d.ptr if d else None,
                                             int(self.fd_order), b.ptr, C.byref(eps)))
        self.eps = eps.value
        return b.obj


class JacobiPrec:
    """Block-Jacobi preconditioner (``JacobiPrec``, KspPrec.C:9-124); with
    ``Context.set_preconditioner(PC_ILU0)`` the same calls set up and apply
    the block ILU(0) preconditioner (``IluPrec``, KspPrec.C:138-330)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def setup(self):
        self.ctx._check(self.ctx.L.aerof_gpu_prec_setup(self.ctx.h))

    def apply(self, x, transpose=False):
        ctx = self.ctx
        a = _Arg(x, np.float64, (ctx.N, 5))
        y = _like(x, (ctx.N, 5))
        b = _Arg(y, np.float64, writable=True)
        ctx._check(ctx.L.aerof_gpu_prec_apply(ctx.h, a.ptr, b.ptr, int(transpose)))
        return b.obj

    def applyT(self, x):
        return self.apply(x, transpose=True)


class GmresSolver:
    """``GmresSolver`` (KspSolver.C:351-492): right-preconditioned GMRES."""

    def __init__(self, ctx: Context, krylov: int = 30, maxits: int = 30, eps: float = 1e-2):
        self.ctx, self.krylov, self.maxits, self.eps = ctx, krylov, maxits, eps

    def solve(self, b, transpose=False):
        ctx = self.ctx
        bb = _Arg(b, np.float64, (ctx.N, 5))
        x = _like(b, (ctx.N, 5))
        xx = _Arg(x, np.float64, writable=True)
        its, res = C.c_int(), C.c_double()
        ctx._check(ctx.L.aerof_gpu_gmres(ctx.h, bb.ptr, xx.ptr, self.krylov, self.maxits, self.eps,
                                         int(transpose), C.byref(its), C.byref(res)))
        return xx.obj, its.value, res.value

    def solveT(self, b):
        return self.solve(b, transpose=True)


class ImplicitSteadySolver:
    """Pseudo-transient backward-Euler Newton with GMRES, preconditioned by
    block-Jacobi or block ILU(0) (Context.set_preconditioner)."""

    def __init__(self, ctx: Context, precision: int = PREC_FP32, cfl0: float = 10.0, cfl_min: float = 0.0,
                 cfl_max: float = 1e4, ser: float = 0.7, ksp_eps: float = 1e-2, krylov: int = 30,
                 maxits: int = 30, tol: float = 1e-8, max_steps: int = 500):
        self.ctx = ctx
        self.p = NewtonParams(cfl0, cfl_min, cfl_max, ser, ksp_eps, tol, krylov, maxits, max_steps, precision)

    def solve(self, U):
        ctx = self.ctx
        out = U.clone() if _is_torch(U) else np.array(U, dtype=np.float64, copy=True, order="C")
        a = _Arg(out, np.float64, (ctx.N, 5), writable=True)
        hist = np.zeros(self.p.max_steps + 1)
        res = NewtonResult()
        ctx._check(ctx.L.aerof_gpu_newton(ctx.h, a.ptr, C.byref(self.p), C.byref(res),
                                          C.c_void_p(hist.ctypes.data)))
        return a.obj, {"steps": res.steps, "linear_its": res.linear_its, "rel_residual": res.rel_residual,
                       "seconds": res.seconds, "redos": res.redos, "history": hist[: res.steps + 1]}


class Sensitivity:
    """Exact linearisation of the residual and its transpose."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def _call(self, fn, U, x, width_in, width_out):
        ctx = self.ctx
        u = _Arg(U, np.float64, (ctx.N, 5))
        a = _Arg(x, np.float64, (ctx.N, width_in))
        y = _like(x, (ctx.N, width_out))
        b = _Arg(y, np.float64, writable=True)
        ctx._check(fn(ctx.h, u.ptr, a.ptr, b.ptr))
        return b.obj

    def jvp(self, U, v):
        return self._call(self.ctx.L.aerof_gpu_jvp, U, v, 5, 5)

    def vjp(self, U, w):
        return self._call(self.ctx.L.aerof_gpu_vjp, U, w, 5, 5)

    def dRdX(self, U, Xdot):
        return self._call(self.ctx.L.aerof_gpu_dRdX, U, Xdot, 3, 5)

    def dRdX_T(self, U, lam):
        return self._call(self.ctx.L.aerof_gpu_dRdX_T, U, lam, 5, 3)

    def adjoint_products(self, U, lam):
        """(J^T lam, (dR/dX)^T lam) from one reverse sweep."""
        ctx = self.ctx
        u = _Arg(U, np.float64, (ctx.N, 5))
        l = _Arg(lam, np.float64, (ctx.N, 5))
        a = _Arg(_like(lam, (ctx.N, 5)), np.float64, writable=True)
        b = _Arg(_like(lam, (ctx.N, 3)), np.float64, writable=True)
        ctx._check(ctx.L.aerof_gpu_adjoint_products(ctx.h, u.ptr, l.ptr, a.ptr, b.ptr))
        return a.obj, b.obj

    def h2_evaluate(self, U):
        """MatVecProdH2::evaluate: store the exact linearisation at U on the
        device (560 bytes per edge)."""
        ctx = self.ctx
        u = _Arg(U, np.float64, (ctx.N, 5))
        ctx._check(ctx.L.aerof_gpu_h2_evaluate(ctx.h, u.ptr))

    def h2_apply(self, p, transpose=False):
        """MatVecProdH2::apply (J p) or applyTranspose (J^T p) with the
        stored operator."""
        ctx = self.ctx
        a = _Arg(p, np.float64, (ctx.N, 5))
        b = _Arg(_like(p, (ctx.N, 5)), np.float64, writable=True)
        ctx._check(ctx.L.aerof_gpu_h2_apply(ctx.h, a.ptr, b.ptr, int(transpose)))
        return b.obj

    def h2_release(self):
        self.ctx._check(self.ctx.L.aerof_gpu_h2_release(self.ctx.h))

    def set_exact_operator(self, stored: bool):
        """Exact products of `solve`: re-evaluated per product (False) or
        from the operator stored once per solve (True)."""
        self.ctx._check(self.ctx.L.aerof_gpu_set_exact_operator(self.ctx.h, int(bool(stored))))

    def solve_batch(self, U, B, transpose=False, krylov=30, maxits=300, eps=1e-10, inner_its=20):
        """Solve J x_k = b_k (or J^T x_k = b_k) for every B[k] ([nrhs, N, 5])
        with one operator set-up (stored exact linearisation).  Returns X,
        iterations and final residual norms per right-hand side."""
        ctx = self.ctx
        u = _Arg(U, np.float64, (ctx.N, 5))
        nrhs = int(B.shape[0])
        bb = _Arg(B, np.float64, (nrhs, ctx.N, 5))
        xx = _Arg(_like(B, (nrhs, ctx.N, 5)), np.float64, writable=True)
        its = np.zeros(nrhs, dtype=np.int32)
        res = np.zeros(nrhs, dtype=np.float64)
        ctx._check(ctx.L.aerof_gpu_linearized_solve_batch(ctx.h, u.ptr, nrhs, bb.ptr, xx.ptr, krylov, maxits, eps,
                                                          int(transpose), int(inner_its),
                                                          C.c_void_p(its.ctypes.data), C.c_void_p(res.ctypes.data)))
        return xx.obj, its, res

    def solve(self, U, b, transpose=False, krylov=30, maxits=300, eps=1e-10, inner_its=0):
        """Solve J x = b (direct) or J^T x = b (adjoint) with the exact
        operator.  inner_its > 0: flexible GMRES preconditioned by that many
        mixed-precision GMRES iterations on the first-order operator."""
        ctx = self.ctx
        u = _Arg(U, np.float64, (ctx.N, 5))
        bb = _Arg(b, np.float64, (ctx.N, 5))
        x = _like(b, (ctx.N, 5))
        xx = _Arg(x, np.float64, writable=True)
        its, res = C.c_int(), C.c_double()
        ctx._check(ctx.L.aerof_gpu_linearized_solve(ctx.h, u.ptr, bb.ptr, xx.ptr, krylov, maxits, eps,
                                                    int(transpose), int(inner_its), C.byref(its), C.byref(res)))
        return xx.obj, its.value, res.value


IluPrec = JacobiPrec
