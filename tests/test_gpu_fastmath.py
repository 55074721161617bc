"""Error of the fast FP64 reciprocal and reciprocal square root used by the
flux kernels (rcp_ / rsqrt_ in physics.cuh: the hardware rcp.approx /
rsqrt.approx seeds refined by Newton-Raphson, the cubic series step
r + r(e + e^2) for 1/x and two steps y + y/2 (1 - x y^2) for 1/sqrt x),
measured in ulps against correctly rounded values (computed on the host with
60-digit decimal arithmetic) beside CUDA's own 1.0/x and rsqrt(x), over a log-uniform
sweep of positive normal inputs and the ranges the flux arithmetic sees."""
import ctypes as C
import os
from decimal import Decimal, localcontext
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def probe(gpu_lib, tmp_path_factory):
    so = str(tmp_path_factory.mktemp("probe") / "libfastmath_probe.so")
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                           "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-shared",
                           os.path.join(HERE, "probes", "fastmath_probe.cu"), "-o", so])
    L = C.CDLL(so)
    L.fastmath_probe.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    L.fastmath_probe.restype = C.c_int
    return L


def _ulps(a, ref):
    """|a - ref| in units of the last place of ref (float64)."""
    return np.abs(a - ref) / np.spacing(np.abs(ref))


def test_fast_reciprocals_ulp_bounds(probe):
    rng = np.random.default_rng(20261203)
    x = np.concatenate([
        2.0 ** rng.uniform(-1000, 1000, 200000),          # log-uniform over normal doubles
        rng.uniform(0.5, 2.0, 100000),                     # densities, pressures near 1
        rng.uniform(1e-6, 1e3, 100000),                    # squared norms, sound speeds
        np.array([1.0, 2.0, 0.5, 3.0, 1.0 / 3.0, 1.4, 0.4, np.nextafter(1.0, 2.0), np.nextafter(1.0, 0.0)]),
    ]).astype(np.float64)
    out = np.empty((4, x.size))
    assert probe.fastmath_probe(x.ctypes.data, x.size, out.ctypes.data) == 0
    rcp_fast, rcp_cuda, rsq_fast, rsq_cuda = out
    # correctly rounded references: 60-digit decimal arithmetic, rounded once
    # to double (extended precision followed by a cast can round twice)
    with localcontext() as ctx:
        ctx.prec = 60
        rcp_ref = np.array([float(1 / Decimal(v)) for v in x.tolist()])
        rsq_ref = np.array([float(1 / Decimal(v).sqrt()) for v in x.tolist()])
    # CUDA's 1.0/x is the IEEE quotient: the extended-precision reference agrees
    assert _ulps(rcp_cuda, rcp_ref).max() <= 0.5
    e_rcp = _ulps(rcp_fast, rcp_ref)
    e_rsq = _ulps(rsq_fast, rsq_ref)
    e_rsq_cuda = _ulps(rsq_cuda, rsq_ref)
    print(f"rcp_ max {e_rcp.max():.3g} ulp (mean {e_rcp.mean():.3g}); rsqrt_ max {e_rsq.max():.3g} ulp "
          f"(mean {e_rsq.mean():.3g}); CUDA rsqrt max {e_rsq_cuda.max():.3g} ulp")
    assert e_rcp.max() <= 1.0
    assert e_rsq.max() <= 2.0
    assert np.isfinite(out).all()
