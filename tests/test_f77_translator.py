"""The Fortran 77 subset translator behind the Fortran golden vectors
(oracle/f77_to_c.py): precedence and associativity, literal kinds, integer
powers, column-major arrays, labelled and block DO loops, IF chains and the
intrinsics, on a routine written here for the purpose."""
import ctypes as C
import os
import importlib.util
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = """
      SUBROUTINE PROBE(n, a, b, out)
c     a comment line
      IMPLICIT NONE
      INTEGER n, i, j
      REAL*8 a, b, out(*), m(3,2)
      REAL*8 t
      out(1) = -a**2
      out(2) = a/b/2.d0
      out(3) = 0.1 + 0.d0
      out(4) = 0.1d0
      out(5) = 2.d0**3 - a**2**1
      out(6) = MAX(a, b, 3.d0) + MIN(a, b)
      out(7) = DSIGN(2.d0, -b) + DABS(-a) + DSQRT(b*b)
      DO 10 j = 1, 2
         DO i = 1, 3
            m(i, j) = 10.d0*i + j
         END DO
10    CONTINUE
      out(8) = m(2, 1)
      out(9) = m(3, 2)
      t = 0.d0
      do i = 1, n
        t = t + i
      enddo
      if (n .gt. 3) then
         out(10) = t
      else if (n .eq. 3) then
         out(10) = -t
      else
         out(10) = 0.d0
      end if
      out(11) = a - b - 1.d0
      out(12) = -a*b + 1.d0 
     &   + 2.d0
      END
"""


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    spec = importlib.util.spec_from_file_location("f77_to_c", os.path.join(ROOT, "oracle", "f77_to_c.py"))
    f77_to_c = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(f77_to_c)
    d = tmp_path_factory.mktemp("f77")
    f = d / "probe.f"
    f.write_text(SRC)
    c = d / "probe.c"
    f77_to_c.main(["f77_to_c.py", str(c), str(f)])
    so = d / "libprobe.so"
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-w", "-fPIC", "-shared", str(c), "-o", str(so), "-lm"])
    L = C.CDLL(str(so))
    return L


def _run(L, n, a, b):
    out = np.zeros(12)
    L.probe_f77_(C.byref(C.c_int(n)), C.byref(C.c_double(a)), C.byref(C.c_double(b)),
                 out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def test_translation_semantics(probe):
    a, b = 1.7, 0.3
    o = _run(probe, 4, a, b)
    assert o[0] == -(a * a)                             # ** above unary minus
    assert o[1] == (a / b) / 2.0                        # left to right
    assert o[2] == float(np.float32(0.1))               # a single precision literal
    assert o[3] == 0.1
    assert o[4] == 8.0 - a * a                          # ** right associative: a**(2**1)
    assert o[5] == 3.0 + b
    assert o[6] == -2.0 + a + abs(b)
    assert o[7] == 21.0 and o[8] == 32.0                # m(i, j) = 10 i + j, column-major
    assert o[9] == 10.0                                 # 1 + 2 + 3 + 4
    assert o[10] == (a - b) - 1.0
    assert o[11] == (-(a * b) + 1.0) + 2.0              # continuation line
    assert _run(probe, 3, a, b)[9] == -6.0
    assert _run(probe, 2, a, b)[9] == 0.0
