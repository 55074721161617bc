"""Generate golden vectors from the reference's own header-only code.

Runs oracle/_ref/ref_golden (built from the AERO-F sources by
``make -C oracle ref REF=<aerof tree>``) on seeded inputs and stores inputs
and outputs in tests/golden/reference_pointwise.npz.  Only this script needs
the reference tree; the tests read the committed .npz.

    python tests/golden/make_golden.py --ref /path/to/aerof
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_golden")
SEED = 20261203


def run(kind: str, rows: np.ndarray, width: int) -> np.ndarray:
    lines = [f"{kind} {rows.shape[0]}"]
    lines += [" ".join(f"{x:.17g}" for x in r) for r in rows]
    out = subprocess.run([DRIVER], input="\n".join(lines) + "\n", capture_output=True, text=True,
                         check=True).stdout
    vals = [list(map(float, ln.split())) for ln in out.splitlines() if ln and not ln.startswith("***")]
    arr = np.array(vals, dtype=np.float64)
    assert arr.shape == (rows.shape[0], width), (kind, arr.shape)
    return arr


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("AEROF_REFERENCE_TREE"),
                    help="AERO-F source tree (or set AEROF_REFERENCE_TREE)")
    a = ap.parse_args()
    if not a.ref:
        ap.error("name the AERO-F source tree with --ref or AEROF_REFERENCE_TREE")
    subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={a.ref}"])
    rng = np.random.Generator(np.random.PCG64(SEED))
    out = {}

    # reconstruction: beta=1/3, states near a Mach 0.8 free stream, plus the
    # a*b==0 (equal states, zero slope) and a*b<0 (opposite slope) branches
    n = 400
    Vi = np.column_stack([1 + 0.05 * rng.standard_normal(n), 1 + 0.1 * rng.standard_normal(n),
                          0.1 * rng.standard_normal(n), 0.1 * rng.standard_normal(n),
                          1.116 * (1 + 0.05 * rng.standard_normal(n))])
    Vj = Vi + 0.05 * rng.standard_normal((n, 5))
    ddij = 0.05 * rng.standard_normal((n, 5))
    ddji = 0.05 * rng.standard_normal((n, 5))
    Vj[:40] = Vi[:40]; ddij[:20] = 0.0; ddji[:20] = 0.0          # a*b == 0
    ddij[40:80] = -3.0 * (Vj[40:80] - Vi[40:80])                 # a*b < 0
    rec_in = np.column_stack([np.full(n, 1.0 / 3.0), Vi, ddij, Vj, ddji])
    out["rec_in"] = rec_in
    out["vanalbada_out"] = run("vanalbada", rec_in, 10)
    out["linear_out"] = run("linear", rec_in, 10)

    U = np.column_stack([1 + 0.1 * rng.random(n), rng.standard_normal((n, 3)), 3 + rng.random(n)])
    out["cons_in"] = U
    out["cons2prim_out"] = run("cons2prim", U, 5)
    out["prim2cons_out"] = run("prim2cons", out["cons2prim_out"], 5)

    m = 100
    Vm = out["cons2prim_out"][:m]
    mats = rng.standard_normal((m, 25))
    dv_in = np.column_stack([Vm, mats])
    out["dVdU_in"] = dv_in
    out["dVdU_out"] = run("dVdU", dv_in, 25)
    out["dUdV_out"] = run("dUdV", dv_in, 25)

    chk = np.array([[1, 0, 0, 0, 1], [-1, 0, 0, 0, 1], [1, 0, 0, 0, -1], [0, 0, 0, 0, 1],
                    [1, 0, 0, 0, 0], [1e-300, 0, 0, 0, 1e-300]], dtype=np.float64)
    out["check_in"] = chk
    out["check_out"] = run("check", chk, 1)

    blocks = rng.standard_normal((m, 25))
    for b in blocks[: m // 2]:
        b[[0, 6, 12, 18, 24]] += 6.0                                # diagonally dominant half
    out["invert_in"] = blocks
    out["invert_out"] = run("invert5", blocks, 26)

    dst = os.path.join(HERE, "reference_pointwise.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    sys.exit(main())
