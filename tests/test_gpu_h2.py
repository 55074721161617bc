"""GPU stored exact linearisation (MatVecProdH2 evaluate / apply /
applyTranspose): J p against the oracle's dual-number linearisation, J^T w
against the matrix-free reverse sweep and by the adjoint identity, and the
linearised solves that apply it."""
import numpy as np
import pytest

from aerof_dev_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(7, 2), (7, 3), (7, 1), (17, 2)])
def case(request, gpu_lib, oracle_mod):
    n, rec = request.param
    m = W.make_lattice_mesh(n, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    o = oracle_mod.Oracle(m)
    U = W.smooth_state(m["X"], 0.8)
    ctx = gpu_lib.Context.from_mesh(m, Ub, reconstruction=rec)
    S = gpu_lib.Sensitivity(ctx)
    S.h2_evaluate(U)
    return rec, m, Ub, o, U, ctx, S


def test_h2_apply_matches_oracle(case):
    rec, m, Ub, o, U, ctx, S = case
    v = np.random.default_rng(21).standard_normal(U.shape) * 1e-2
    assert rel_l2(S.h2_apply(v), o.jvp(U, Ub, v, order=rec)) < 1e-11


def test_h2_apply_matches_matrix_free(case):
    rec, m, Ub, o, U, ctx, S = case
    rng = np.random.default_rng(22)
    v = rng.standard_normal(U.shape)
    w = rng.standard_normal(U.shape)
    assert rel_l2(S.h2_apply(v), S.jvp(U, v)) < 1e-12
    assert rel_l2(S.h2_apply(w, transpose=True), S.vjp(U, w)) < 1e-12


def test_h2_adjoint_identity(case):
    rec, m, Ub, o, U, ctx, S = case
    rng = np.random.default_rng(23)
    v = rng.standard_normal(U.shape)
    w = rng.standard_normal(U.shape)
    a = np.sum(w * S.h2_apply(v))
    b = np.sum(S.h2_apply(w, transpose=True) * v)
    assert abs(a - b) <= 1e-11 * max(abs(a), 1e-300)


def test_h2_is_deterministic(case):
    rec, m, Ub, o, U, ctx, S = case
    w = np.random.default_rng(24).standard_normal(U.shape)
    a = S.h2_apply(w, transpose=True)
    b = S.h2_apply(w, transpose=True)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("transpose", [False, True])
def test_linearized_solve_with_stored_operator(case, transpose):
    rec, m, Ub, o, U, ctx, S = case
    b = np.random.default_rng(25).standard_normal(U.shape)
    S.set_exact_operator(True)
    try:
        x, its, res = S.solve(U, b, transpose=transpose, krylov=30, maxits=600, eps=1e-10, inner_its=10)
    finally:
        S.set_exact_operator(False)
    # checked with the matrix-free products
    Ax = S.vjp(U, x) if transpose else S.jvp(U, x)
    assert np.linalg.norm(Ax - b) <= 1e-9 * np.linalg.norm(b)
    x2, its2, _ = S.solve(U, b, transpose=transpose, krylov=30, maxits=600, eps=1e-10, inner_its=10)
    assert rel_l2(x, x2) < 1e-8


def test_h2_needs_evaluate(gpu_lib):
    m = W.make_lattice_mesh(5, jitter=0.2, codes="channel")
    ctx = gpu_lib.Context.from_mesh(m, W.freestream(0.8), reconstruction=2)
    S = gpu_lib.Sensitivity(ctx)
    U = W.smooth_state(m["X"], 0.8)
    p = np.ones_like(U)
    with pytest.raises(gpu_lib.AerofError):
        S.h2_apply(p)
    S.h2_evaluate(U)
    S.h2_apply(p)
    # new coordinates invalidate the stored operator
    ctx.update_coordinates(m["X"] * 1.01)
    with pytest.raises(gpu_lib.AerofError):
        S.h2_apply(p)
    S.h2_evaluate(U)
    S.h2_release()
    with pytest.raises(gpu_lib.AerofError):
        S.h2_apply(p, transpose=True)


@pytest.mark.parametrize("nb,wide", [("64", "1"), ("128", "0")])
def test_h2_block_sizes(gpu_lib, monkeypatch, nb, wide):
    # 64-node blocks; the compact transpose kernel (gradient cotangents of
    # the two endpoints recomputed from the stored partials when gathered)
    monkeypatch.setenv("AEROF_BLOCK_NODES", nb)
    monkeypatch.setenv("AEROF_H2T_WIDE", wide)
    m = W.make_lattice_mesh(13, jitter=0.25, codes="channel")
    U = W.smooth_state(m["X"], 0.8)
    ctx = gpu_lib.Context.from_mesh(m, W.freestream(0.8), reconstruction=3)
    S = gpu_lib.Sensitivity(ctx)
    S.h2_evaluate(U)
    rng = np.random.default_rng(26)
    v = rng.standard_normal(U.shape)
    w = rng.standard_normal(U.shape)
    assert rel_l2(S.h2_apply(v), S.jvp(U, v)) < 1e-12
    assert rel_l2(S.h2_apply(w, transpose=True), S.vjp(U, w)) < 1e-12


def test_batched_solve_matches_single_solves(case):
    rec, m, Ub, o, U, ctx, S = case
    if m["X"].shape[0] > 400:
        pytest.skip("small mesh only")
    rng = np.random.default_rng(27)
    B = rng.standard_normal((3,) + U.shape)
    for transpose in (False, True):
        X, its, res = S.solve_batch(U, B, transpose=transpose, krylov=30, maxits=600, eps=1e-10, inner_its=10)
        assert X.shape == B.shape and len(its) == 3
        for k in range(3):
            Ax = S.vjp(U, X[k]) if transpose else S.jvp(U, X[k])
            assert np.linalg.norm(Ax - B[k]) <= 1e-9 * np.linalg.norm(B[k])
            assert res[k] <= 1.01e-10 * np.linalg.norm(B[k])
    # the stored operator stays evaluated at U after the batch
    v = rng.standard_normal(U.shape)
    assert rel_l2(S.h2_apply(v), S.jvp(U, v)) < 1e-12
