"""CPU tests of the oracle's solver restatements on small seeded systems."""
import numpy as np
import pytest

from lfric_core_b200 import meshgen as mg
from oracle import oracle as orc


def w0_setup(n=6, nl=5, seed=1):
    p = mg.w0_problem(n, nl, seed=seed)
    npc, cic = p.mesh.colour_lookup()
    op = orc.LmaOperator(p.ncell_2d, nl, 8, 8, p.map, p.map, p.undf, p.undf, p.lma, npc, cic)
    return p, op


def w2_setup(n=6, nl=5, seed=2):
    p = mg.w2_problem(n, nl, seed=seed)
    npc, cic = p.mesh.colour_lookup()
    op = orc.LmaOperator(p.ncell_2d, nl, 6, 6, p.map, p.map, p.undf, p.undf, p.lma, npc, cic)
    prm = mg.w2v_cma_params(nl)
    sub = mg.lma_block(p.lma, p.mesh.ncell_3d, 6, mg.W2V_DFS)
    band = orc.assemble_cma(sub, p.ncell_2d, nl, prm)
    diag = op.diagonal()
    prec = orc.Preconditioner.cma(p.ncell_2d, prm["nrow"], 3, p.map[:, 4], prm["indirection"], band,
                                  diag, p.undf)
    return p, op, prec, band, diag


def dense_of(op, n):
    A = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        A[:, j] = op.apply(e)
    return A


def test_coloured_apply_matches_dense_assembly():
    p, op = w0_setup(3, 2)
    A = dense_of(op, p.undf)
    # scatter the LMA densely in numpy and compare
    B = np.zeros_like(A)
    L = p.lma.reshape(8, 8, -1)  # [df2][df][ik]
    for c in range(p.ncell_2d):
        for k in range(2):
            for df in range(8):
                for df2 in range(8):
                    B[p.map[c, df] - 1 + k, p.map[c, df2] - 1 + k] += L[df2, df, c * 2 + k]
    np.testing.assert_allclose(A, B, atol=1e-14)
    np.testing.assert_allclose(np.diag(A), op.diagonal(), atol=1e-15)


@pytest.mark.parametrize("kind", ["cg", "bicgstab", "gmres"])
def test_oracle_solvers_converge(kind):
    p, op = w0_setup()
    P = orc.Preconditioner.diagonal(op.diagonal())
    x, info = orc.solve(kind, op, P, p.rhs, r_tol=1e-8, max_iter=2000)
    assert info.converged
    r = p.rhs - op.apply(x)
    assert np.linalg.norm(r) / np.linalg.norm(p.rhs) < 2e-8


def test_cma_preconditioner_is_exact_on_columns():
    p, op, prec, band, diag = w2_setup(3, 4)
    x = np.random.default_rng(0).standard_normal(p.undf)
    y = prec.apply(x)
    prm = mg.w2v_cma_params(4)
    for c in range(p.ncell_2d):
        b = band.reshape(p.ncell_2d, prm["nrow"], 3)[c]
        T = np.diag(b[:, 1]) + np.diag(b[1:, 0], -1) + np.diag(b[:-1, 2], 1)
        rows = p.map[c, 4] - 1 + np.arange(prm["nrow"])
        np.testing.assert_allclose(T @ y[rows], x[rows], atol=1e-12)
    other = np.ones(p.undf, bool)
    for c in range(p.ncell_2d):
        other[p.map[c, 4] - 1 + np.arange(prm["nrow"])] = False
    np.testing.assert_allclose(y[other], x[other] / diag[other], rtol=1e-15)


def test_gmres_cma_converges():
    p, op, prec, _, _ = w2_setup()
    x, info = orc.solve("gmres", op, prec, p.rhs, r_tol=1e-8, gcrk=10, max_iter=100)
    assert info.converged
    assert np.linalg.norm(p.rhs - op.apply(x)) / np.linalg.norm(p.rhs) < 1e-8


def test_reduction_order_does_not_change_iteration_count():
    p, op = w0_setup(8, 6)
    P = orc.Preconditioner.diagonal(op.diagonal())
    L = orc.lib()
    its = []
    for order in (0, 1):
        L.or_set_reduction_order(order)
        _, info = orc.solve("cg", op, P, p.rhs, r_tol=1e-8, max_iter=2000)
        its.append(info.iterations)
    L.or_set_reduction_order(0)
    assert its[0] == its[1]


def test_zero_rhs_converges_in_zero_iterations():
    p, op = w0_setup(3, 2)
    P = orc.Preconditioner.diagonal(op.diagonal())
    for kind in ("cg", "bicgstab", "gmres"):
        x, info = orc.solve(kind, op, P, np.zeros(p.undf))
        assert info.converged and info.iterations == 0
        assert np.all(x == 0)


def test_transpose_apply_is_adjoint():
    q = mg.w2_problem(3, 2, seed=9, keep_parts=True)
    npc, cic = q.mesh.colour_lookup()
    m3, u3 = q.extra["map_w3"], q.extra["undf_w3"]
    D = orc.LmaOperator(q.ncell_2d, 2, 1, 6, m3, q.map, u3, q.undf, q.extra["div"], npc, cic)
    Dt = orc.LmaOperator(q.ncell_2d, 2, 1, 6, m3, q.map, u3, q.undf, q.extra["div"], npc, cic,
                         transpose=True)
    rng = np.random.default_rng(1)
    u = rng.standard_normal(q.undf)
    w = rng.standard_normal(u3)
    np.testing.assert_allclose(w @ D.apply(u), u @ Dt.apply(w), rtol=1e-12)


@pytest.mark.parametrize("kind", ["fgmres", "gcr"])
def test_oracle_flexible_solvers_converge(kind):
    p, op, prec, _, _ = w2_setup(6, 7)
    x, info = orc.solve(kind, op, prec, p.rhs, r_tol=1e-8, max_iter=200, gcrk=8)
    assert info.converged
    r = p.rhs - op.apply(x)
    assert np.linalg.norm(r) / np.linalg.norm(p.rhs) < 2e-8
    if kind == "gcr":
        assert 1 <= info.iv_final <= 8


def test_oracle_fgmres_adds_correction_to_initial_guess():
    """fgmres_solve starts its residual from b (it assumes x0 = 0) and adds
    the correction to x: with x0 != 0 the result is x0 + A^-1 b."""
    p, op = w0_setup(5, 4)
    P = orc.Preconditioner.diagonal(op.diagonal())
    x_zero, _ = orc.solve("fgmres", op, P, p.rhs, r_tol=1e-10, max_iter=400, gcrk=10)
    x0 = mg.normal(5, p.undf)
    x_one, _ = orc.solve("fgmres", op, P, p.rhs, x0=x0, r_tol=1e-10, max_iter=400, gcrk=10)
    np.testing.assert_allclose(x_one, x0 + x_zero, rtol=0, atol=1e-12)


def test_oracle_gcr_relative_to_b_and_fgmres_zero_rhs():
    p, op, prec, _, _ = w2_setup(4, 3)
    z = np.zeros(p.undf)
    for kind in ("fgmres", "gcr"):
        x, info = orc.solve(kind, op, prec, z, r_tol=1e-8, max_iter=10, gcrk=4)
        assert info.converged and info.iterations == 0 and np.all(x == 0.0)


def test_oracle_jacobi_and_chebyshev_and_precondition_only():
    p, op = w0_setup(5, 4)
    d = op.diagonal()
    P = orc.Preconditioner.diagonal(d)
    # Jacobi with a damping that converges for this diagonally dominant-ish operator
    x, info = orc.solve("jacobi", op, P, p.rhs, r_tol=1e-6, a_tol=0.0, max_iter=5000,
                        rho_relax=0.5)
    assert info.converged
    r = p.rhs - op.apply(x)
    assert np.linalg.norm(r) <= 1e-6 * info.initial_norm * (1 + 1e-9)
    # Chebyshev with the spectrum of D^-1 A from a dense eigensolve
    A = dense_of(op, p.undf)
    ev = np.linalg.eigvals(A / d[:, None]).real
    x, info = orc.solve("chebyshev", op, P, p.rhs, max_iter=60, lmin=ev.min(), lmax=ev.max())
    assert info.final_rel < 1e-3
    # precondition only: x = D^-1 b
    x, info = orc.solve("precondition_only", op, P, p.rhs)
    np.testing.assert_array_equal(x, p.rhs / d)
    assert info.final_norm == pytest.approx(np.linalg.norm(p.rhs - op.apply(x)), rel=1e-12)
