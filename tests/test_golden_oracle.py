"""The oracle against the known-answer data of the reference's own pFUnit
kernel tests (tests/golden/kernel_goldens.json, made by extract_goldens.py).
CPU only."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as orc

G = json.loads((Path(__file__).parent / "golden" / "kernel_goldens.json").read_text())


def test_matrix_vector_golden():
    # matrix_vector_mod_test.pf:49-91: one cell, one layer, 4x2 matrix
    g = G["matrix_vector"]
    d = np.array(g["d"])  # (4, 2)
    x = np.array(g["x"])
    m = np.asfortranarray(d.reshape(1, 4, 2)).ravel(order="F")
    y = np.zeros(4)
    orc.lib().or_matrix_vector_code(1, 1, y, x, 1, m, 4, np.arange(1, 5, dtype=np.int32), 2,
                                    np.arange(1, 3, dtype=np.int32))
    np.testing.assert_allclose(y, d @ x, rtol=0, atol=g["tol"])


def test_tri_solve_golden():
    # sci_tri_solve_kernel_mod_test.pf:20-52; the reference tolerance is 1e10
    # (pins nothing), the 15-digit answer vector is re-pinned here at 1e-14
    g = G["tri_solve"]
    nz = g["nz"]
    y = np.zeros(nz)
    orc.lib().or_tri_solve_code(nz, y, np.array(g["x"]), np.full(nz, g["A0"]), np.full(nz, g["AP"]),
                                np.full(nz, g["AM"]), np.array([1], dtype=np.int32))
    np.testing.assert_allclose(y, g["answer"], rtol=0, atol=1e-14)
    # and it is the solution of the tridiagonal system
    A = np.diag(np.full(nz, g["A0"])) + np.diag(np.full(nz - 1, g["AP"]), 1) + \
        np.diag(np.full(nz - 1, g["AM"]), -1)
    np.testing.assert_allclose(A @ y, g["x"], atol=1e-13)


def _band(g, ncell=1):
    nrow = g["nrow"]
    band = np.zeros((ncell, nrow, 3))
    for i in range(nrow):
        row = g["first_row"] if i == 0 else g["last_row"] if i == nrow - 1 else g["interior_row"]
        band[:, i, :] = [0.0 if v is None else v for v in row]
    dense = np.zeros((nrow, nrow))
    for i in range(nrow):
        for j, off in enumerate((-1, 0, 1)):
            if 0 <= i + off < nrow:
                dense[i, i + off] = band[0, i, j]
    return band.ravel(), dense  # band is Fortran (3, nrow, ncell)


def test_cma_appinv_golden():
    # columnwise_op_appinv_kernel_mod_test.pf:68-160: A . appinv(x) == x
    g = G["cma_appinv"]
    band, dense = _band(g)
    nrow = g["nrow"]
    rng = np.random.default_rng(7)
    x = rng.random(nrow)
    y = np.zeros(nrow)
    ind = np.arange(1, nrow + 1, dtype=np.int32)
    orc.lib().or_columnwise_op_appinv_code(1, y, x, band, nrow, 3, np.array([1], dtype=np.int32), ind)
    np.testing.assert_allclose(dense @ y, x, atol=1e-14)


def test_cma_app_golden():
    # columnwise_op_app_kernel_mod_test.pf: banded product == dense matmul
    g = G["cma_app"]
    band, dense = _band(g)
    nrow = g["nrow"]
    x = np.random.default_rng(3).random(nrow)
    y = np.zeros(nrow)
    ind = np.arange(1, nrow + 1, dtype=np.int32)
    one = np.array([1], dtype=np.int32)
    orc.lib().or_columnwise_op_app_code(1, y, x, band, nrow, nrow, 3, 1, 1, 1, 1, one, ind, one, ind)
    np.testing.assert_allclose(y, dense @ x, atol=1e-15)


def test_cma_asm_golden():
    # columnwise_op_asm_kernel_mod_test.pf:34-107
    g = G["cma_asm"]
    nl = g["nlayers"]
    nrow = nl + 1
    ls = np.array(g["local_stencil"])
    lma = np.zeros((2, 2, nl))  # [df2][df1][ik]
    for i in range(2):
        for j in range(2):
            lma[j, i, :] = ls[i, j]
    cbd = np.array([[k, k + 1] for k in range(1, nl + 1)], dtype=np.int32)
    band = np.zeros(3 * nrow)
    orc.lib().or_columnwise_op_asm_code(1, nl, 1, nl, lma.ravel(), band, nrow, nrow, 3, 1, 1, 1, 1,
                                        2, cbd, 2, cbd)
    b = band.reshape(nrow, 3)
    np.testing.assert_allclose(b[0, 1:], g["band_first"][1:], atol=1e-15)
    np.testing.assert_allclose(b[-1, :2], g["band_last"][:2], atol=1e-15)
    for i in range(1, nrow - 1):
        np.testing.assert_allclose(b[i], g["band_interior"], atol=1e-15)


def test_field_vector_identities():
    # sci_field_vector_mod_test.pf: set_scalar, axpy, aypx, axpby, scale, norm, dot
    L = orc.lib()
    n = 5000
    rng = np.random.default_rng(11)
    x = rng.standard_normal(n)
    y = rng.standard_normal(n)
    z = np.empty(n)
    L.or_setval_c(z, 3.5, n)
    assert np.all(z == 3.5)
    w = y.copy()
    L.or_inc_x_plus_by(w, 0.25, x, n)
    np.testing.assert_allclose(w, y + 0.25 * x, rtol=1e-15)
    w = y.copy()
    L.or_inc_ax_plus_y(-2.0, w, x, n)
    np.testing.assert_allclose(w, -2.0 * y + x, rtol=1e-15, atol=1e-15)
    L.or_ax_plus_by(z, 2.0, x, 3.0, y, n)
    np.testing.assert_allclose(z, 2 * x + 3 * y, rtol=1e-14, atol=1e-14)
    w = x.copy()
    L.or_inc_a_times_x(1.5, w, n)
    np.testing.assert_allclose(w, 1.5 * x, rtol=0)
    np.testing.assert_allclose(np.sqrt(L.or_sumsq(x, n)), np.linalg.norm(x), rtol=1e-14)
    np.testing.assert_allclose(L.or_dot(x, y, n), x @ y, rtol=1e-12)


@pytest.mark.parametrize("n", [0, 1, 255, 2048, 2049, 10000, 1 << 20])
def test_blocked_sum_matches_exact(n):
    """The fixed blocked order is a valid sum order: it agrees with an exact
    (math.fsum) sum to rounding, and with the literal sequential loop."""
    import math
    rng = np.random.default_rng(n + 1)
    x = rng.standard_normal(n)
    y = rng.standard_normal(n)
    L = orc.lib()
    exact = math.fsum((x * y).tolist()) if n else 0.0
    L.or_set_reduction_order(0)
    blocked = L.or_dot(x, y, n)
    L.or_set_reduction_order(1)
    seq = L.or_dot(x, y, n)
    L.or_set_reduction_order(0)
    scale = math.fsum(np.abs(x * y).tolist()) if n else 1.0
    assert abs(blocked - exact) <= 1e-14 * max(scale, 1e-300) + 0.0
    assert abs(seq - exact) <= 1e-12 * max(scale, 1e-300) + 0.0


def _dense_of_band(Cb, cell=1):
    """Dense (nrow, ncol) matrix of one column of a band (zero outside the band)."""
    D = np.zeros((Cb.nrow, Cb.ncol))
    b = Cb.band.reshape(Cb.ncell_2d, Cb.nrow, Cb.bw)[cell - 1]
    for i in range(1, Cb.nrow + 1):
        jm = -((-(Cb.alpha * i - Cb.gamma_p)) // Cb.beta)
        for q in range(Cb.bw):
            j = jm + q
            if 1 <= j <= Cb.ncol:
                D[i - 1, j - 1] = b[i - 1, q]
    return D


def test_cma_mul_golden():
    """columnwise_op_mul_kernel_mod_test.pf: D^T D of the W3 <- Wtheta
    difference operator, against the dense product (sizes from get_cma_size)."""
    g = G["cma_mul"]
    nl = g["nlayers"]
    # W3 <- Wtheta: nrow nl, ncol nl+1, alpha = beta = 1, g_m 1, g_p 0, bw 2
    D = orc.Band(1, nl, nl + 1, 2, 1, 1, 1, 0, np.tile(g["D_band"], nl))
    DT = orc.Band(1, nl + 1, nl, 2, 1, 1, 0, 1, np.tile(g["DT_band"], nl + 1))
    C = orc.cma_product(DT, D)
    assert (C.nrow, C.ncol, C.bw, C.gamma_m, C.gamma_p) == (nl + 1, nl + 1, 3, 1, 1)
    Dd = np.zeros((nl, nl + 1))
    for i in range(nl):
        Dd[i, i], Dd[i, i + 1] = g["D_band"]
    np.testing.assert_allclose(_dense_of_band(C), Dd.T @ Dd, atol=g["reference_tol"])
    np.testing.assert_array_equal(_dense_of_band(C), Dd.T @ Dd)


def test_cma_scaledadd_golden():
    """columnwise_op_scaledadd_kernel_mod_test.pf: mu M + nu D^T D on W3."""
    g = G["cma_scaledadd"]
    nl = g["nlayers"]
    M = orc.Band(1, nl, nl, 1, 1, 1, 0, 0, np.tile(g["M_band"], nl))
    DTD = orc.Band(1, nl, nl, 3, 1, 1, 1, 1, np.tile(g["DTD_band"], nl))
    C = orc.cma_scaledadd(M, DTD, g["mu"], g["nu"])
    dense = g["mu"] * np.eye(nl) + g["nu"] * (2 * np.eye(nl) + np.eye(nl, k=1) + np.eye(nl, k=-1))
    np.testing.assert_allclose(_dense_of_band(C), dense, atol=g["reference_tol"])


def test_cma_m2v_lumped_inv_golden():
    """columnwise_op_asm_m2v_lumped_inv_kernel_mod_test.pf: inverse lumped W2V
    mass, 3 on the end rows and 3/2 inside (band index 1)."""
    g = G["cma_m2v_lumped_inv"]
    nl = g["nlayers"]
    st = np.zeros((2, 2, nl))  # Fortran (ncell_3d, 2, 2) as [df2][df1][ik]
    for k in range(nl):
        st[:, :, k] = np.array(g["local_stencil"]).T
    cbd = np.array([[k + 1, k + 2] for k in range(nl)], dtype=np.int32)  # col_bmap(df, k)
    C = orc.cma_m2v_lumped_inv(st, 1, nl, 2, cbd, nl + 1, 3, (1, 1, 1, 1))
    first = C.band.reshape(nl + 1, 3)[:, 0]
    expect = [g["answer_end_rows"]] + [g["answer_interior_rows"]] * (nl - 1) + [g["answer_end_rows"]]
    np.testing.assert_allclose(first, expect, rtol=0, atol=g["reference_tol"])
    assert np.all(C.band.reshape(nl + 1, 3)[:, 1:] == 0.0)


def test_cma_diag_hmht_golden():
    """columnwise_op_asm_diag_hmht_kernel_mod_test.pf: sum_k rho_k^2 / sigma_k
    on the W3 diagonal."""
    g = G["cma_diag_hmht"]
    nl = g["nlayers"]
    Dh = np.zeros((4, 1, nl))  # Fortran (ncell_3d, 1, 4) as [df3][df1][ik]
    M2h = np.zeros((4, 4, nl))
    for k in range(nl):
        Dh[:, 0, k] = g["rho"]
        M2h[:, :, k] = np.diag(g["sigma"])
    cbd = np.arange(1, nl + 1, dtype=np.int32).reshape(nl, 1)
    C = orc.cma_diag_hmht(Dh, M2h, 1, nl, 1, 4, cbd, nl, 1, (1, 1, 0, 0))
    np.testing.assert_allclose(C.band, g["answer"], rtol=0, atol=g["reference_tol"])


def test_operator_x_plus_ay_golden():
    # operator_algebra_kernel_mod_test.pf test_x_plus_ay: one cell, one layer,
    # 3x2 operators constant per column, a = 2
    g = G["operator_x_plus_ay"]
    ndf1, ndf2 = g["ndf1"], g["ndf2"]
    x = np.array([[g["x"][j]] * ndf1 for j in range(ndf2)]).ravel()  # Fortran (1, ndf1, ndf2)
    y = np.array([[g["y"][j]] * ndf1 for j in range(ndf2)]).ravel()
    out = orc.operator_x_plus_ay(x, g["a"], y, 1, 1, ndf1, ndf2).reshape(ndf2, ndf1)
    for j in range(ndf2):
        assert np.all(np.abs(out[j] - g["answer"][j]) <= g["tol"])
